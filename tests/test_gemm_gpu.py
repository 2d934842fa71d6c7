"""tcgen05 BF16 GEMM (FP32 accumulation) against a plain PyTorch FP32 matmul of the same BF16 inputs."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (256, 64, 128), (300, 48, 200), (1000, 128, 1728), (77, 16, 8),
                                   (4096, 64, 448)])
def test_gemm_matches_fp32_reference(g2lib, M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    C = g2lib.gemm_bf16_tn(A, B, err=err)
    ref = A.float() @ B.float().t()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rel = (C - ref).norm() / ref.norm()
    assert rel < 1e-5, float(rel)
    # accumulate into an existing C
    C2 = g2lib.gemm_bf16_tn(A, B, C=C.clone(), accumulate=True, err=err)
    torch.cuda.synchronize()
    assert ((C2 - 2 * ref).norm() / (2 * ref).norm()) < 1e-5


def test_gemm_rejects_bad_shapes(g2lib):
    import torch
    A = torch.zeros(16, 12, dtype=torch.bfloat16, device="cuda")
    B = torch.zeros(16, 12, dtype=torch.bfloat16, device="cuda")
    with pytest.raises(g2lib.Giem2gError):
        g2lib.gemm_bf16_tn(A, B)
