"""The fused y-pass (forward y-FFT, contraction and inverse y-FFT in one persistent kernel, csrc/ypipe.cu)
against the separate passes and the oracle.

The fused kernel sums in the same order as the stand-alone contraction whose slice count and arithmetic
form it shares (FP64: k_contract_wl SL = 4, variant 5; complex64: SL = 2 packed, variant 21; paired
complex64: SL = 2 packed, variant 14), and its transforms are the same four-step FFTs as k_fy / k_by, so
the two paths agree exactly.  Grids cover one batch of kx pairs (Nx = 4), several batches, the benchmark's
128x128x32 and Ny from 32 to 256.  The oracle bound is the apply tolerance (1e-12 FP64, 2e-5 complex64).
"""
import numpy as np
import pytest

from giem2g_b200.synthetic import csiga_from_sigma
from tests.helpers import random_sigma, random_spatial_tensor, random_vec, rel, tiny_model

pytestmark = pytest.mark.gpu

# stand-alone contraction variants with the fused kernel's summation order, per form
MATCH = {0: 5, 1: 21, 2: 14}


def _op(g2, m, seed=11):
    symm, asym = random_spatial_tensor(m, seed=seed)
    op = g2.IEOperator.from_model(m)
    op.set_background(m.csigma, m.thick, m.omega)
    op.set_ie_kernel_spatial(symm, asym)
    op.calc_fft_of_ie_kernel()
    sig = random_sigma(m, 4)
    csiga = csiga_from_sigma(sig, m.freq)
    op.set_anomaly_conductivity(csiga)
    return op, symm, asym, csiga


def _run(g2, op, vs, form, dt):
    import torch
    xs = [torch.from_numpy(v.ravel()).to("cuda", dt) for v in vs]
    ys = [torch.full_like(x, complex(np.nan, np.nan)) for x in xs]
    if form == 2:
        g2.apply_device_batch(op, [x.data_ptr() for x in xs], [y.data_ptr() for y in ys], 1)
    else:
        op.apply_device(xs[0].data_ptr(), ys[0].data_ptr(), form)
    op.check_device_error()
    return [y.cpu().numpy() for y in ys[: (2 if form == 2 else 1)]]


@pytest.mark.parametrize("shape", [(4, 32, 32), (8, 64, 32), (32, 32, 32), (16, 128, 32), (128, 128, 32),
                                   (4, 256, 32)])
def test_fused_equals_separate_passes_and_oracle(g2lib, orc, shape):
    import torch
    m = tiny_model(*shape)
    op, symm, asym, csiga = _op(g2lib, m)
    n_sep = {f: op.contract_variants(f) - 2 for f in (0, 1, 2)}
    assert all(n > 0 for n in n_sep.values())  # the fused variants are offered at Nz = 32
    csigb, sqsigb = orc.background_cells(m)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    vs = [random_vec(m, s) for s in (41, 42)]
    refs = [orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v) for v in vs]
    for form, dt, tol in ((0, torch.complex128, 1e-12), (1, torch.complex64, 2e-5), (2, torch.complex64, 2e-5)):
        op.set_contract_variant(form, MATCH[form])
        sep = _run(g2lib, op, vs, form, dt)
        for fv in range(2):
            op.set_contract_variant(form, n_sep[form] + fv)
            fused = _run(g2lib, op, vs, form, dt)
            for a, b, ref in zip(fused, sep, refs):
                assert np.array_equal(a, b), (form, fv, float(np.abs(a - b).max()))
                assert rel(a.astype(np.complex128).reshape(ref.shape), ref) < tol, (form, fv)
    op.delete()


def test_fused_apply_launches_three_kernels(g2lib):
    import torch
    m = tiny_model(32, 32, 32)
    op, *_ = _op(g2lib, m)
    x = torch.from_numpy(random_vec(m, 5).ravel()).to("cuda")
    y = torch.empty_like(x)
    op.set_contract_variant(0, op.contract_variants(0) - 2)  # the fused pass, variant 0
    n0 = g2lib.kernel_launch_count()
    op.apply_device(x.data_ptr(), y.data_ptr(), 0)
    assert g2lib.kernel_launch_count() - n0 == 3 and op.last_kernel_launches() == 3
    op.set_contract_variant(0, MATCH[0])  # the separate passes
    n0 = g2lib.kernel_launch_count()
    op.apply_device(x.data_ptr(), y.data_ptr(), 0)
    assert g2lib.kernel_launch_count() - n0 == 5 and op.last_kernel_launches() == 5
    op.delete()


def test_fused_apply_repeats_exactly(g2lib):
    """Many consecutive fused applies (counters zeroed per launch, dynamic work grabbing) give the same bits."""
    import torch
    m = tiny_model(64, 64, 32)
    op, *_ = _op(g2lib, m)
    op.set_contract_variant(1, op.contract_variants(1) - 2)  # the fused pass, variant 0
    x = torch.from_numpy(random_vec(m, 6).ravel()).to("cuda", torch.complex64)
    y0, y = torch.empty_like(x), torch.empty_like(x)
    op.apply_device(x.data_ptr(), y0.data_ptr(), 1)
    for _ in range(20):
        op.apply_device(x.data_ptr(), y.data_ptr(), 1)
    op.check_device_error()
    assert torch.equal(y, y0)
    op.delete()
