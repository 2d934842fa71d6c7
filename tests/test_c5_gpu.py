"""The largest configuration (256x256x48 cells of 25x25x20 m, a seeded lognormal field with three 1 S/m
ellipsoids, 0.01 Hz): size-independent properties of the GPU operator on the full grid, where the CPU oracle
would take minutes per apply.

* the FP64 apply is linear: A(a x + b y) = a A x + b A y to 1e-12 relative;
* the complex64 apply and the paired complex64 apply (two vectors per tensor read, every paired tile shape)
  agree with the FP64 apply on the same vectors to 2e-5, the complex64 apply tolerance;
* a mixed-precision batched solve of both polarisations converges to outer relative residual 1e-6 (the
  solver's FP64 true residual), and its EY field lies within 1e-5 of an FP64 solve at tolerance 1e-8.
The same operator code is checked against the oracle on the smaller grids (test_apply_gpu, test_variants_gpu,
test_fullsize_gpu).
"""
import numpy as np
import pytest

from giem2g_b200.sources import plane_wave_integral
from giem2g_b200.synthetic import config_c5
from tests.helpers import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c5(g2lib):
    m, sig = config_c5(seed=5)
    op = g2lib.IEOperator.from_model(m)
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    op.calc_fft_of_ie_kernel()
    op.set_anomaly_sigma(sig, m.freq)
    yield m, op
    op.delete()


def _apply(op, x, prec):
    import torch
    y = torch.empty_like(x)
    op.apply_device(x.data_ptr(), y.data_ptr(), prec)
    op.check_device_error()
    return y


def test_c5_fp64_apply_linear(c5):
    import torch
    m, op = c5
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(op.nvec, dtype=torch.complex128, device="cuda", generator=g)
    y = torch.randn(op.nvec, dtype=torch.complex128, device="cuda", generator=g)
    a, b = 0.7 - 0.2j, -1.3 + 0.5j
    lhs = _apply(op, a * x + b * y, 0)
    rhs = a * _apply(op, x, 0) + b * _apply(op, y, 0)
    assert rel(lhs.cpu().numpy(), rhs.cpu().numpy()) < 1e-12


def test_c5_complex64_and_paired_applies(c5, g2lib):
    import torch
    m, op = c5
    g = torch.Generator(device="cuda").manual_seed(6)
    xs = [torch.randn(op.nvec, dtype=torch.complex128, device="cuda", generator=g) for _ in range(2)]
    ref = [_apply(op, x, 0).cpu().numpy() for x in xs]
    x32 = [x.to(torch.complex64) for x in xs]
    got = _apply(op, x32[0], 1).cpu().numpy()
    assert rel(got.astype(np.complex128), ref[0]) < 2e-5
    for var in range(op.contract_variants(2)):
        op.set_contract_variant(2, var)
        ys = [torch.empty_like(x) for x in x32]
        g2lib.apply_device_batch(op, [x.data_ptr() for x in x32], [y.data_ptr() for y in ys], 1)
        op.check_device_error()
        for y, r in zip(ys, ref):
            assert rel(y.cpu().numpy().astype(np.complex128), r) < 2e-5, ("pair", var)


def test_c5_mixed_batched_solve(c5, g2lib):
    import torch
    m, op = c5
    tol = 1e-6
    rhs = [torch.from_numpy(np.ascontiguousarray(plane_wave_integral(m, p)).ravel()).to("cuda") for p in (1, 0)]
    sol = [torch.empty_like(x) for x in rhs]
    b = g2lib.Batch([op, op], precision=1)
    infos = b.solve_device([x.data_ptr() for x in rhs], [y.data_ptr() for y in sol], tol=tol)
    torch.cuda.synchronize()
    b.delete()
    for info, e in zip(infos, sol):
        assert info.stat == 1 and info.be < tol and 0 < info.iterations < 100
    ref = torch.empty_like(rhs[0])
    info64 = op.solve_device(rhs[0].data_ptr(), ref.data_ptr(), None, tol=1e-8, precision=0)
    assert info64.stat == 1
    assert rel(sol[0].cpu().numpy(), ref.cpu().numpy()) < 1e-5
