"""GPU parity of the IE operator apply and the tensor spectral transform against the CPU oracle.

Tolerances: complex128 path <= 1e-12 relative (2-norm over the whole vector); complex64 path
<= 2e-5 relative.  Calls go through the C ABI (giem2g_apply_ie_operator and the device variant).
"""
import numpy as np
import pytest

from tests.helpers import random_sigma, random_spatial_tensor, random_vec, rel, tiny_model
from giem2g_b200.synthetic import config_small_block, csiga_from_sigma

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _setup(g2, orc, m, symm, asym, sig):
    op = g2.IEOperator.from_model(m)
    op.set_background(m.csigma, m.thick, m.omega)
    op.set_ie_kernel_spatial(symm, asym)
    op.calc_fft_of_ie_kernel()
    csiga = csiga_from_sigma(sig, m.freq)
    op.set_anomaly_conductivity(csiga)
    csigb, sqsigb = orc.background_cells(m)
    return op, csiga, csigb, sqsigb


@pytest.mark.parametrize("shape", [(2, 2, 1), (4, 4, 3), (8, 4, 5), (4, 16, 2), (16, 8, 7), (4, 4, 8), (8, 4, 16),
                                   (4, 4, 32), (2, 4, 48)])
def test_spectrum_and_apply_random_tensor(g2lib, orc, shape):
    m = tiny_model(*shape)
    symm, asym = random_spatial_tensor(m)
    sig = random_sigma(m)
    op, csiga, csigb, sqsigb = _setup(g2lib, orc, m, symm, asym, sig)
    sh_o, ah_o = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    sh_g, ah_g = op.get_ie_kernel_spectral()
    assert rel(sh_g, sh_o) < TOL64
    assert rel(ah_g, ah_o) < TOL64
    v = random_vec(m)
    out_o = orc.apply(m.Nx, m.Ny, m.Nz, sh_o, ah_o, csiga, csigb, sqsigb, m.dz, v)
    out_t = orc.apply_toeplitz(m.Nx, m.Ny, m.Nz, symm, asym, csiga, csigb, sqsigb, m.dz, v)
    assert rel(out_o, out_t) < 1e-13
    out_g = op.apply_precond(v)
    assert rel(out_g, out_o) < TOL64
    op.delete()


def test_apply_block_model_physical_tensor(g2lib, orc):
    m, sig = config_small_block()
    symm, asym = orc.green_tensor(m)
    op, csiga, csigb, sqsigb = _setup(g2lib, orc, m, symm, asym, sig)
    sh_o, ah_o = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    for seed in (1, 2):
        v = random_vec(m, seed)
        out_o = orc.apply(m.Nx, m.Ny, m.Nz, sh_o, ah_o, csiga, csigb, sqsigb, m.dz, v)
        out_g = op.apply_precond(v)
        assert rel(out_g, out_o) < TOL64
    op.delete()


def test_apply_complex64_device(g2lib, orc):
    import torch
    m, sig = config_small_block()
    symm, asym = orc.green_tensor(m)
    op, csiga, csigb, sqsigb = _setup(g2lib, orc, m, symm, asym, sig)
    sh_o, ah_o = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    v = random_vec(m, 5)
    out_o = orc.apply(m.Nx, m.Ny, m.Nz, sh_o, ah_o, csiga, csigb, sqsigb, m.dz, v)
    dv = torch.from_numpy(v.astype(np.complex64).ravel()).cuda()
    do = torch.empty_like(dv)
    torch.cuda.synchronize()
    op.apply_device(dv.data_ptr(), do.data_ptr(), precision=1)
    torch.cuda.synchronize()
    assert rel(do.cpu().numpy().reshape(v.shape), out_o) < TOL32
    dv64 = torch.from_numpy(v.ravel()).cuda()
    do64 = torch.empty_like(dv64)
    op.apply_device(dv64.data_ptr(), do64.data_ptr(), precision=0)
    torch.cuda.synchronize()
    assert rel(do64.cpu().numpy().reshape(v.shape), out_o) < TOL64
    assert op.last_kernel_launches() == 5
    op.delete()


def test_device_apply_follows_torch_stream(g2lib, orc):
    """A device-pointer apply waits for the torch work that wrote its input, and torch waits for its
    output.  Torch's stream spins for about 20 ms before it converts the input to complex64; the apply,
    issued at once on the operator's non-blocking stream, still reads the converted vector, and torch
    reads the result with no synchronisation in between."""
    import torch
    m, sig = config_small_block()
    symm, asym = orc.green_tensor(m)
    op, csiga, csigb, sqsigb = _setup(g2lib, orc, m, symm, asym, sig)
    sh_o, ah_o = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    v = random_vec(m, 7)
    out_o = orc.apply(m.Nx, m.Ny, m.Nz, sh_o, ah_o, csiga, csigb, sqsigb, m.dz, v)
    dv64 = torch.from_numpy(v.ravel()).cuda()
    torch.cuda.synchronize()
    torch.cuda._sleep(40_000_000)  # a bounded spin of 4e7 clock cycles on torch's current stream
    dv = dv64.to(torch.complex64)
    do = torch.empty_like(dv)
    op.apply_device(dv.data_ptr(), do.data_ptr(), precision=1)
    got = do.cpu().numpy()
    assert rel(got.reshape(v.shape), out_o) < TOL32
    op.delete()


@pytest.mark.parametrize("shape", [(4, 4, 8), (8, 4, 16), (4, 4, 32), (2, 4, 48)])
def test_complex64_specialised_and_generic_contraction(g2lib, orc, shape, monkeypatch):
    """complex64 path for the specialised Nz kernels and the generic kernel give the oracle's result."""
    import torch
    m = tiny_model(*shape)
    symm, asym = random_spatial_tensor(m)
    sig = random_sigma(m)
    sh_o, ah_o = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    csigb, sqsigb = orc.background_cells(m)
    v = random_vec(m, 9)
    csiga = csiga_from_sigma(sig, m.freq)
    out_o = orc.apply(m.Nx, m.Ny, m.Nz, sh_o, ah_o, csiga, csigb, sqsigb, m.dz, v)
    for generic in ("0", "1"):
        monkeypatch.setenv("GIEM2G_GENERIC_CONTRACT", generic)
        op, *_ = _setup(g2lib, orc, m, symm, asym, sig)
        dv = torch.from_numpy(v.astype(np.complex64).ravel()).cuda()
        do = torch.empty_like(dv)
        op.apply_device(dv.data_ptr(), do.data_ptr(), precision=1)
        op.check_device_error()
        assert rel(do.cpu().numpy().reshape(v.shape), out_o) < TOL32
        dv64 = torch.from_numpy(v.ravel()).cuda()
        do64 = torch.empty_like(dv64)
        op.apply_device(dv64.data_ptr(), do64.data_ptr(), precision=0)
        op.check_device_error()
        assert rel(do64.cpu().numpy().reshape(v.shape), out_o) < TOL64
        op.delete()


def test_precision_mode_of_the_host_apply_and_solve(g2lib, orc):
    """giem2g_set_precision: mode 1 makes the reference-facing apply run in complex64 (within the complex64
    tolerance of the oracle, and not the FP64 result), and solves with precision -1 follow the mode."""
    m = tiny_model(8, 8, 8)
    symm, asym = random_spatial_tensor(m, seed=5)
    sig = random_sigma(m, 6)
    op, csiga, csigb, sqsigb = _setup(g2lib, orc, m, symm, asym, sig)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    v = random_vec(m, 7)
    ref = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v)
    y64 = op.apply_precond(v)
    op.set_precision(1)
    y32 = op.apply_precond(v)
    assert rel(y64, ref) < TOL64
    assert rel(y32, ref) < TOL32 and rel(y32, ref) > 1e-10
    op.set_precision(0)
    assert rel(op.apply_precond(v), ref) < TOL64
    with pytest.raises(g2lib.Giem2gError):
        op.set_precision(2)
    op.delete()
    # solves: precision -1 takes the operator's mode
    mb, sgb = config_small_block()
    op = g2lib.IEOperator.from_model(mb)
    op.calc_ie_kernel(mb.csigma, mb.thick, mb.omega)
    op.calc_fft_of_ie_kernel()
    op.set_anomaly_sigma(sgb, mb.freq)
    from giem2g_b200.sources import plane_wave_integral
    E0 = plane_wave_integral(mb, 1)
    _, i1 = op.solve_equation(E0, tol=1e-6, precision=1)
    op.set_precision(1)
    _, im = op.solve_equation(E0, tol=1e-6, precision=-1)
    assert im.applies_fp32 > 0 and im.iterations == i1.iterations and im.applies_fp32 == i1.applies_fp32
    op.set_precision(0)
    _, i0 = op.solve_equation(E0, tol=1e-6, precision=-1)
    assert i0.applies_fp32 == 0
    op.delete()
