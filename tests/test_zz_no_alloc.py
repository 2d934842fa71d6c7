"""The static-scratch apply (giem2g_apply_ie_operator_device_static) through the C ABI.

It must give the regular device apply's result (same tolerances as the apply parity tests:
complex128 1e-12, complex64 2e-5 relative) on consecutive calls, allocate no device memory,
and reject grids whose intermediates do not fit its fixed array.  Collected last so it also
runs after every other GPU test in the same process.
"""
import ctypes

import numpy as np
import pytest

from giem2g_b200.synthetic import config_grf, config_small_block, csiga_from_sigma
from tests.helpers import random_vec, rel

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _op(g2, m, sig):
    op = g2.IEOperator.from_model(m)
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    op.calc_fft_of_ie_kernel()
    op.set_anomaly_conductivity(csiga_from_sigma(sig, m.freq))
    return op


def _static(g2, op, x, y, prec):
    return g2.lib().giem2g_apply_ie_operator_device_static(ctypes.c_void_p(op.handle), ctypes.c_void_p(x.data_ptr()),
                                                           ctypes.c_void_p(y.data_ptr()), prec)


@pytest.mark.parametrize("prec", [0, 1])
def test_static_apply_matches_device_apply(g2lib, orc, prec):
    """Two calls in a row against the regular device apply and against the oracle's apply of the same
    spectral tensor; the operator's apply counter counts the static calls too."""
    import torch
    m, sig = config_small_block()
    op = _op(g2lib, m, sig)
    sh, ah = op.get_ie_kernel_spectral()
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    dt = torch.complex128 if prec == 0 else torch.complex64
    tol = TOL64 if prec == 0 else TOL32
    vs = [random_vec(m, s) for s in (11, 12)]
    n0 = g2lib.lib().giem2g_apply_count(ctypes.c_void_p(op.handle))
    for v in vs:  # two calls in a row, different inputs
        x = torch.from_numpy(v.ravel()).to("cuda", dt)
        ref = torch.empty_like(x)
        got = torch.full_like(x, complex(np.nan, np.nan))
        op.apply_device(x.data_ptr(), ref.data_ptr(), prec)
        rc = _static(g2lib, op, x, got, prec)
        assert rc == 0, g2lib.lib().giem2g_last_error()
        op.check_device_error()
        torch.cuda.synchronize()
        got_np = got.cpu().numpy().astype(np.complex128)
        assert rel(got_np, ref.cpu().numpy().astype(np.complex128)) < tol
        want = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v)
        assert rel(got_np.reshape(want.shape), want) < tol
    assert g2lib.lib().giem2g_apply_count(ctypes.c_void_p(op.handle)) - n0 == 4
    op.delete()


def test_static_apply_allocates_nothing(g2lib):
    import torch
    m, sig = config_small_block()
    op = _op(g2lib, m, sig)
    x = torch.from_numpy(random_vec(m, 5).ravel()).to("cuda")
    y1, y2 = torch.empty_like(x), torch.empty_like(x)
    assert _static(g2lib, op, x, y1, 0) == 0  # first call on the device: set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _static(g2lib, op, x, y2, 0) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.equal(y1, y2)
    op.delete()


def test_static_apply_rejects_large_grid(g2lib):
    import torch
    # 64x64x32: 18*Nx*Ny*Nz complex = 37.7 MB at complex128 (rejected), 18.9 MB at complex64 (fits)
    m, sig = config_grf(64, 64, 32, seed=3)
    op = _op(g2lib, m, sig)
    x64 = torch.from_numpy(random_vec(m, 7).ravel()).to("cuda")
    y64 = torch.zeros_like(x64)
    rc = _static(g2lib, op, x64, y64, 0)
    assert rc == -1 and g2lib.lib().giem2g_last_status() == -1
    assert b"static maximum" in g2lib.lib().giem2g_last_error()
    torch.cuda.synchronize()
    assert not torch.any(y64 != 0)
    x32 = x64.to(torch.complex64)
    ref, got = torch.empty_like(x32), torch.empty_like(x32)
    op.apply_device(x32.data_ptr(), ref.data_ptr(), 1)
    assert _static(g2lib, op, x32, got, 1) == 0
    op.check_device_error()
    torch.cuda.synchronize()
    assert rel(got.cpu().numpy(), ref.cpu().numpy()) < TOL32
    op.delete()
