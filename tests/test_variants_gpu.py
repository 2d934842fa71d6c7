"""Every contraction tile variant (FP64, complex64, paired complex64) against the oracle apply.

The autotuner may pick any variant, so each one must meet the apply tolerances: 1e-12 (complex128) and
2e-5 (complex64) relative to the oracle.  The small grids give each persistent CTA at most one unit; the
larger ones (thousands of units over the SMs) run every stage ring through many rounds, the steady state
of the benchmark grid.
"""
import numpy as np
import pytest

from giem2g_b200.synthetic import csiga_from_sigma
from tests.helpers import random_sigma, random_spatial_tensor, random_vec, rel, tiny_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(8, 8, 8), (4, 8, 16), (4, 4, 32), (2, 4, 48),
                                   (128, 64, 8), (64, 64, 16), (64, 32, 32), (32, 32, 48)])
def test_all_contraction_variants(g2lib, orc, shape):
    import torch
    m = tiny_model(*shape)
    symm, asym = random_spatial_tensor(m, seed=11)
    op = g2lib.IEOperator.from_model(m)
    op.set_background(m.csigma, m.thick, m.omega)
    op.set_ie_kernel_spatial(symm, asym)
    op.calc_fft_of_ie_kernel()
    sig = random_sigma(m, 4)
    csiga = csiga_from_sigma(sig, m.freq)
    op.set_anomaly_conductivity(csiga)
    csigb, sqsigb = orc.background_cells(m)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    vs = [random_vec(m, s) for s in (31, 32)]
    refs = [orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v) for v in vs]
    tried = 0
    for prec, dt, tol in ((0, torch.complex128, 1e-12), (1, torch.complex64, 2e-5)):
        for var in range(max(1, op.contract_variants(prec))):
            if op.contract_variants(prec):
                op.set_contract_variant(prec, var)
            x = torch.from_numpy(vs[0].ravel()).to("cuda", dt)
            y = torch.empty_like(x)
            op.apply_device(x.data_ptr(), y.data_ptr(), prec)
            op.check_device_error()
            got = y.cpu().numpy().astype(np.complex128).reshape(refs[0].shape)
            assert rel(got, refs[0]) < tol, (prec, var)
            tried += 1
    for var in range(op.contract_variants(2)):
        op.set_contract_variant(2, var)
        xs = [torch.from_numpy(v.ravel()).to("cuda", torch.complex64) for v in vs]
        ys = [torch.empty_like(x) for x in xs]
        g2lib.apply_device_batch(op, [x.data_ptr() for x in xs], [y.data_ptr() for y in ys], 1)
        op.check_device_error()
        for y, ref in zip(ys, refs):
            got = y.cpu().numpy().astype(np.complex128).reshape(ref.shape)
            assert rel(got, ref) < 2e-5, ("pair", var)
        tried += 1
    assert tried >= 3
    op.delete()
