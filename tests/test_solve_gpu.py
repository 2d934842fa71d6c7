"""GPU nested FGMRES (SolveEquation) against the CPU oracle's restatement of GFGMRES.

Plain mode (complex128 throughout): same outer iteration count, Arnoldi misfit history within 1e-6
relative, solution within 1e-9 relative.  Mixed mode (complex64 inner solver): converges to the
requested outer residual and the field matches the FP64 oracle solution within 10x the tolerance.
"""
import numpy as np
import pytest

from giem2g_b200.synthetic import config_small_block, csiga_from_sigma
from tests.helpers import rel, tiny_model, random_sigma

pytestmark = pytest.mark.gpu


def _prepare(g2, orc, m, sig):
    symm, asym = orc.green_tensor(m)
    op = g2.IEOperator.from_model(m)
    op.set_background(m.csigma, m.thick, m.omega)
    op.set_ie_kernel_spatial(symm, asym)
    op.calc_fft_of_ie_kernel()
    csiga = csiga_from_sigma(sig, m.freq)
    op.set_anomaly_conductivity(csiga)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, symm, asym)
    csigb, sqsigb = orc.background_cells(m)
    return op, sh, ah, csiga, csigb, sqsigb


@pytest.mark.parametrize("pol", [0, 1])
def test_solve_plain_matches_oracle(g2lib, orc, pol):
    m, sig = config_small_block()
    op, sh, ah, csiga, csigb, sqsigb = _prepare(g2lib, orc, m, sig)
    E0 = orc.plane_wave(m, pol)
    Eo, info_o, hist_o = orc.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, None, 30, 10, 100, 1e-8)
    Eg, info_g = op.solve_equation(E0, tol=1e-8, max_restart=100, outer_buf=30, inner_buf=10, precision=0)
    assert info_g.stat == info_o.stat == 1
    assert info_g.iterations == info_o.iterations
    assert np.allclose(info_g.misfits, hist_o, rtol=1e-6, atol=0)
    assert rel(Eg, Eo) < 1e-9
    assert abs(info_g.be - info_o.be) <= 1e-6 * info_o.be
    op.delete()


def test_solve_restarts_and_guess(g2lib, orc):
    """Small restart buffers force restarts (Arnoldi-residual restart); warm start through E0."""
    m = tiny_model(8, 8, 4, freq=10.0)
    sig = random_sigma(m, seed=4, lo=-2.5, hi=0.5)
    op, sh, ah, csiga, csigb, sqsigb = _prepare(g2lib, orc, m, sig)
    E0 = orc.plane_wave(m, 1)
    Eo, io, ho = orc.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, None, 3, 2, 50, 1e-10)
    Eg, ig = op.solve_equation(E0, tol=1e-10, max_restart=50, outer_buf=3, inner_buf=2, precision=0)
    assert ig.iterations == io.iterations and ig.stat == io.stat
    assert np.allclose(ig.misfits, ho, rtol=1e-5, atol=0)
    assert rel(Eg, Eo) < 1e-8
    # warm start from the solution: converges at once (beta/bn < tol)
    Eg2, ig2 = op.solve_equation(E0, E0=Eg, tol=1e-8, max_restart=50, outer_buf=3, inner_buf=2, precision=0)
    Eo2, io2, _ = orc.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, Eo, 3, 2, 50, 1e-8)
    assert ig2.iterations == io2.iterations == 0
    assert rel(Eg2, Eo2) < 1e-8
    op.delete()


def test_solve_nonconverged_status(g2lib, orc):
    """MaxRestart = 1 with a tiny basis stops early with NON_CONVERGED (-1), as the oracle does."""
    m, sig = config_small_block()
    op, sh, ah, csiga, csigb, sqsigb = _prepare(g2lib, orc, m, sig)
    E0 = orc.plane_wave(m, 0)
    _, io, _ = orc.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, None, 2, 1, 1, 1e-12)
    _, ig = op.solve_equation(E0, tol=1e-12, max_restart=1, outer_buf=2, inner_buf=1, precision=0)
    assert io.stat == ig.stat == -1
    assert ig.iterations == io.iterations == 2
    op.delete()


def test_solve_mixed_precision_field_error(g2lib, orc):
    m, sig = config_small_block()
    op, sh, ah, csiga, csigb, sqsigb = _prepare(g2lib, orc, m, sig)
    E0 = orc.plane_wave(m, 1)
    Eo, io, _ = orc.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, None, 30, 10, 100, 1e-8)
    Eg, ig = op.solve_equation(E0, tol=1e-6, max_restart=100, outer_buf=30, inner_buf=10, precision=1)
    assert ig.stat == 1 and ig.be < 1e-6
    assert ig.applies_fp32 > 0
    assert rel(Eg, Eo) < 1e-5
    op.delete()
