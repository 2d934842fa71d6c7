"""Host pieces of the learned preconditioner's training data (no GPU): the operator system that the
Krylov-history pairs are built in must be SolveEquation's (ie_solver_module.F90:62-80), checked against the
oracle's background cells."""
import numpy as np
import pytest


def test_operator_system_matches_oracle_background(orc, monkeypatch):
    torch = pytest.importorskip("torch")
    from giem2g_b200 import learned
    from giem2g_b200.sources import plane_wave_integral
    from giem2g_b200.synthetic import config_c4, csiga_from_sigma
    monkeypatch.setattr(torch.Tensor, "cuda", lambda self, *a, **k: self)  # keep it on the CPU
    m, sig = config_c4(seed=3)
    E0 = plane_wave_integral(m, 1)
    a, rhs = learned._operator_system(m, sig, E0)
    csigb, sqsigb = orc.background_cells(m)
    csiga = csiga_from_sigma(sig, m.freq)
    a_ref = 2.0 * sqsigb[:, None, None] / (csiga + np.conj(csigb)[:, None, None])
    assert np.allclose(a.numpy(), a_ref, rtol=1e-14, atol=0)
    assert np.allclose(rhs.numpy(), sqsigb[None, :, None, None] * E0, rtol=1e-14, atol=0)
