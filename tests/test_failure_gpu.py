"""Failure detection without a GPU fault: bad inputs are injected on the host and the statuses checked,
and the bounded-wait mechanism is made to run out on purpose (a wait that nothing completes), after which
the same process keeps using the GPU."""
import time

import numpy as np
import pytest

from giem2g_b200.sources import plane_wave_integral
from giem2g_b200.synthetic import config_small_block

pytestmark = pytest.mark.gpu


def _op(g2):
    m, sig = config_small_block()
    op = g2.IEOperator.from_model(m)
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    op.calc_fft_of_ie_kernel()
    op.set_anomaly_sigma(sig, m.freq)
    return m, op


def test_bounded_wait_ends_with_error_status(g2lib):
    t0 = time.perf_counter()
    code = g2lib.lib().giem2g_selftest_bounded_wait(200)
    dt = time.perf_counter() - t0
    assert code == 77
    assert 0.15 < dt < 30.0
    # the context is still usable
    m, op = _op(g2lib)
    E, info = op.solve_equation(plane_wave_integral(m, 1), tol=1e-8)
    assert info.stat == 1
    op.delete()


@pytest.mark.parametrize("precision", [0, 1])
def test_nan_right_hand_side_reports_numeric_status(g2lib, precision):
    m, op = _op(g2lib)
    E0 = plane_wave_integral(m, 0)
    bad = E0.copy()
    bad[0, 1, 2, 3] = np.nan
    with pytest.raises(g2lib.Giem2gError, match="status -5"):
        op.solve_equation(bad, tol=1e-8, precision=precision)
    E, info = op.solve_equation(E0, tol=1e-8, precision=precision)  # the operator recovers
    assert info.stat == 1
    op.delete()


def test_corrupt_tensor_reports_numeric_status(g2lib):
    m, sig = config_small_block()
    op = g2lib.IEOperator.from_model(m)
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    S, A = op.get_ie_kernel_spatial()  # the spectral transform works in place: take the spatial tensor first
    op.set_anomaly_sigma(sig, m.freq)
    Sb = S.copy()
    Sb[1, 2, 0, 3] = np.inf
    op.set_ie_kernel_spatial(Sb, A)
    op.calc_fft_of_ie_kernel()
    with pytest.raises(g2lib.Giem2gError, match="status -5"):
        op.solve_equation(plane_wave_integral(m, 1), tol=1e-8)
    op.set_ie_kernel_spatial(S, A)
    op.calc_fft_of_ie_kernel()
    E, info = op.solve_equation(plane_wave_integral(m, 1), tol=1e-8)
    assert info.stat == 1
    op.delete()
