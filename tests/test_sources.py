"""Plane-wave right-hand side of the product (giem2g_b200.sources) against the oracle's restatement of
PlaneWaveIntegral (sources_module.F90:67-101)."""
import numpy as np
import pytest

from giem2g_b200.sources import plane_wave_integral
from giem2g_b200.synthetic import IEModel, THREE_LAYER_SIGMA, THREE_LAYER_THICK, config_small_block
from tests.helpers import rel


def _models():
    m, _ = config_small_block()
    yield m
    yield IEModel(4, 4, 8, 70.0, 130.0, 100.0 + np.arange(9) * 60.0, THREE_LAYER_SIGMA.copy(),
                  THREE_LAYER_THICK.copy(), 0.3)
    yield IEModel(2, 2, 3, 50.0, 50.0, np.array([0.0, 10.0, 30.0, 70.0]), np.array([0.05]), np.array([]), 3.0)
    yield IEModel(2, 2, 6, 50.0, 50.0, np.arange(7) * 400.0, np.array([0.1, 0.01, 10.0]), np.array([1000.0, 2000.0]), 0.001)


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("pol", [0, 1])
def test_plane_wave_matches_oracle(orc, idx, pol):
    m = list(_models())[idx]
    ref = orc.plane_wave(m, pol)
    got = plane_wave_integral(m, pol)
    assert rel(got, ref) < 1e-13
    assert np.count_nonzero(got[1 - pol]) == 0 and np.count_nonzero(got[2]) == 0
