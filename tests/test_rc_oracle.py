"""Receiver continuation in the oracle: checks that do not need the GPU.

The reference ships no fields at receivers to compare with, so the restatement is pinned by physics
and by the independently pinned IE tensor:
  * far from a source cell, the receiver tensor (point value, single lateral integral) agrees with the IE
    tensor (cell average, double lateral integral) divided by the receiver cell's thickness, when the two
    receivers at the top and bottom of that cell are averaged (second order in cell size / distance);
  * the H tensor is the curl of the E tensor over i*omega*mu0 (Faraday's law), checked with Richardson-
    extrapolated central differences of receiver shifts;
  * the FFT route of ReCalculation equals the direct lag sums;
  * PlaneWave at points integrates to PlaneWaveIntegral over a cell, and its H is dE/dz / (i omega mu0).
"""
import numpy as np
import pytest

from giem2g_b200.synthetic import IEModel, THREE_LAYER_SIGMA, THREE_LAYER_THICK
from tests.helpers import random_vec, rel, tiny_model

XX, XY, XZ, YY, YZ, ZX, ZY, ZZ = range(8)
HXX, HXY, HXZ, HYX, HYZ, HZX, HZY = range(8, 15)


def _model(Nx, Ny, freq=1.0):
    z = np.array([100.0, 150.0, 200.0, 250.0])
    return IEModel(Nx, Ny, 3, 50.0, 50.0, z, THREE_LAYER_SIGMA.copy(), THREE_LAYER_THICK.copy(), freq)


def test_prepare_receivers(orc):
    m = tiny_model(4, 4, 4)  # z borders 0, 30, 73.3, 130, 200
    rv = orc.prepare_receivers(m, [-5.0, 0.0, 30.0, 50.0, 200.0, 700.0])
    assert list(rv.anom_cell) == [0, 0, 1, 1, 5, 5]
    assert rv.zrecv[3] == 30.0  # moved to the top of its cell
    assert list(rv.recv_layer) == [1, 1, 1, 1, 1, 2]


def test_single_int_weights_finite(orc):
    rmin = np.hypot(50.0, 50.0) / 2
    WT, lms = orc.vbt_weights_single(-25.0, 125.0, 50.0, 50.0, rmin)
    assert np.all(np.isfinite(WT)) and np.all(np.diff(lms) > 0)
    assert np.abs(WT).max() > 0


def test_far_field_matches_ie_tensor(orc):
    m = _model(16, 2)
    S, A = orc.green_tensor(m)
    rv = orc.prepare_receivers(m, [150.0, 200.0])  # top and bottom of cell 1
    G = orc.rc_tensor(m, rv)
    lx, ly, zr = 10, 0, 1

    def pk(i, j):
        i, j = min(i, j), max(i, j)
        return i + j * (j + 1) // 2

    for zs in range(3):
        rc = 0.5 * (G[ly, lx, :, 0, zs] + G[ly, lx, :, 1, zs])
        ie_xx = S[lx, ly, 0, pk(zr, zs)] / m.dz[zr]
        ie_zz = S[lx, ly, 3, pk(zr, zs)] / m.dz[zr]
        ie_xz = A[lx, ly, 0, zs * m.Nz + zr] / m.dz[zr]  # G_asym(Izr, Izs), column-major
        ie_zx = -A[lx, ly, 0, zr * m.Nz + zs] / m.dz[zr]
        assert abs(rc[XX] - ie_xx) < 0.01 * abs(ie_xx)
        assert abs(rc[ZZ] - ie_zz) < 0.03 * abs(ie_zz)
        assert abs(rc[XZ] - ie_xz) < 0.02 * abs(ie_xz)
        assert abs(rc[ZX] - ie_zx) < 0.05 * abs(ie_zx)


def _curl_vs_h(orc, m, h, z0, lag, zc):
    zs = [z0, z0, z0, z0, z0 - h, z0 + h, z0]
    xs = [-h, h, 0, 0, 0, 0, 0]
    ys = [0, 0, -h, h, 0, 0, 0]
    rv = orc.prepare_receivers(m, zs, xs, ys)
    g = orc.rc_tensor(m, rv)[lag[1], lag[0], :, :, zc]
    iwm = 1j * orc.mu0() * m.omega
    Es = [np.array([g[XX], g[XY], g[ZX]]), np.array([g[XY], g[YY], g[ZY]]), np.array([g[XZ], g[YZ], g[ZZ]])]
    Hs = [np.array([g[HXX], g[HYX], g[HZX]]), np.array([g[HXY], -g[HXX], g[HZY]]),
          np.array([g[HXZ], g[HYZ], 0 * g[HXX]])]
    out = []
    for e, hh in zip(Es, Hs):
        dx = (e[:, 1] - e[:, 0]) / (2 * h)
        dy = (e[:, 3] - e[:, 2]) / (2 * h)
        dz = (e[:, 5] - e[:, 4]) / (2 * h)
        out.append((np.array([dy[2] - dz[1], dz[0] - dx[2], dx[1] - dy[0]]) / iwm, hh[:, 6]))
    return out


@pytest.mark.parametrize("z0,lag,zc", [(50.0, (3, 2), 1), (400.0, (-2, 1), 0)])
def test_h_tensor_is_curl_of_e_tensor(orc, z0, lag, zc):
    m = _model(8, 8)
    a, b = _curl_vs_h(orc, m, 1.0, z0, lag, zc), _curl_vs_h(orc, m, 0.5, z0, lag, zc)
    for (c1, H), (c2, _) in zip(a, b):
        ex = (4 * c2 - c1) / 3  # Richardson: O(h^4)
        assert np.abs(ex - H).max() < 1e-5 * np.abs(H).max()


def test_fft_route_equals_direct_sums(orc):
    m = tiny_model(6, 4, 3)
    rv = orc.prepare_receivers(m, [0.0, 73.0, 500.0], [0.0, 20.0, -10.0], [5.0, 0.0, 0.0])
    G = orc.rc_tensor(m, rv)
    rng = np.random.default_rng(5)
    csiga = rng.uniform(0.01, 1.0, (m.Nz, m.Ny, m.Nx)) - 1e-8j
    csigb, _ = orc.background_cells(m)
    E = random_vec(m, 9)
    Ea, Ha = orc.rc_apply(m.Nx, m.Ny, m.Nz, G, csiga, csigb, E)
    Ea2, Ha2 = orc.rc_apply(m.Nx, m.Ny, m.Nz, G, csiga, csigb, E, direct=True)
    assert rel(Ea, Ea2) < 1e-13 and rel(Ha, Ha2) < 1e-13


def test_plane_wave_points_consistent_with_cell_integral(orc):
    m = tiny_model(2, 2, 4, freq=3.0)
    E0 = orc.plane_wave(m, 0)
    iwm = 1j * orc.mu0() * m.omega
    for iz in range(m.Nz):
        zz = np.linspace(m.z[iz], m.z[iz + 1], 401)
        F = orc.plane_wave_points(m, 0, zz)
        avg = np.trapezoid(F[:, 0], zz) / (m.z[iz + 1] - m.z[iz])
        assert abs(avg - E0[0, iz, 0, 0]) < 1e-6 * abs(E0[0, iz, 0, 0])
        dEdz = np.gradient(F[:, 0], zz)
        assert abs(dEdz[200] / iwm - F[200, 4]) < 1e-4 * abs(F[200, 4])
    Fy = orc.plane_wave_points(m, 1, [0.0, 250.0])
    Fx = orc.plane_wave_points(m, 0, [0.0, 250.0])
    assert np.allclose(Fy[:, 1], Fx[:, 0]) and np.allclose(Fy[:, 3], -Fx[:, 4])
    assert abs(Fx[0, 0] - 1.0) < 1e-12
