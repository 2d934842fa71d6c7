"""CPU tests of the oracle itself (the checker the GPU path is compared with).

The reference has no tests or golden vectors and cannot be built here, so the oracle is pinned by
independent means:
  * the FFT-based apply (the reference's spectral algorithm with its +-kx slots, MirrorY rows and
    Nyquist corrections) equals a dense block-Toeplitz brute force of the same operator;
  * an independent numpy restatement of the spectral apply (numpy FFTs, explicit 3Nz x 3Nz blocks);
  * an independent numpy restatement of one tensor lag (apq/shell recursion over lambda);
  * the plane-wave RHS against the analytic half-space average of exp(-eta z);
  * FGMRES: the returned solution satisfies the system to the reported residual;
  * the committed golden fixtures (tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from giem2g_b200.synthetic import IEModel, THREE_LAYER_SIGMA, THREE_LAYER_THICK, config_small_block, csiga_from_sigma
from tests.helpers import random_sigma, random_spatial_tensor, random_vec, rel, tiny_model

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("shape", [(2, 2, 1), (4, 4, 3), (8, 4, 5), (6, 4, 3), (4, 8, 2), (3, 5, 2)])
def test_fft_apply_equals_block_toeplitz(orc, shape):
    m = tiny_model(*shape)
    S, A = random_spatial_tensor(m)
    sig = random_sigma(m)
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, S, A)
    v = random_vec(m)
    a = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v)
    b = orc.apply_toeplitz(m.Nx, m.Ny, m.Nz, S, A, csiga, csigb, sqsigb, m.dz, v)
    if shape[0] % 2 == 0 and shape[1] % 2 == 0:
        assert rel(a, b) < 1e-13
    else:  # odd sizes: the reference's Nyquist correction is not exact there (documented)
        assert rel(a, b) < 1.0


def test_fft_apply_equals_toeplitz_physical_tensor(orc):
    m = tiny_model(8, 4, 4, freq=3.0)
    S, A = orc.green_tensor(m)
    sig = random_sigma(m, 5)
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, S, A)
    v = random_vec(m, 3)
    a = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v)
    b = orc.apply_toeplitz(m.Nx, m.Ny, m.Nz, S, A, csiga, csigb, sqsigb, m.dz, v)
    assert rel(a, b) < 1e-13


def _np_apply(m, S, A, csiga, csigb, sqsigb, v):
    """Independent numpy statement: zero-padded 2-D FFT, parity-extended kernel FFT, explicit blocks."""
    Nx, Ny, Nz = m.Nx, m.Ny, m.Nz
    P = Nz * (Nz + 1) // 2
    n1, n2 = 2 * Nx, 2 * Ny
    # full spatial kernel K[c_out, c_in, z, z', ly_ext, lx_ext]
    def full_sym(p):
        M = np.zeros((Nz, Nz), complex)
        for j in range(Nz):
            for i in range(j + 1):
                M[i, j] = M[j, i] = p[i + j * (j + 1) // 2]
        return M
    K = np.zeros((3, 3, Nz, Nz, n2, n1), complex)
    for lx in range(-(Nx - 1), Nx):
        for ly in range(-(Ny - 1), Ny):
            ax, ay = abs(lx), abs(ly)
            sx, sy = (-1.0 if lx < 0 else 1.0), (-1.0 if ly < 0 else 1.0)
            gs = [full_sym(S[ax, ay, c]) for c in range(4)]
            gxz = A[ax, ay, 0].reshape(Nz, Nz).T * sx   # [row z][col z']
            gyz = A[ax, ay, 1].reshape(Nz, Nz).T * sy
            blk = K[:, :, :, :, ly % n2, lx % n1]
            blk[0, 0] = gs[0]
            blk[0, 1] = blk[1, 0] = gs[1] * sx * sy
            blk[1, 1] = gs[2]
            blk[2, 2] = gs[3]
            blk[0, 2] = gxz
            blk[1, 2] = gyz
            blk[2, 0] = -gxz.T
            blk[2, 1] = -gyz.T
    Kh = np.fft.fft2(K, axes=(4, 5))
    a = 2.0 * sqsigb[:, None, None] / (csiga + np.conj(csigb)[:, None, None])
    g = (csiga - csigb[:, None, None]) * a
    u = np.zeros((3, Nz, n2, n1), complex)
    u[:, :, :Ny, :Nx] = v * g[None]
    uh = np.fft.fft2(u, axes=(2, 3))
    wh = np.einsum("abzwyx,bwyx->azyx", Kh, uh)
    w = np.fft.ifft2(wh, axes=(2, 3))[:, :, :Ny, :Nx]
    return sqsigb[None, :, None, None] * (a[None] * v - w / m.dz[None, :, None, None])


def test_spectral_apply_matches_independent_numpy(orc):
    m = tiny_model(4, 4, 3, freq=2.0)
    S, A = orc.green_tensor(m)
    sig = random_sigma(m, 9)
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, S, A)
    v = random_vec(m, 4)
    a = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v)
    b = _np_apply(m, S, A, csiga, csigb, sqsigb, v)
    assert rel(a, b) < 1e-13


def test_plane_wave_half_space_analytic(orc):
    m = IEModel(2, 2, 5, 50.0, 50.0, np.array([0.0, 10.0, 35.0, 60.0, 120.0, 300.0]), np.array([0.02]),
                np.array([]), 5.0)
    E0 = orc.plane_wave(m, 1)[1, :, 0, 0]
    k2 = 1j * m.csigma[1] * orc.mu0() * m.omega
    eta = np.sqrt(-k2)
    ana = (np.exp(-eta * m.z[:-1]) - np.exp(-eta * m.z[1:])) / (eta * m.dz)
    assert rel(E0, ana) < 1e-13


def test_solution_satisfies_system(orc):
    m, sig = config_small_block()
    m = IEModel(16, 16, 4, 100.0, 100.0, np.arange(5) * 50.0, m.sigma, m.thick, 1.0)
    sig = np.full((16, 16, 4), 0.01)
    sig[6:10, 6:10, 1:3] = 1.0
    S, A = orc.green_tensor(m)
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, S, A)
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    E0 = orc.plane_wave(m, 0)
    Es, info, hist = orc.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, None, 30, 10, 100, 1e-10)
    assert info.stat == 1 and info.be < 1e-10
    assert np.all(np.diff(hist) < 0)
    # chi = Esol / a solves A chi = sqrt(Re sb) E0
    a = 2.0 * sqsigb[:, None, None] / (csiga + np.conj(csigb)[:, None, None])
    chi = Es / a[None]
    r = orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, chi) - sqsigb[None, :, None, None] * E0
    assert np.linalg.norm(r) / np.linalg.norm(sqsigb[None, :, None, None] * E0) < 1e-9


def test_golden_fixture_reproduced(orc):
    import importlib.util
    spec = importlib.util.spec_from_file_location("mg", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = np.load(os.path.join(HERE, "golden", "golden_8x8x4.npz"))
    m, sig = mg.golden_model()
    assert np.array_equal(sig, d["sigma"])
    S, A = orc.green_tensor(m)
    assert rel(S, d["symm"]) < 1e-13 and rel(A, d["asym"]) < 1e-13
    sh, ah = orc.tensor_spectrum(m.Nx, m.Ny, m.Nz, S, A)
    assert rel(sh, d["symm_hat"]) < 1e-13 and rel(ah, d["asym_hat"]) < 1e-13
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = orc.background_cells(m)
    assert rel(orc.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, d["v"]), d["Av"]) < 1e-13
    Es, info, hist = orc.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, d["E0"], None, 30, 10, 100, 1e-10)
    assert info.iterations == d["info"][0] and info.stat == d["info"][1]
    assert rel(Es, d["Esol"]) < 1e-11


def test_tensor_lag_matches_independent_numpy(orc):
    """One lag of CalcIntegralGreenTensor3dElementGeneral restated in numpy (zz and xz blocks,
    which carry no round-off-dominated terms) against the oracle."""
    m = IEModel(4, 2, 5, 70.0, 130.0, 100.0 + np.arange(6) * 90.0, THREE_LAYER_SIGMA.copy(),
                THREE_LAYER_THICK.copy(), 0.7)
    lx, ly = 1, 1
    Nz, Nl = m.Nz, m.Nl
    mu0, w = orc.mu0(), m.omega
    cs = m.csigma
    k2 = 1j * cs * mu0 * w
    thick = np.r_[0, m.thick]
    depth = np.r_[0, np.cumsum(m.thick)]
    L = orc.layer_numbers(m)
    z, dz = m.z, np.r_[0, np.diff(m.z)]
    WT0, lms = orc.vbt_weights(lx * m.dx + m.dx / 2, ly * m.dy + m.dy / 2, m.dx, m.dy, np.hypot(m.dx, m.dy) / 2)
    DXX, DXY, DYY, DX, DY, D0 = range(6)
    WT = np.zeros((501, 6))
    WT[:, D0], WT[:, DXX], WT[:, DXY], WT[:, DX], WT[:, DYY], WT[:, DY] = (WT0[:, i] for i in range(6))
    W0 = np.zeros(6)
    W0[DXX] = abs(WT[:, DXX]).max()
    W0[[DXY, DYY, DX, DY]] = abs(WT[:, [DXY, DYY, DX, DY]]).max()
    W0[D0] = abs(WT[:, D0]).max()
    Gzz = np.zeros((Nz + 1, Nz + 1), complex)
    Gxz = np.zeros((Nz + 1, Nz + 1), complex)
    for K in range(501):
        if np.max(np.abs(WT[K] / W0)) <= 1e-12:
            continue
        lm = lms[K]
        wdx, wd0 = WT[K, DX] * lm, WT[K, D0] * lm
        eta = np.r_[0, [np.sqrt(lm * lm - k2[i]) for i in range(1, Nl + 1)]]
        el = np.r_[0, [np.exp(-2 * eta[i] * thick[i]) for i in range(1, Nl)], 0]
        p = np.zeros((Nl + 1, 2), complex)
        q = np.zeros((Nl + 1, 2), complex)
        ceta = np.sqrt(lm * lm - k2[0]) / eta[1]
        p[1] = [(1 - ceta) / (1 + ceta), (cs[0] / cs[1] - ceta) / (cs[0] / cs[1] + ceta)]
        for i in range(2, Nl + 1):
            ww = el[i - 1] * p[i - 1]
            ww = (ww - 1) / (ww + 1) * np.array([eta[i - 1] / eta[i], eta[i - 1] / eta[i] * cs[i] / cs[i - 1]])
            p[i] = (1 + ww) / (1 - ww)
        a = np.array([eta[Nl] / eta[Nl - 1], eta[Nl] / eta[Nl - 1] * cs[Nl - 1] / cs[Nl]])
        q[Nl - 1] = (1 - a) / (1 + a)
        for i in range(Nl - 2, 0, -1):
            ww = el[i + 1] * q[i + 1]
            ww = (ww - 1) / (ww + 1) * np.array([eta[i + 1] / eta[i], eta[i + 1] / eta[i] * cs[i] / cs[i + 1]])
            q[i] = (1 + ww) / (1 - ww)
        Arr = np.array([[0, 0]] + [1 / eta[i] / (1 - p[i] * q[i] * el[i]) for i in range(1, Nl + 1)])
        ex = np.r_[0, [np.exp(-eta[L[i]] * dz[i]) for i in range(1, Nz + 1)]]
        pez = np.zeros((Nz + 1, 2), complex)
        l = L[0]
        e = np.exp(-2 * eta[l] * (z[0] - depth[l - 1])) if l > 1 else (np.exp(-2 * eta[1] * z[0]) if l == 1 else 1.0)
        for i in range(1, Nz + 1):
            e = 1.0 if l != L[i] else e
            l = L[i]
            pez[i] = e * p[l]
            e = e * ex[i] ** 2
        qez = np.zeros((Nz + 1, 2), complex)
        l = L[Nz]
        e = np.exp(-2 * eta[l] * (depth[l] - z[Nz])) if l != Nl else 0.0
        for i in range(Nz, 0, -1):
            e = 1.0 if l != L[i] else e
            l = L[i]
            qez[i] = e * q[l]
            e = e * ex[i] ** 2
        fc2 = np.zeros(Nz + 1, complex)
        tf2 = np.zeros(Nz + 1, complex)
        tf3 = np.zeros(Nz + 1, complex)
        for i in range(1, Nz):
            l = L[i]
            c_ = 1 + pez[i, 1] * ex[i] ** 2
            fc2[i] = ex[i] * (1 + pez[i, 1]) / c_
            tf2[i] = (1 - fc2[i]) / cs[l]
            tf3[i] = (1 - ex[i]) / eta[l] * (1 + pez[i, 1] * ex[i]) / c_ / cs[l]
        for s in range(1, Nz + 1):
            l = L[s]
            a_ = (1 - ex[s]) * Arr[l]
            a1 = a_ / eta[l]
            a2 = a1 / eta[l]
            eta2 = eta[l] ** 2
            ft2 = a1[1] * (1 + pez[s, 1]) * (1 + qez[s, 1] * ex[s])
            fb2 = a1[1] * (1 + pez[s, 1] * ex[s]) * (1 + qez[s, 1])
            w2 = -a2[1] * ((1 - pez[s, 1]) * (1 + qez[s, 1] * ex[s]) + (1 + pez[s, 1] * ex[s]) * (1 - qez[s, 1]))
            g3 = (w2 + 2 / eta2 * dz[s]) * (1j * mu0 * w) + eta2 / cs[l] * w2
            Gzz[s, s] += g3 * wd0
            Gxz[s, s] += (fb2 - ft2) * wdx / cs[l]
            t_zz, t_xz = ft2 * wd0 * lm * lm, ft2 * wdx
            for r in range(s - 1, 0, -1):
                Gzz[r, s] += t_zz * tf3[r]
                Gxz[r, s] += t_xz * tf2[r]
                t_zz *= fc2[r]
                t_xz *= fc2[r]
    S, A = orc.green_tensor(m)
    P = Nz * (Nz + 1) // 2
    zz = np.array([Gzz[i + 1, j + 1] for j in range(Nz) for i in range(j + 1)]) / np.pi / 4
    assert rel(zz, S[lx, ly, 3]) < 1e-12
    xz_up = np.array([Gxz[i + 1, j + 1] for j in range(Nz) for i in range(j + 1)]) / np.pi / 4
    xz_o = A[lx, ly, 0].reshape(Nz, Nz)  # [col][row]
    xz_o_up = np.array([xz_o[j, i] for j in range(Nz) for i in range(j + 1)])
    assert rel(xz_up, xz_o_up) < 1e-12
