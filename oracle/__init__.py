"""CPU FP64 oracle for GIEM2G's integral-equation solve path.

TEST INFRASTRUCTURE ONLY.  This package restates the reference's Fortran
routines in C (``giem2g_oracle.c``) and exposes them through ctypes.  The
product (``giem2g_b200``) never imports it; only ``tests/``, the smoke check and
the benchmark's CPU-baseline leg do, as the checker.

Parity status: the reference ships no tests or golden vectors and cannot be
built in this environment (Fortran/MPI/FFTW), so parity against reference
outputs is UNPINNED.  The oracle is anchored on a dense block-Toeplitz brute
force and on an independent numpy restatement (tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc_giem2g.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "giem2g_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_green_tensor.argtypes = [vp, vp, vp, ip]
        L.orc_tensor_spectrum.argtypes = [ip, ip, ip, vp, vp, vp, vp, ip]
        L.orc_apply.argtypes = [ip, ip, ip, vp, vp, vp, vp, vp, vp, vp, vp, ip]
        L.orc_apply_toeplitz.argtypes = [ip, ip, ip, vp, vp, vp, vp, vp, vp, vp, vp]
        L.orc_plane_wave.argtypes = [vp, ip, vp]
        L.orc_solve.argtypes = [ip, ip, ip, vp, vp, vp, vp, vp, vp, vp, vp, ip, ip, ip, dp, vp, vp, vp, ip, ip]
        L.orc_vbt_weights.argtypes = [dp, dp, dp, dp, dp, vp, vp]
        L.orc_background_cells.argtypes = [vp, vp, vp]
        L.orc_layer_numbers.argtypes = [vp, vp]
        L.orc_prepare_receivers.argtypes = [vp, ip, vp, vp, vp]
        L.orc_vbt_weights_single.argtypes = [dp, dp, dp, dp, dp, vp, vp]
        L.orc_rc_tensor.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, ip]
        L.orc_rc_tensor_lags.argtypes = [vp, ip, vp, vp, vp, vp, vp, ip, vp, vp, vp, ip]
        L.orc_rc_apply_direct.argtypes = [ip, ip, ip, ip, vp, vp, vp, vp, vp, vp, ip]
        L.orc_rc_apply_fft.argtypes = [ip, ip, ip, ip, vp, vp, vp, vp, vp, vp, ip]
        L.orc_plane_wave_points.argtypes = [vp, ip, ip, vp, vp]
        L.orc_eps0.restype = dp
        L.orc_mu0.restype = dp
        _lib = L
    return _lib


class _Model(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("z", ctypes.c_void_p), ("Nl", ctypes.c_int),
        ("csigma", ctypes.c_void_p), ("thick", ctypes.c_void_p), ("omega", ctypes.c_double),
    ]


class OrcResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("bea", ctypes.c_double), ("be", ctypes.c_double),
                ("stat", ctypes.c_int), ("applies", ctypes.c_int)]


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _model_struct(m):
    z = _f64(m.z)
    cs = _c128(m.csigma)
    th = _f64(m.thick) if len(m.thick) else np.zeros(1)
    s = _Model(m.Nx, m.Ny, m.Nz, m.dx, m.dy, z.ctypes.data, m.Nl, cs.ctypes.data, th.ctypes.data, m.omega)
    return s, (z, cs, th)


def green_tensor(m, nthreads: int = 0):
    """Spatial tensor: symm[Nx,Ny,4,P], asym[Nx,Ny,2,Nz*Nz] (calc_ie_tensor_module.F90:54)."""
    P = m.Nz * (m.Nz + 1) // 2
    symm = np.zeros((m.Nx, m.Ny, 4, P), np.complex128)
    asym = np.zeros((m.Nx, m.Ny, 2, m.Nz * m.Nz), np.complex128)
    s, keep = _model_struct(m)
    lib().orc_green_tensor(ctypes.byref(s), _p(symm), _p(asym), nthreads)
    return symm, asym


def background_cells(m):
    csigb = np.zeros(m.Nz, np.complex128)
    sqsigb = np.zeros(m.Nz, np.float64)
    s, keep = _model_struct(m)
    lib().orc_background_cells(ctypes.byref(s), _p(csigb), _p(sqsigb))
    return csigb, sqsigb


def layer_numbers(m):
    L = np.zeros(m.Nz + 1, np.int32)
    s, keep = _model_struct(m)
    lib().orc_layer_numbers(ctypes.byref(s), _p(L))
    return L


def tensor_spectrum(Nx, Ny, Nz, symm, asym, nthreads: int = 0):
    symm, asym = _c128(symm), _c128(asym)
    sh = np.zeros_like(symm)
    ah = np.zeros_like(asym)
    lib().orc_tensor_spectrum(Nx, Ny, Nz, _p(symm), _p(asym), _p(sh), _p(ah), nthreads)
    return sh, ah


def apply(Nx, Ny, Nz, sh, ah, csiga, csigb, sqsigb, dz, v_in, nthreads: int = 0):
    sh, ah, csiga, csigb = _c128(sh), _c128(ah), _c128(csiga), _c128(csigb)
    sqsigb, dz, v_in = _f64(sqsigb), _f64(dz), _c128(v_in)
    out = np.zeros_like(v_in)
    lib().orc_apply(Nx, Ny, Nz, _p(sh), _p(ah), _p(csiga), _p(csigb), _p(sqsigb), _p(dz), _p(v_in), _p(out), nthreads)
    return out


def apply_toeplitz(Nx, Ny, Nz, symm, asym, csiga, csigb, sqsigb, dz, v_in):
    symm, asym, csiga, csigb = _c128(symm), _c128(asym), _c128(csiga), _c128(csigb)
    sqsigb, dz, v_in = _f64(sqsigb), _f64(dz), _c128(v_in)
    out = np.zeros_like(v_in)
    lib().orc_apply_toeplitz(Nx, Ny, Nz, _p(symm), _p(asym), _p(csiga), _p(csigb), _p(sqsigb), _p(dz), _p(v_in), _p(out))
    return out


def plane_wave(m, pol: int):
    """pol 0 = EX, 1 = EY.  Returns E0[3,Nz,Ny,Nx] (sources_module.F90:67)."""
    E0 = np.zeros((3, m.Nz, m.Ny, m.Nx), np.complex128)
    s, keep = _model_struct(m)
    lib().orc_plane_wave(ctypes.byref(s), pol, _p(E0))
    return E0


def solve(Nx, Ny, Nz, sh, ah, csiga, csigb, sqsigb, dz, E_bkg, E0_guess=None, outer_buf=30, inner_buf=10,
          max_restart=100, tol=1e-8, history_len=4096, nthreads: int = 0):
    """SolveEquation (ie_solver_module.F90:43).  Returns (Esol, OrcResult, outer misfit history)."""
    sh, ah, csiga, csigb = _c128(sh), _c128(ah), _c128(csiga), _c128(csigb)
    sqsigb, dz, E_bkg = _f64(sqsigb), _f64(dz), _c128(E_bkg)
    g = _c128(E0_guess) if E0_guess is not None else None
    Esol = np.zeros_like(E_bkg)
    info = OrcResult()
    hist = np.zeros(history_len, np.float64)
    lib().orc_solve(Nx, Ny, Nz, _p(sh), _p(ah), _p(csiga), _p(csigb), _p(sqsigb), _p(dz), _p(E_bkg),
                    _p(g) if g is not None else None, outer_buf, inner_buf, max_restart, tol, _p(Esol),
                    ctypes.byref(info), _p(hist), history_len, nthreads)
    return Esol, info, hist[: max(0, min(info.iterations, history_len))].copy()


def vbt_weights(x, y, hx, hy, rmin):
    WT = np.zeros((501, 6), np.float64)
    lms = np.zeros(501, np.float64)
    lib().orc_vbt_weights(x, y, hx, hy, rmin, _p(WT), _p(lms))
    return WT, lms


def vbt_weights_single(x, y, hx, hy, rmin):
    """VBTransformWeightsAllSingleInt (VolumeBesselTransforms.F90:198-229): WT[501, 6], lms[501]."""
    WT = np.zeros((501, 6), np.float64)
    lms = np.zeros(501, np.float64)
    lib().orc_vbt_weights_single(x, y, hx, hy, rmin, _p(WT), _p(lms))
    return WT, lms


@dataclass
class Receivers:
    """Receivers after PrepareRecvs (data_types_module.F90:124-152)."""
    zrecv: np.ndarray
    x_shift: np.ndarray
    y_shift: np.ndarray
    recv_layer: np.ndarray
    anom_cell: np.ndarray

    @property
    def Nr(self):
        return len(self.zrecv)


def prepare_receivers(m, zrecv, x_shift=None, y_shift=None) -> Receivers:
    z = _f64(np.array(zrecv, dtype=np.float64))
    Nr = len(z)
    xs = _f64(np.zeros(Nr) if x_shift is None else x_shift)
    ys = _f64(np.zeros(Nr) if y_shift is None else y_shift)
    rl = np.zeros(Nr, np.int32)
    ac = np.zeros(Nr, np.int32)
    s, keep = _model_struct(m)
    lib().orc_prepare_receivers(ctypes.byref(s), Nr, _p(z), _p(rl), _p(ac))
    return Receivers(z, xs, ys, rl, ac)


def rc_tensor(m, rv: Receivers, nthreads: int = 0):
    """Spatial receiver tensor [2Ny, 2Nx, 15, Nr, Nz] (calc_rc_tensor_module.F90:38-229)."""
    G = np.zeros((2 * m.Ny, 2 * m.Nx, 15, rv.Nr, m.Nz), np.complex128)
    s, keep = _model_struct(m)
    lib().orc_rc_tensor(ctypes.byref(s), rv.Nr, _p(rv.zrecv), _p(rv.x_shift), _p(rv.y_shift), _p(rv.recv_layer),
                        _p(rv.anom_cell), _p(G), nthreads)
    return G


def rc_tensor_lags(m, rv: Receivers, ix, iy, nthreads: int = 0):
    """Selected lag-plane indices of the receiver tensor: [n, 15, Nr, Nz]."""
    ix = np.ascontiguousarray(ix, dtype=np.int32)
    iy = np.ascontiguousarray(iy, dtype=np.int32)
    out = np.zeros((len(ix), 15, rv.Nr, m.Nz), np.complex128)
    s, keep = _model_struct(m)
    lib().orc_rc_tensor_lags(ctypes.byref(s), rv.Nr, _p(rv.zrecv), _p(rv.x_shift), _p(rv.y_shift), _p(rv.recv_layer),
                             _p(rv.anom_cell), len(ix), _p(ix), _p(iy), _p(out), nthreads)
    return out


def rc_apply(Nx, Ny, Nz, G, csiga, csigb, E, direct: bool = False, nthreads: int = 0):
    """ReCalculation (Continuation_Function_Module.F90:198-239): anomalous fields at the receivers,
    Ea, Ha [Ny, Nx, 3, Nr], from the anomaly field E [3, Nz, Ny, Nx].  direct=True sums the lags
    directly instead of going through the FFT."""
    G, csiga, csigb, E = _c128(G), _c128(csiga), _c128(csigb), _c128(E)
    Nr = G.shape[3]
    Ea = np.zeros((Ny, Nx, 3, Nr), np.complex128)
    Ha = np.zeros_like(Ea)
    fn = lib().orc_rc_apply_direct if direct else lib().orc_rc_apply_fft
    fn(Nx, Ny, Nz, Nr, _p(G), _p(csiga), _p(csigb), _p(E), _p(Ea), _p(Ha), nthreads)
    return Ea, Ha


def plane_wave_points(m, pol: int, zrecv):
    """PlaneWave (sources_module.F90:26-66): F[Nr, 6] = Ex Ey Ez Hx Hy Hz at the receiver depths."""
    z = _f64(np.array(zrecv, dtype=np.float64))
    F = np.zeros((len(z), 6), np.complex128)
    s, keep = _model_struct(m)
    lib().orc_plane_wave_points(ctypes.byref(s), pol, len(z), _p(z), _p(F))
    return F


def eps0() -> float:
    return lib().orc_eps0()


def mu0() -> float:
    return lib().orc_mu0()
