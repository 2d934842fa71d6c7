"""B200-native implementation of GIEM2G's integral-equation solve path.

The compute runs in ``_lib/libgiem2g_b200.so`` (hand-written sm_100a CUDA behind the C ABI
declared in ``include/giem2g.h``).  This module is a thin ctypes host layer that mirrors
the reference's Fortran module interface for the path:

  IEOperator.set_anomaly_sigma   SetAnomalySigma   (ie_solver_module.F90:116)
  IEOperator.calc_ie_kernel      CalcIntegralGreenTensor (calc_ie_tensor_module.F90:54)
  IEOperator.calc_fft_of_ie_kernel CalcFFTofIETensor (Integral_Equation_Module.F90:310)
  IEOperator.apply_precond       APPLY_PRECOND     (apply_ie_operator_module.F90:39)
  IEOperator.solve_equation      SolveEquation     (ie_solver_module.F90:43)

There is no CPU fallback: importing the library fails loudly if the extension is missing.
"""
from __future__ import annotations

import ctypes
import os
import sys
from contextlib import contextmanager
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_lib", "libgiem2g_b200.so")
_lib = None

CONVERGED, NON_TRUE_CONVERGED, NON_CONVERGED, INTERUPTED = 1, 2, -1, -3  # fgmres_interfaces.F90:25-30


class Giem2gError(RuntimeError):
    pass


class BackgroundT(ctypes.Structure):      # giem2g_interfaces.F90:33-37
    _fields_ = [("Nl", ctypes.c_int), ("csigb", ctypes.c_void_p), ("thickness", ctypes.c_void_p)]


class AnomalyT(ctypes.Structure):         # giem2g_interfaces.F90:39-44
    _fields_ = [("Nx", ctypes.c_int), ("Ny", ctypes.c_int), ("Nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("z", ctypes.c_void_p), ("dz", ctypes.c_void_p)]


class DataT(ctypes.Structure):            # giem2g_interfaces.F90:46-58
    _fields_ = [("tensor_size", ctypes.c_longlong), ("ie_kernel_buffer_length", ctypes.c_longlong),
                ("fft_buffers_length", ctypes.c_longlong), ("comm64", ctypes.c_longlong),
                ("giem2g_tensor", ctypes.c_void_p), ("dz", ctypes.c_void_p), ("sqsigb", ctypes.c_void_p),
                ("csigb", ctypes.c_void_p), ("kernel_buffer", ctypes.c_void_p),
                ("fft_buffer_in", ctypes.c_void_p), ("fft_buffer_out", ctypes.c_void_p)]


PRECOND_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                              ctypes.c_void_p)


class FgmresCtl(ctypes.Structure):        # data_types_module.F90:49-55 (+ precision)
    _fields_ = [("misfit", ctypes.c_double), ("fgmres_maxit", ctypes.c_int), ("gmres_buf", ctypes.c_int),
                ("fgmres_buf", ctypes.c_int), ("precision", ctypes.c_int)]


class ResultT(ctypes.Structure):          # fgmres_interfaces.F90:34-39 (+ counters)
    _fields_ = [("iterations", ctypes.c_int), ("bea", ctypes.c_double), ("be", ctypes.c_double),
                ("stat", ctypes.c_int), ("applies_fp64", ctypes.c_int), ("applies_fp32", ctypes.c_int),
                ("device_ms", ctypes.c_double), ("precond_steps", ctypes.c_int)]


EXPORTED_SYMBOLS = [
    "giem2g_calc_data_sizes", "giem2g_prepare_ie_kernel", "giem2g_calc_ie_kernel",
    "giem2g_calc_fft_of_ie_kernel", "giem2g_set_anomaly_conductivity", "giem2g_apply_ie_operator",
    "giem2g_set_logger", "giem2g_print_stats", "giem2g_delete_ie_operator",
    "giem2g_last_status", "giem2g_last_error", "giem2g_set_background", "giem2g_set_ie_kernel_spatial",
    "giem2g_get_ie_kernel_spatial", "giem2g_get_ie_kernel_spectral", "giem2g_apply_ie_operator_device",
    "giem2g_get_stream", "giem2g_last_apply_ms", "giem2g_last_kernel_launches", "giem2g_apply_count", "giem2g_solve",
    "giem2g_solve_device", "giem2g_get_misfit_history", "giem2g_check_device_error",
    "giem2g_contract_variants", "giem2g_set_contract_variant", "giem2g_kernel_launch_count",
    "giem2g_apply_ie_operator_device_static", "giem2g_batch_create", "giem2g_batch_solve_device",
    "giem2g_solve_batched", "giem2g_batch_misfit_history", "giem2g_batch_delete",
    "giem2g_apply_ie_operator_device_batch", "giem2g_gemm_bf16_tn", "giem2g_im2col3d_bf16",
    "giem2g_col2im3d_f32", "giem2g_set_outer_preconditioner", "giem2g_set_fft_lines", "giem2g_set_fft_lines_precision",
    "giem2g_set_kernel_timing", "giem2g_last_contract_ms",
    "giem2g_rc_create", "giem2g_rc_receivers", "giem2g_rc_calc_kernel", "giem2g_rc_calc_fft_of_kernel",
    "giem2g_rc_get_kernel", "giem2g_rc_set_anomaly_conductivity", "giem2g_rc_recalculate",
    "giem2g_rc_recalculate_device", "giem2g_rc_get_stream", "giem2g_rc_delete", "giem2g_set_precision",
    "giem2g_set_preconditioner", "giem2g_preconditioner_calls", "giem2g_apply_preconditioner",
    "giem2g_selftest_bounded_wait",
]


def library_path() -> str:
    return _LIB_PATH


def lib():
    """Load the CUDA library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise Giem2gError(f"CUDA extension not built: {_LIB_PATH} missing (run giem2g_b200.build.build())")
    L = ctypes.CDLL(_LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.giem2g_calc_data_sizes.argtypes = [AnomalyT, ctypes.POINTER(DataT)]
    L.giem2g_calc_data_sizes.restype = None
    L.giem2g_prepare_ie_kernel.argtypes = [AnomalyT, DataT]
    L.giem2g_prepare_ie_kernel.restype = None
    L.giem2g_calc_ie_kernel.argtypes = [vp, BackgroundT, AnomalyT, dp]
    L.giem2g_calc_ie_kernel.restype = None
    L.giem2g_calc_fft_of_ie_kernel.argtypes = [vp]
    L.giem2g_calc_fft_of_ie_kernel.restype = None
    L.giem2g_set_anomaly_conductivity.argtypes = [vp, vp]
    L.giem2g_set_anomaly_conductivity.restype = None
    L.giem2g_apply_ie_operator.argtypes = [vp, vp, vp]
    L.giem2g_apply_ie_operator.restype = None
    L.giem2g_print_stats.argtypes = [vp]
    L.giem2g_print_stats.restype = None
    L.giem2g_delete_ie_operator.argtypes = [vp]
    L.giem2g_delete_ie_operator.restype = None
    L.giem2g_last_status.restype = ip
    L.giem2g_last_error.restype = ctypes.c_char_p
    L.giem2g_set_background.argtypes = [vp, BackgroundT, dp]
    L.giem2g_set_ie_kernel_spatial.argtypes = [vp, vp, vp]
    L.giem2g_get_ie_kernel_spatial.argtypes = [vp, vp, vp]
    L.giem2g_get_ie_kernel_spectral.argtypes = [vp, vp, vp]
    L.giem2g_apply_ie_operator_device.argtypes = [vp, vp, vp, ip]
    L.giem2g_get_stream.argtypes = [vp]
    L.giem2g_get_stream.restype = vp
    L.giem2g_last_apply_ms.argtypes = [vp]
    L.giem2g_last_apply_ms.restype = dp
    L.giem2g_last_kernel_launches.argtypes = [vp]
    L.giem2g_apply_count.argtypes = [vp]
    L.giem2g_apply_count.restype = ctypes.c_longlong
    L.giem2g_solve.argtypes = [vp, vp, vp, vp, FgmresCtl, ctypes.POINTER(ResultT)]
    L.giem2g_solve_device.argtypes = [vp, vp, vp, vp, FgmresCtl, ctypes.POINTER(ResultT)]
    L.giem2g_get_misfit_history.argtypes = [vp, vp, ip]
    L.giem2g_check_device_error.argtypes = [vp]
    L.giem2g_contract_variants.argtypes = [vp, ip]
    L.giem2g_kernel_launch_count.restype = ctypes.c_longlong
    L.giem2g_set_contract_variant.argtypes = [vp, ip, ip]
    pp = ctypes.POINTER(ctypes.c_void_p)
    L.giem2g_apply_ie_operator_device_static.argtypes = [vp, vp, vp, ip]
    L.giem2g_batch_create.argtypes = [pp, ip, FgmresCtl]
    L.giem2g_batch_create.restype = vp
    L.giem2g_batch_solve_device.argtypes = [vp, pp, pp, pp, FgmresCtl, ctypes.POINTER(ResultT)]
    L.giem2g_solve_batched.argtypes = [vp, pp, pp, pp, FgmresCtl, ctypes.POINTER(ResultT)]
    L.giem2g_batch_misfit_history.argtypes = [vp, ip, vp, ip]
    L.giem2g_batch_delete.argtypes = [vp]
    L.giem2g_batch_delete.restype = None
    L.giem2g_apply_ie_operator_device_batch.argtypes = [vp, ip, pp, pp, ip]
    L.giem2g_gemm_bf16_tn.argtypes = [vp, vp, vp, ip, ip, ip, ip, ip, ip, ip, vp, vp]
    L.giem2g_im2col3d_bf16.argtypes = [vp, vp, ip, ip, ip, ip, ip, ip, ip, vp]
    L.giem2g_col2im3d_f32.argtypes = [vp, vp, ip, ip, ip, ip, ip, ip, ip, vp]
    L.giem2g_set_outer_preconditioner.argtypes = [vp, ip, PRECOND_FN, vp]
    L.giem2g_set_fft_lines.argtypes = [vp, ip]
    L.giem2g_set_fft_lines_precision.argtypes = [vp, ip, ip]
    L.giem2g_set_precision.argtypes = [vp, ip]
    L.giem2g_set_preconditioner.argtypes = [vp, ip, ctypes.c_char_p]
    L.giem2g_preconditioner_calls.argtypes = [vp]
    L.giem2g_preconditioner_calls.restype = ctypes.c_longlong
    L.giem2g_apply_preconditioner.argtypes = [vp, vp, vp]
    L.giem2g_selftest_bounded_wait.argtypes = [ip]
    L.giem2g_set_kernel_timing.argtypes = [vp, ip]
    L.giem2g_last_contract_ms.argtypes = [vp]
    L.giem2g_last_contract_ms.restype = dp
    L.giem2g_rc_create.argtypes = [BackgroundT, AnomalyT, ip, vp, vp, vp]
    L.giem2g_rc_create.restype = vp
    L.giem2g_rc_receivers.argtypes = [vp, vp, vp, vp]
    L.giem2g_rc_calc_kernel.argtypes = [vp, BackgroundT, dp]
    L.giem2g_rc_calc_fft_of_kernel.argtypes = [vp]
    L.giem2g_rc_get_kernel.argtypes = [vp, vp]
    L.giem2g_rc_set_anomaly_conductivity.argtypes = [vp, vp]
    L.giem2g_rc_recalculate.argtypes = [vp, vp, vp, vp]
    L.giem2g_rc_recalculate_device.argtypes = [vp, vp, vp, vp]
    L.giem2g_rc_get_stream.argtypes = [vp]
    L.giem2g_rc_get_stream.restype = vp
    L.giem2g_rc_delete.argtypes = [vp]
    L.giem2g_rc_delete.restype = None
    _lib = L
    return L


LOGGER_FN = ctypes.CFUNCTYPE(None, ctypes.c_char_p)
_logger_ref = None


def set_logger(fn=None):
    """giem2g_set_logger (giem2g_interfaces.F90:234-238): fn(str) receives every log line; None = stdout."""
    global _logger_ref
    _logger_ref = LOGGER_FN(lambda b: fn(b.decode(errors="replace"))) if fn else None
    lib().giem2g_set_logger(_logger_ref)


def kernel_launch_count() -> int:
    """Cumulative count of this library's kernel launches in this process."""
    return int(lib().giem2g_kernel_launch_count())


def _check(rc=None, what=""):
    L = lib()
    st = L.giem2g_last_status() if rc is None else rc
    if st != 0:
        raise Giem2gError(f"{what}: status {st}: {L.giem2g_last_error().decode(errors='replace')}")


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


@contextmanager
def _torch_ordered(stream_ptr):
    """Order a device-pointer call on a library stream against torch's current stream.

    The library's streams are non-blocking: they do not wait for torch's work, so a call whose inputs
    were just written by torch (a dtype conversion, a copy, randn) could read them half-written, and
    torch could read the call's outputs before they are complete.  On entry the library stream waits for
    torch's current stream; on exit torch's current stream waits for the library stream.  Both are
    device-side waits (events), the host does not block.  Without torch, before torch has set up CUDA,
    or when torch's current stream is the library stream itself, nothing is done here (the C ABI's
    contract: the caller orders its own work)."""
    torch = sys.modules.get("torch")
    pair = None
    if torch is not None and torch.cuda.is_initialized():
        cur = torch.cuda.current_stream()
        if cur.cuda_stream != stream_ptr:
            pair = (cur, torch.cuda.ExternalStream(stream_ptr))
            pair[1].wait_stream(pair[0])
    try:
        yield
    finally:
        if pair is not None:
            pair[0].wait_stream(pair[1])


@dataclass
class SolveInfo:
    iterations: int
    bea: float
    be: float
    stat: int
    applies_fp64: int
    applies_fp32: int
    device_ms: float
    misfits: np.ndarray
    precond_steps: int = 0


class IEOperator:
    """One IE operator resident on the current CUDA device (IntegralEquationOperator)."""

    def __init__(self, Nx, Ny, Nz, dx, dy, z):
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.dx, self.dy = float(dx), float(dy)
        self._z = np.ascontiguousarray(z, dtype=np.float64)
        self._dz = np.ascontiguousarray(np.diff(self._z), dtype=np.float64)
        self._anom = AnomalyT(self.Nx, self.Ny, self.Nz, self.dx, self.dy, self._z.ctypes.data, self._dz.ctypes.data)
        L = lib()
        self._data = DataT()
        L.giem2g_calc_data_sizes(self._anom, ctypes.byref(self._data))
        _check(what="giem2g_calc_data_sizes")
        L.giem2g_prepare_ie_kernel(self._anom, self._data)
        _check(what="giem2g_prepare_ie_kernel")
        self.handle = self._data.giem2g_tensor
        self._keep = []

    @classmethod
    def from_model(cls, m):
        return cls(m.Nx, m.Ny, m.Nz, m.dx, m.dy, m.z)

    @property
    def nvec(self):
        return 3 * self.Nx * self.Ny * self.Nz

    @property
    def kernel_buffer_length(self):
        return self._data.ie_kernel_buffer_length

    def _bkg(self, csigma, thick):
        cs = _c128(csigma)
        th = np.ascontiguousarray(thick, dtype=np.float64) if len(thick) else np.zeros(1)
        self._keep = [cs, th]
        return BackgroundT(len(cs) - 1, cs.ctypes.data, th.ctypes.data)

    def set_background(self, csigma, thick, omega):
        _check(lib().giem2g_set_background(self.handle, self._bkg(csigma, thick), float(omega)), "giem2g_set_background")

    def calc_ie_kernel(self, csigma, thick, omega):
        """CalcIntegralGreenTensor on the GPU (FP64)."""
        lib().giem2g_calc_ie_kernel(self.handle, self._bkg(csigma, thick), self._anom, float(omega))
        _check(what="giem2g_calc_ie_kernel")

    def set_ie_kernel_spatial(self, symm, asym):
        s, a = _c128(symm), _c128(asym)
        _check(lib().giem2g_set_ie_kernel_spatial(self.handle, s.ctypes.data, a.ctypes.data), "set_ie_kernel_spatial")

    def get_ie_kernel_spatial(self):
        P = self.Nz * (self.Nz + 1) // 2
        s = np.zeros((self.Nx, self.Ny, 4, P), np.complex128)
        a = np.zeros((self.Nx, self.Ny, 2, self.Nz * self.Nz), np.complex128)
        _check(lib().giem2g_get_ie_kernel_spatial(self.handle, s.ctypes.data, a.ctypes.data), "get_ie_kernel_spatial")
        return s, a

    def get_ie_kernel_spectral(self):
        P = self.Nz * (self.Nz + 1) // 2
        s = np.zeros((self.Nx, self.Ny, 4, P), np.complex128)
        a = np.zeros((self.Nx, self.Ny, 2, self.Nz * self.Nz), np.complex128)
        _check(lib().giem2g_get_ie_kernel_spectral(self.handle, s.ctypes.data, a.ctypes.data), "get_ie_kernel_spectral")
        return s, a

    def calc_fft_of_ie_kernel(self):
        lib().giem2g_calc_fft_of_ie_kernel(self.handle)
        _check(what="giem2g_calc_fft_of_ie_kernel")

    def set_anomaly_conductivity(self, csiga):
        """csiga: complex [Nz,Ny,Nx] (Fortran (Nx,Ny,Nz))."""
        c = _c128(csiga)
        assert c.size == self.Nx * self.Ny * self.Nz
        lib().giem2g_set_anomaly_conductivity(self.handle, c.ctypes.data)
        _check(what="giem2g_set_anomaly_conductivity")

    def set_anomaly_sigma(self, siga_file_order, freq, displacement_currents=True):
        """SetAnomalySigma: real sigma in file order [Ny,Nx,Nz] -> csiga."""
        from .synthetic import csiga_from_sigma
        self.set_anomaly_conductivity(csiga_from_sigma(siga_file_order, freq, displacement_currents))

    def apply_precond(self, v_in):
        """APPLY_PRECOND through giem2g_apply_ie_operator (host arrays, complex128)."""
        vi = _c128(v_in)
        assert vi.size == self.nvec
        vo = np.empty_like(vi)
        lib().giem2g_apply_ie_operator(self.handle, vi.ctypes.data, vo.ctypes.data)
        _check(what="giem2g_apply_ie_operator")
        return vo

    def apply_device(self, d_in: int, d_out: int, precision: int = 0):
        with _torch_ordered(self.stream):
            _check(lib().giem2g_apply_ie_operator_device(self.handle, d_in, d_out, precision), "apply_device")

    def contract_variants(self, precision: int) -> int:
        return lib().giem2g_contract_variants(self.handle, precision)

    def set_contract_variant(self, precision: int, variant: int):
        _check(lib().giem2g_set_contract_variant(self.handle, precision, variant), "set_contract_variant")

    def set_precision(self, mode: int):
        """giem2g_set_precision: 1 makes apply_precond compute in complex64 and is the precision of
        solves called with precision=-1."""
        _check(lib().giem2g_set_precision(self.handle, int(mode)), "set_precision")

    def set_preconditioner(self, kind: int, weights_path: str | None = None):
        """giem2g_set_preconditioner: the learned U-Net evaluated inside the library (kind 1: warm start of the
        inner GMRES, 2: replaces it, 0: off).  Default weights: weights/unet3d_c4.npz next to this module."""
        if weights_path is None and kind:
            weights_path = os.path.join(_HERE, "weights", "unet3d_c4.npz")
        _check(lib().giem2g_set_preconditioner(self.handle, int(kind), weights_path.encode() if weights_path else None),
               "set_preconditioner")

    def apply_preconditioner(self, d_v: int, d_z: int):
        """giem2g_apply_preconditioner: d_z = the registered network's guess of A^-1 v (device pointers)."""
        with _torch_ordered(self.stream):
            _check(lib().giem2g_apply_preconditioner(self.handle, d_v, d_z), "apply_preconditioner")

    def preconditioner_calls(self) -> int:
        return int(lib().giem2g_preconditioner_calls(self.handle))

    def set_fft_lines(self, lines: int, precision: int | None = None):
        if precision is None:
            _check(lib().giem2g_set_fft_lines(self.handle, lines), "set_fft_lines")
        else:
            _check(lib().giem2g_set_fft_lines_precision(self.handle, precision, lines), "set_fft_lines")

    def set_kernel_timing(self, on: bool):
        _check(lib().giem2g_set_kernel_timing(self.handle, 1 if on else 0), "set_kernel_timing")

    def last_contract_ms(self) -> float:
        return float(lib().giem2g_last_contract_ms(self.handle))

    def check_device_error(self):
        _check(lib().giem2g_check_device_error(self.handle), "device error word")

    @property
    def stream(self) -> int:
        return lib().giem2g_get_stream(self.handle)

    def last_apply_ms(self) -> float:
        return lib().giem2g_last_apply_ms(self.handle)

    def last_kernel_launches(self) -> int:
        return lib().giem2g_last_kernel_launches(self.handle)

    def _ctl(self, tol, max_restart, outer_buf, inner_buf, precision):
        return FgmresCtl(float(tol), int(max_restart), int(inner_buf), int(outer_buf), int(precision))

    def _info(self, r):
        h = np.zeros(max(1, r.iterations), np.float64)
        n = lib().giem2g_get_misfit_history(self.handle, h.ctypes.data, len(h))
        return SolveInfo(r.iterations, r.bea, r.be, r.stat, r.applies_fp64, r.applies_fp32, r.device_ms, h[:n].copy(),
                         r.precond_steps)

    def solve_equation(self, E_bkg, E0=None, tol=1e-8, max_restart=100, outer_buf=30, inner_buf=10, precision=0):
        """SolveEquation with host arrays (Nx,Ny,Nz,3) complex128; returns (Esol, SolveInfo)."""
        eb = _c128(E_bkg)
        es = np.empty_like(eb)
        e0 = _c128(E0) if E0 is not None else None
        r = ResultT()
        rc = lib().giem2g_solve(self.handle, eb.ctypes.data, es.ctypes.data, e0.ctypes.data if e0 is not None else None,
                                self._ctl(tol, max_restart, outer_buf, inner_buf, precision), ctypes.byref(r))
        _check(rc, "giem2g_solve")
        return es, self._info(r)

    def solve_device(self, d_ebkg: int, d_esol: int, d_e0=None, tol=1e-8, max_restart=100, outer_buf=30,
                     inner_buf=10, precision=0):
        r = ResultT()
        with _torch_ordered(self.stream):
            rc = lib().giem2g_solve_device(self.handle, d_ebkg, d_esol, d_e0,
                                           self._ctl(tol, max_restart, outer_buf, inner_buf, precision),
                                           ctypes.byref(r))
        _check(rc, "giem2g_solve_device")
        return self._info(r)

    def set_outer_preconditioner(self, mode, fn=None):
        """giem2g_set_outer_preconditioner: fn(d_v, d_z, n, stream) -> 0 writes a guess of A^-1 v (mode 1:
        warm start of the inner GMRES, mode 2: Z itself); mode 0 removes it."""
        if mode == 0 or fn is None:
            self._precond_ref = None
            _check(lib().giem2g_set_outer_preconditioner(self.handle, 0, PRECOND_FN(), None), "set_outer_preconditioner")
            return

        def cb(user, d_v, d_z, n, stream):
            try:
                return int(fn(d_v, d_z, n, stream))
            except Exception as exc:  # a failing hook is dropped for the rest of the solve
                self._precond_error = exc
                return 1
        self._precond_ref = PRECOND_FN(cb)
        _check(lib().giem2g_set_outer_preconditioner(self.handle, int(mode), self._precond_ref, None),
               "set_outer_preconditioner")

    def print_stats(self):
        lib().giem2g_print_stats(self.handle)

    def delete(self):
        if self.handle:
            lib().giem2g_delete_ie_operator(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass


class RCOperator:
    """Receiver continuation on the current CUDA device (RC_OPERATOR, Continuation_Function_Module.F90).

    Receivers: depths zrecv with lateral shifts; receiver r at anomaly cell (ix, iy) is the point
    ((ix+1/2) dx + x_shift, (iy+1/2) dy + y_shift, zrecv).  Fields at the receivers come back as
    complex [Ny, Nx, 3, Nr] (the reference's Ea(Nr,3,Nx,Ny)).

      RCOperator(...)            PrepareRecvs + PrepareContinuationOperator
      calc_rc_kernel             CalcRecalculationGreenTensor (calc_rc_tensor_module.F90:38)
      calc_fft_of_rc_kernel      CalcFFTofRCTensor (Continuation_Function_Module.F90:330)
      set_anomaly_sigma          FinalizeRCOperator (:165)
      recalculate                ReCalculation (:198): anomalous E and H at the receivers
    """

    def __init__(self, Nx, Ny, Nz, dx, dy, z, thick, zrecv, x_shift=None, y_shift=None):
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.dx, self.dy = float(dx), float(dy)
        self._z = np.ascontiguousarray(z, dtype=np.float64)
        self._dz = np.ascontiguousarray(np.diff(self._z), dtype=np.float64)
        self._anom = AnomalyT(self.Nx, self.Ny, self.Nz, self.dx, self.dy, self._z.ctypes.data, self._dz.ctypes.data)
        zr = np.ascontiguousarray(np.atleast_1d(zrecv), dtype=np.float64)
        self.Nr = len(zr)
        xs = np.ascontiguousarray(np.zeros(self.Nr) if x_shift is None else x_shift, dtype=np.float64)
        ys = np.ascontiguousarray(np.zeros(self.Nr) if y_shift is None else y_shift, dtype=np.float64)
        self.x_shift, self.y_shift = xs, ys
        th = np.ascontiguousarray(thick, dtype=np.float64) if len(thick) else np.zeros(1)
        cs = np.zeros(len(thick) + 2, np.complex128)  # values unused here: only the layer depths
        bkg = BackgroundT(len(thick) + 1, cs.ctypes.data, th.ctypes.data)
        self.handle = lib().giem2g_rc_create(bkg, self._anom, self.Nr, zr.ctypes.data, xs.ctypes.data, ys.ctypes.data)
        if not self.handle:
            _check(what="giem2g_rc_create")
            raise Giem2gError("giem2g_rc_create failed")
        self._keep = []

    @classmethod
    def from_model(cls, m, zrecv, x_shift=None, y_shift=None):
        return cls(m.Nx, m.Ny, m.Nz, m.dx, m.dy, m.z, m.thick, zrecv, x_shift, y_shift)

    def receivers(self):
        """(depths used, receiver layers, anomaly cells above each receiver) after PrepareRecvs."""
        z = np.zeros(self.Nr)
        rl = np.zeros(self.Nr, np.int32)
        ac = np.zeros(self.Nr, np.int32)
        _check(lib().giem2g_rc_receivers(self.handle, z.ctypes.data, rl.ctypes.data, ac.ctypes.data), "rc_receivers")
        return z, rl, ac

    def calc_rc_kernel(self, csigma, thick, omega):
        cs = _c128(csigma)
        th = np.ascontiguousarray(thick, dtype=np.float64) if len(thick) else np.zeros(1)
        self._keep = [cs, th]
        bkg = BackgroundT(len(cs) - 1, cs.ctypes.data, th.ctypes.data)
        _check(lib().giem2g_rc_calc_kernel(self.handle, bkg, float(omega)), "giem2g_rc_calc_kernel")

    def calc_fft_of_rc_kernel(self):
        _check(lib().giem2g_rc_calc_fft_of_kernel(self.handle), "giem2g_rc_calc_fft_of_kernel")

    def get_kernel(self):
        """The current tensor (spatial or spectral): complex [2Ny, 2Nx, 15, Nr, Nz]."""
        G = np.zeros((2 * self.Ny, 2 * self.Nx, 15, self.Nr, self.Nz), np.complex128)
        _check(lib().giem2g_rc_get_kernel(self.handle, G.ctypes.data), "giem2g_rc_get_kernel")
        return G

    def set_anomaly_conductivity(self, csiga):
        """csiga: complex [Nz,Ny,Nx] at the kernel's frequency."""
        c = _c128(csiga)
        assert c.size == self.Nx * self.Ny * self.Nz
        _check(lib().giem2g_rc_set_anomaly_conductivity(self.handle, c.ctypes.data), "rc_set_anomaly_conductivity")

    def set_anomaly_sigma(self, siga_file_order, freq, displacement_currents=True):
        from .synthetic import csiga_from_sigma
        self.set_anomaly_conductivity(csiga_from_sigma(siga_file_order, freq, displacement_currents))

    def recalculate(self, E):
        """E [3,Nz,Ny,Nx] (an IE solution) -> anomalous (Ea, Ha), each complex [Ny, Nx, 3, Nr]."""
        Ei = _c128(E)
        assert Ei.size == 3 * self.Nx * self.Ny * self.Nz
        Ea = np.zeros((self.Ny, self.Nx, 3, self.Nr), np.complex128)
        Ha = np.zeros_like(Ea)
        _check(lib().giem2g_rc_recalculate(self.handle, Ei.ctypes.data, Ea.ctypes.data, Ha.ctypes.data),
               "giem2g_rc_recalculate")
        return Ea, Ha

    def recalculate_device(self, d_E: int, d_Ea: int, d_Ha: int):
        with _torch_ordered(self.stream):
            _check(lib().giem2g_rc_recalculate_device(self.handle, d_E, d_Ea, d_Ha), "giem2g_rc_recalculate_device")

    @property
    def stream(self) -> int:
        return lib().giem2g_rc_get_stream(self.handle)

    def delete(self):
        if self.handle:
            lib().giem2g_rc_delete(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass


def _ptrs(xs):
    arr = (ctypes.c_void_p * len(xs))()
    for i, x in enumerate(xs):
        arr[i] = x
    return arr


class Batch:
    """Several independent solves advanced in lockstep (giem2g_batch_*).

    `ops` lists one IEOperator per instance; an operator may appear twice in a row for the two
    polarisations of one frequency (their complex64 applies then share tensor reads).
    """

    def __init__(self, ops, outer_buf=30, inner_buf=10, precision=1, max_restart=100):
        self.ops = list(ops)
        self.n = len(self.ops)
        self._ctl_args = (max_restart, outer_buf, inner_buf, precision)
        ctl = self.ops[0]._ctl(1e-6, max_restart, outer_buf, inner_buf, precision)
        self.handle = lib().giem2g_batch_create(_ptrs([o.handle for o in self.ops]), self.n, ctl)
        if not self.handle:
            _check(what="giem2g_batch_create")

    def _ctl(self, tol):
        mr, ob, ib, pr = self._ctl_args
        return self.ops[0]._ctl(tol, mr, ob, ib, pr)

    def solve_device(self, d_ebkg, d_esol, d_e0=None, tol=1e-6):
        """Device pointers (lists of ints); returns a list of SolveInfo."""
        res = (ResultT * self.n)()
        e0 = _ptrs(d_e0) if d_e0 is not None else None
        with _torch_ordered(self.ops[0].stream):  # the batch runs on its first operator's stream
            rc = lib().giem2g_batch_solve_device(self.handle, _ptrs(d_ebkg), _ptrs(d_esol), e0, self._ctl(tol), res)
        _check(rc, "giem2g_batch_solve_device")
        return [self._info(i, res[i]) for i in range(self.n)]

    def solve(self, E_bkg, E0=None, tol=1e-6):
        """Host arrays (complex128, (3,Nz,Ny,Nx) each); E0 is None or a list whose entries may be None (no
        guess for that instance).  Returns (list of solutions, list of SolveInfo)."""
        ins = [_c128(e) for e in E_bkg]
        outs = [np.empty_like(e) for e in ins]
        e0 = [_c128(e) if e is not None else None for e in E0] if E0 is not None else None
        res = (ResultT * self.n)()
        rc = lib().giem2g_solve_batched(self.handle, _ptrs([a.ctypes.data for a in ins]),
                                        _ptrs([a.ctypes.data for a in outs]),
                                        _ptrs([a.ctypes.data if a is not None else None for a in e0])
                                        if e0 is not None else None,
                                        self._ctl(tol), res)
        _check(rc, "giem2g_solve_batched")
        return outs, [self._info(i, res[i]) for i in range(self.n)]

    def _info(self, i, r):
        return SolveInfo(r.iterations, r.bea, r.be, r.stat, r.applies_fp64, r.applies_fp32, r.device_ms,
                         self.history(i))

    def history(self, i, max_len=4096):
        out = np.zeros(max_len)
        m = lib().giem2g_batch_misfit_history(self.handle, i, out.ctypes.data, max_len)
        return out[:m]

    def delete(self):
        if self.handle:
            lib().giem2g_batch_delete(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.delete()
        except Exception:
            pass


def apply_device_batch(op, d_in, d_out, precision=1):
    """giem2g_apply_ie_operator_device_batch over lists of device pointers."""
    with _torch_ordered(op.stream):
        _check(lib().giem2g_apply_ie_operator_device_batch(op.handle, len(d_in), _ptrs(d_in), _ptrs(d_out),
                                                           precision), "apply_device_batch")


def gemm_bf16_tn(A, B, C=None, accumulate=False, err=None, stream=None):
    """C = A @ B.T on the tcgen05 tensor cores (A [M,K], B [N,K] bf16 CUDA tensors, C [M,N] float32)."""
    import torch
    M, K = A.shape
    N = B.shape[0]
    if C is None:
        C = torch.empty(M, N, dtype=torch.float32, device=A.device)
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    _check(lib().giem2g_gemm_bf16_tn(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, A.stride(0), B.stride(0),
                                     C.stride(0), 1 if accumulate else 0,
                                     err.data_ptr() if err is not None else None, s), "gemm_bf16_tn")
    return C
