"""The C-ABI library loads on a CPU-only machine, exports every symbol include/giem2g.h declares, and
fails loudly (status, message) instead of computing anything without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "giem2g.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(giem2g_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_reference_entry_points():
    names = _declared()
    for ref in ["giem2g_calc_data_sizes", "giem2g_prepare_ie_kernel", "giem2g_calc_ie_kernel",
                "giem2g_calc_fft_of_ie_kernel", "giem2g_set_anomaly_conductivity", "giem2g_apply_ie_operator",
                "giem2g_set_logger", "giem2g_print_stats", "giem2g_delete_ie_operator"]:
        assert ref in names


def test_library_exports_every_declared_symbol(g2lib):
    L = ctypes.CDLL(g2lib.library_path())
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing
    assert set(g2lib.EXPORTED_SYMBOLS) <= set(_declared())


def test_struct_layouts_match_reference(g2lib):
    # BIND(C) layouts of giem2g_interfaces.F90:33-58 on LP64
    assert ctypes.sizeof(g2lib.BackgroundT) == 24
    assert ctypes.sizeof(g2lib.AnomalyT) == 48
    assert ctypes.sizeof(g2lib.DataT) == 4 * 8 + 7 * 8


def test_calc_data_sizes_without_gpu(g2lib):
    z = np.arange(9) * 50.0
    dz = np.diff(z)
    an = g2lib.AnomalyT(32, 32, 8, 100.0, 100.0, z.ctypes.data, dz.ctypes.data)
    d = g2lib.DataT()
    g2lib.lib().giem2g_calc_data_sizes(an, ctypes.byref(d))
    assert g2lib.lib().giem2g_last_status() == 0
    Nx, Ny, Nz = 32, 32, 8
    assert d.ie_kernel_buffer_length == (2 * Nz * (Nz + 1) + 2 * Nz * Nz) * Nx * Ny
    assert d.fft_buffers_length == 2 * Nx * 3 * Nz * 2 * Ny
    assert d.giem2g_tensor


def test_no_cpu_fallback(g2lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(g2lib.Giem2gError):
        g2lib.IEOperator(4, 4, 2, 10.0, 10.0, np.array([0.0, 5.0, 10.0]))


def test_unsupported_shape_rejected(g2lib):
    z = np.arange(3) * 5.0
    dz = np.diff(z)
    an = g2lib.AnomalyT(6, 4, 2, 10.0, 10.0, z.ctypes.data, dz.ctypes.data)
    d = g2lib.DataT()
    g2lib.lib().giem2g_calc_data_sizes(an, ctypes.byref(d))
    g2lib.lib().giem2g_prepare_ie_kernel(an, d)
    assert g2lib.lib().giem2g_last_status() != 0
    assert b"powers of two" in g2lib.lib().giem2g_last_error() or b"CUDA" in g2lib.lib().giem2g_last_error()
