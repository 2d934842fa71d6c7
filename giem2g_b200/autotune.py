"""Autotuner for the contraction tile shape.

The contraction kernel has several compile-time tile shapes (j-slices per unit, units per stage,
pipeline depth) per precision and Nz (giem2g_contract_variants; precision 2 is the paired complex64
apply of two vectors).  The best one depends on Nz, the
precision and the grid, so the tuner times every variant with CUDA events on the operator's own
buffers and keeps the fastest in the operator; results are cached per (Nx, Ny, Nz, precision) in a JSON
file next to this module when one is given.  Each candidate is timed in `rounds` rounds of `reps` full
applies and scored by its fastest round, so a transient slowdown (another process, a clock dip) during
one round does not decide the pick.
"""
from __future__ import annotations

import json
import os


def _time_rounds(run, stream, reps: int, rounds: int) -> float:
    """Fastest of `rounds` CUDA-event timings of `reps` calls of run() (ms per call), after 2 warm-up calls."""
    import torch
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):  # the calls run back to back on the operator's stream
        for _ in range(2):
            run()
    best = None
    for _ in range(rounds):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(reps):
                run()
            e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        best = ms if best is None else min(best, ms)
    return best


def autotune_contraction(op, reps: int = 5, cache_path: str | None = None, rounds: int = 3) -> dict:
    import torch

    key = f"{op.Nx}x{op.Ny}x{op.Nz}"
    cache = {}
    if cache_path and os.path.exists(cache_path):
        try:
            cache = json.load(open(cache_path))
        except Exception:
            cache = {}
    stream = torch.cuda.ExternalStream(op.stream)
    picks = {}
    from . import apply_device_batch
    for prec, dt in ((0, torch.complex128), (1, torch.complex64), (2, torch.complex64)):
        nv = op.contract_variants(prec)
        if nv <= 1:
            picks[prec] = {"variant": 0, "ms": None}
            continue
        ck = f"{key}:{prec}"
        if ck in cache:
            op.set_contract_variant(prec, cache[ck]["variant"])
            picks[prec] = cache[ck]
            continue
        x = torch.randn(op.nvec, dtype=dt, device="cuda")
        y = torch.empty_like(x)
        x2, y2 = torch.randn_like(x), torch.empty_like(x)

        def run():
            if prec == 2:  # paired complex64 apply: two vectors per tensor read
                apply_device_batch(op, [x.data_ptr(), x2.data_ptr()], [y.data_ptr(), y2.data_ptr()], 1)
            else:
                op.apply_device(x.data_ptr(), y.data_ptr(), prec)

        best, all_ms = None, []
        for v in range(nv):
            op.set_contract_variant(prec, v)
            ms = _time_rounds(run, stream, reps, rounds)
            all_ms.append(round(ms, 5))
            if best is None or ms < best[1]:
                best = (v, ms)
        op.set_contract_variant(prec, best[0])
        picks[prec] = {"variant": best[0], "ms": best[1], "all_ms": all_ms}
        cache[ck] = picks[prec]
    # FFT lines per CTA, per precision: complex64 timed on the paired apply (the inner solver's), complex128
    # on the FP64 apply; the shared-memory tile per line doubles with the element size, so they can differ
    def time_lines(prec, run):
        best, all_ms = None, []
        for lines in (32, 16, 8):
            op.set_fft_lines(lines, precision=prec)
            ms = _time_rounds(run, stream, reps, rounds)
            all_ms.append(round(ms, 5))
            if best is None or ms < best[1]:
                best = (lines, ms)
        op.set_fft_lines(best[0], precision=prec)
        return {"lines": best[0], "ms": best[1], "all_ms": all_ms}

    x = torch.randn(op.nvec, dtype=torch.complex64, device="cuda")
    x2, y, y2 = torch.randn_like(x), torch.empty_like(x), torch.empty_like(x)
    picks["fft_lines"] = time_lines(1, lambda: apply_device_batch(op, [x.data_ptr(), x2.data_ptr()],
                                                                  [y.data_ptr(), y2.data_ptr()], 1))
    xd = torch.randn(op.nvec, dtype=torch.complex128, device="cuda")
    yd = torch.empty_like(xd)
    picks["fft_lines64"] = time_lines(0, lambda: op.apply_device(xd.data_ptr(), yd.data_ptr(), 0))
    op.check_device_error()
    if cache_path:
        try:
            json.dump(cache, open(cache_path, "w"), indent=1)
        except Exception:
            pass
    return {str(k): v for k, v in picks.items()}


def pin_contraction(op, spec: str) -> dict:
    """Set the tile shapes by hand instead of timing them: spec = "v64,v32,vpair[,fft_lines[,fft_lines64]]"
    (the numbers the tuner reports; one FFT lines value sets both precisions, a second one complex128's).
    Profilers need it, because timings taken under a profiler pick other shapes than the plain run does."""
    parts = [int(t) for t in spec.split(",")]
    if len(parts) not in (3, 4, 5):
        raise ValueError("expected v64,v32,vpair[,fft_lines[,fft_lines64]]")
    picks = {}
    for prec, v in enumerate(parts[:3]):
        if op.contract_variants(prec) > 1:
            if not 0 <= v < op.contract_variants(prec):
                raise ValueError(f"variant {v} out of range for precision {prec}")
            op.set_contract_variant(prec, v)
        picks[str(prec)] = {"variant": v, "ms": None, "pinned": True}
    if len(parts) >= 4:
        op.set_fft_lines(parts[3])
        picks["fft_lines"] = {"lines": parts[3], "ms": None, "pinned": True}
        picks["fft_lines64"] = {"lines": parts[3], "ms": None, "pinned": True}
    if len(parts) == 5:
        op.set_fft_lines(parts[4], precision=0)
        picks["fft_lines64"] = {"lines": parts[4], "ms": None, "pinned": True}
    return picks
