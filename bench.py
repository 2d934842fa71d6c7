#!/usr/bin/env python
"""Benchmark of the IE solve at 128x128x32 on B200 (one JSON line on rank 0).

Workload: the 128x128x32 anomaly (50 x 50 x 25 m cells) over the 3-layer background, seeded
Gaussian-random-field conductivity (log10 sigma mean -2, std 0.7, correlation 400 m), 0.1 Hz,
plane-wave sources of both polarisations.  One step = solving both polarisations to outer relative
residual 1e-6 with the nested FGMRES (outer 30 / inner 10) in mixed precision (complex64 inner
GMRES, FFTs and tensor; FP64 outer Arnoldi, Hessenberg, residual and true-residual check), the two
polarisations as one batch (lockstep solves whose complex64 applies share each tensor read).
`value` = whole-job polarisation solves per second with everything resident in HBM; `e2e` = the
same through the C ABI (giem2g_solve_batched) with pinned host inputs/outputs copied every step.
Multi-GPU: independent replicas (one process per GPU, no data-path collective); the only
communication is the barrier and the max-over-ranks of the timing.

--impl reference: the reference's CPU path.  The Fortran/MPI/FFTW reference cannot be built on
this image, so the CPU restatement in oracle/ (FP64, OpenMP on all host cores) is timed instead.
Set-up solves both polarisations in full once (their outer-iteration counts and times).  Each step
is one outer FGMRES iteration (a bounded sample: the initial residual, 13 applies of the outer
iteration, the final true residual) of one polarisation, alternating EY and EX; the solve time it
stands for counts the two residual applies once and the outer iteration n_outer times:
t_solve = n_outer * (t_sample - 2 t_apply) + 2 t_apply, with t_apply the oracle's apply timed in
set-up.  The line reports the full solves' own rate beside it.

Profiler workloads (no JSON contract; one line of timings):
  --apply-only      a few IE applies at a given grid (kernels k_fx, k_fy, contraction, k_by, k_bx)
  --receivers-only  the receiver-field tensor build and a few recalculations
  --step-breakdown  warm per-kernel device times of one batched step
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve time & IE-apply HBM GB/s at 128×128×32: FP64 vs mixed+learned, rel.res 1e-6"
UNIT = "solves/s"
TOL = 1e-6
OUTER, INNER, MAXRESTART = 30, 10, 100


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def _algorithmic_bytes(Nx, Ny, Nz, S):
    """B_apply = S*(T + 2*N_vec + NxNy*Nz): tensor read, x read + y write, one coefficient per cell."""
    T = Nx * Ny * (2 * Nz * (Nz + 1) + 2 * Nz * Nz)
    nvec = 3 * Nx * Ny * Nz
    return S * (T + 2 * nvec + Nx * Ny * Nz)


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for i, n in enumerate(names):
                    if r[5 + i].lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _profiles_traffic():
    """DRAM traffic per FP64 apply from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "ie_apply_128x128x32.md")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_apply_fp64:"):
                return int(float(line.split(":")[1]))
    except Exception:
        pass
    return None


# ------------------------------------------------------------------------------------------------
def build_problem():
    from giem2g_b200.synthetic import config_c2
    from giem2g_b200.sources import plane_wave_integral
    m, sig = config_c2(seed=2024)
    e_y = plane_wave_integral(m, 1)
    e_x = plane_wave_integral(m, 0)
    return m, sig, e_y, e_x


def cpu_solve_estimate(m, sig, sh, ah, n_outer, nthreads):
    """One outer FGMRES iteration of the oracle's FP64 solver (a bounded sample of the solve: initial residual,
    one outer iteration, final true residual) and the solve time it stands for, n_outer*(t - 2 t_apply) +
    2 t_apply, with the oracle's apply timed alongside.  Returns (sample s, apply s, applies, solve s)."""
    import oracle
    from giem2g_b200.synthetic import csiga_from_sigma
    from giem2g_b200.sources import plane_wave_integral
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = oracle.background_cells(m)
    E0 = plane_wave_integral(m, 1)
    t = time.perf_counter()
    for _ in range(2):
        oracle.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, nthreads=nthreads)
    t_apply = (time.perf_counter() - t) / 2
    t = time.perf_counter()
    _, info, _ = oracle.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, E0, None, 1, INNER, 1, TOL,
                              nthreads=nthreads)
    dt = time.perf_counter() - t
    return dt, t_apply, info.applies, n_outer * (dt - 2.0 * t_apply) + 2.0 * t_apply


WORKLOAD = ("IE solve 128x128x32 (50x50x25 m cells), 3-layer background, 0.1 Hz, pols EY+EX, nested FGMRES 30/10, "
            "outer rel.res 1e-6")


def _config(world):
    """The config both arms print: the problem, its parallel layout and the L2 note (nothing arm-specific)."""
    return {"workload": WORKLOAD, "parallelism": f"replicas x{world}",
            "l2": "working set > L2 (tensor 545 MB c64 + 1.09 GB c128)"}


def run_reference(args, rank, world):
    if rank != 0:
        print(json.dumps({"impl": "reference", "rank": rank, "skipped": "rank 0 runs the CPU reference"}),
              file=sys.stderr)
        return 0
    import oracle
    from giem2g_b200.synthetic import csiga_from_sigma
    oracle.build()
    ncores = os.cpu_count() or 1
    m, sig, e_y, e_x = build_problem()
    t0 = time.perf_counter()
    S, A = oracle.green_tensor(m, nthreads=ncores)
    sh, ah = oracle.tensor_spectrum(m.Nx, m.Ny, m.Nz, S, A, nthreads=ncores)
    del S, A
    t_setup = time.perf_counter() - t0
    csiga = csiga_from_sigma(sig, m.freq)
    csigb, sqsigb = oracle.background_cells(m)
    # the oracle's apply alone (the two residual applies a sample holds once per solve)
    v = np.ascontiguousarray(e_y)
    oracle.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v, nthreads=ncores)
    t0 = time.perf_counter()
    for _ in range(3):
        oracle.apply(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, v, nthreads=ncores)
    t_apply = (time.perf_counter() - t0) / 3
    # full solves of both polarisations: outer-iteration counts and the true solve times (after one untimed
    # full solve: the first solve of a process also pays its thread start-up and first touches of the work space)
    pols = [("EY", e_y), ("EX", e_x)]
    oracle.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, e_y, None, OUTER, INNER, MAXRESTART, TOL,
                 nthreads=ncores)
    n_outer, t_full, applies = [], [], []
    for _, rhs in pols:
        t0 = time.perf_counter()
        _, info, _ = oracle.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, rhs, None, OUTER, INNER,
                                  MAXRESTART, TOL, nthreads=ncores)
        t_full.append(time.perf_counter() - t0)
        n_outer.append(max(1, info.iterations))
        applies.append(info.applies)

    def sample(i):
        _, rhs = pols[i % 2]
        t = time.perf_counter()
        oracle.solve(m.Nx, m.Ny, m.Nz, sh, ah, csiga, csigb, sqsigb, m.dz, rhs, None, 1, INNER, 1, TOL,
                     nthreads=ncores)
        dt = time.perf_counter() - t
        n = n_outer[i % 2]
        return dt, n * (dt - 2.0 * t_apply) + 2.0 * t_apply

    for i in range(args.warmup):
        sample(i)
    t_solves, samples = 0.0, []
    for i in range(args.steps):
        dt, ts = sample(i)
        samples.append(dt)
        t_solves += ts
    value = args.steps / t_solves
    full_value = len(pols) / sum(t_full)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_solves / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded GRF conductivity, plane-wave sources)",
        "config": _config(world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "port",
                         "sample": f"{args.steps} outer FGMRES iterations, EY and EX alternating (1 + 13 + 1 FP64 "
                                   f"applies each, mean {np.mean(samples):.2f} s) of the oracle solver on {ncores} "
                                   f"threads; each stands for one full solve of n_outer = {n_outer} outer "
                                   f"iterations: n_outer*(sample - 2 t_apply) + 2 t_apply, t_apply = "
                                   f"{t_apply:.3f} s"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_setup_s": t_setup, "reference_full_solve_s": t_full, "reference_full_solve_value": full_value,
        "reference_outer_iterations": n_outer, "reference_applies": applies, "reference_apply_s": t_apply,
        "note": "Fortran/MPI/FFTW reference is not buildable on this image; the CPU restatement (oracle/) is timed. "
                "precision: complex128 throughout (the reference has no other)",
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------
def run_b200(args, rank, world, local_rank):
    import torch
    import giem2g_b200 as g2
    from giem2g_b200.synthetic import csiga_from_sigma
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        import datetime
        dist = dist_mod
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        from giem2g_b200.replicas import max_over_ranks as mor
        return mor(x, device=dev)

    g2.set_logger(lambda msg: print(msg, file=sys.stderr))  # stdout carries the one JSON line
    m, sig, e_y, e_x = build_problem()
    op = g2.IEOperator.from_model(m)
    t0 = time.perf_counter()
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    op.calc_fft_of_ie_kernel()
    torch.cuda.synchronize()
    t_tensor = time.perf_counter() - t0
    op.set_anomaly_sigma(sig, m.freq)
    stream = torch.cuda.ExternalStream(op.stream)
    n = op.nvec
    d_ey = torch.from_numpy(np.ascontiguousarray(e_y).ravel()).to(dev)
    d_ex = torch.from_numpy(np.ascontiguousarray(e_x).ravel()).to(dev)
    d_sol_y = torch.empty_like(d_ey)
    d_sol_x = torch.empty_like(d_ex)

    # contraction tile shape: time the variants once (autotuner) and keep the fastest
    from giem2g_b200.autotune import autotune_contraction, pin_contraction
    tuned = pin_contraction(op, args.variants) if args.variants else autotune_contraction(op)

    def solve_pair(prec, tol=TOL):
        iy = op.solve_device(d_ey.data_ptr(), d_sol_y.data_ptr(), None, tol=tol, max_restart=MAXRESTART,
                             outer_buf=OUTER, inner_buf=INNER, precision=prec)
        ix = op.solve_device(d_ex.data_ptr(), d_sol_x.data_ptr(), None, tol=tol, max_restart=MAXRESTART,
                             outer_buf=OUTER, inner_buf=INNER, precision=prec)
        return iy, ix

    # FP64 reference solves (plain path) for the comparison and the field error
    iy64, ix64 = solve_pair(0, tol=1e-8)
    ref_y, ref_x = d_sol_y.clone(), d_sol_x.clone()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    iy64b, ix64b = solve_pair(0, tol=TOL)
    ev1.record(stream)
    torch.cuda.synchronize()
    fp64_pair_ms = ev0.elapsed_time(ev1)

    # the learned outer preconditioner (trained on 64x64x16 C4 models) on the EY solve: warm start of the
    # inner cycle (mode 1) and alone (mode 2, with the solver's fallback to the plain inner GMRES)
    learned = None
    try:
        from giem2g_b200.learned import WEIGHTS, LearnedPreconditioner, UNet3D
        if os.path.exists(WEIGHTS):
            net = UNet3D.from_file(WEIGHTS)
            pre = LearnedPreconditioner(net, m, sig)
            learned = {"weights": os.path.relpath(WEIGHTS, ROOT)}
            for label, mode in (("net_warm_start", 1), ("net_only_with_fallback", 2)):
                pre.attach(op, mode)
                op.solve_device(d_ey.data_ptr(), d_sol_y.data_ptr(), None, tol=TOL, max_restart=MAXRESTART,
                                outer_buf=OUTER, inner_buf=INNER, precision=1)
                li = op.solve_device(d_ey.data_ptr(), d_sol_y.data_ptr(), None, tol=TOL, max_restart=MAXRESTART,
                                     outer_buf=OUTER, inner_buf=INNER, precision=1)
                learned[label] = {"outer_iterations": li.iterations, "net_steps": li.precond_steps,
                                  "ms": li.device_ms, "true_rel_residual": li.be}
            op.set_outer_preconditioner(0)
    except Exception as exc:  # reported, never the headline
        learned = {"error": str(exc)}
        op.set_outer_preconditioner(0)

    # mixed precision, one polarisation after the other (the reference's order); one untimed pair first
    # (work-space reallocation for the precision change, graph capture)
    solve_pair(1)
    torch.cuda.synchronize()
    ev0.record(stream)
    iy_s, ix_s = solve_pair(1)
    ev1.record(stream)
    torch.cuda.synchronize()
    mixed_seq_pair_ms = ev0.elapsed_time(ev1)

    # the product path: both polarisations as one batch (lockstep FGMRES, paired complex64 applies)
    batch = g2.Batch([op, op], outer_buf=OUTER, inner_buf=INNER, precision=1, max_restart=MAXRESTART)
    d_in, d_out = [d_ey.data_ptr(), d_ex.data_ptr()], [d_sol_y.data_ptr(), d_sol_x.data_ptr()]

    def solve_batch():
        return batch.solve_device(d_in, d_out, tol=TOL)

    for _ in range(args.warmup):
        solve_batch()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = g2.kernel_launch_count()
    infos = []
    with ClockSampler(local_rank) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            infos.append(solve_batch())
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = g2.kernel_launch_count() - launches0
    barrier()
    t_dev = ev0.elapsed_time(ev1) / 1e3
    t_max = max_over_ranks(t_dev)
    value = 2.0 * args.steps * world / t_max
    iy, ix = infos[-1]
    err_y = (torch.linalg.vector_norm(d_sol_y - ref_y) / torch.linalg.vector_norm(ref_y)).item()
    err_x = (torch.linalg.vector_norm(d_sol_x - ref_x) / torch.linalg.vector_norm(ref_x)).item()

    # end to end through the public C ABI (giem2g_solve_batched) with pinned host buffers:
    # H2D of both right-hand sides + solve + D2H of both solutions each step
    h_ey = torch.from_numpy(np.ascontiguousarray(e_y)).pin_memory()
    h_ex = torch.from_numpy(np.ascontiguousarray(e_x)).pin_memory()
    h_oy = torch.empty_like(h_ey).pin_memory()
    h_ox = torch.empty_like(h_ex).pin_memory()
    res = (g2.ResultT * 2)()
    ins, outs = g2._ptrs([h_ey.data_ptr(), h_ex.data_ptr()]), g2._ptrs([h_oy.data_ptr(), h_ox.data_ptr()])
    for _ in range(args.warmup):  # untimed: the first call allocates the batch's staging buffers
        if g2.lib().giem2g_solve_batched(batch.handle, ins, outs, None, batch._ctl(TOL), res) != 0:
            raise RuntimeError(g2.lib().giem2g_last_error().decode())
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        rc = g2.lib().giem2g_solve_batched(batch.handle, ins, outs, None, batch._ctl(TOL), res)
        if rc != 0:
            raise RuntimeError(g2.lib().giem2g_last_error().decode())
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e_value = 2.0 * args.steps * world / t_e2e
    vec_bytes = n * 16

    # apply roofline: FP64 and complex64 applies timed with CUDA events on the operator's stream
    def time_apply(prec, reps=20):
        dt = torch.complex128 if prec == 0 else torch.complex64
        x = torch.randn(n, dtype=dt, device=dev)
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):  # back-to-back applies, no wait on another stream between them
            for _ in range(3):
                op.apply_device(x.data_ptr(), y.data_ptr(), prec)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(reps):
                op.apply_device(x.data_ptr(), y.data_ptr(), prec)
            a1.record(stream)
        torch.cuda.synchronize()
        return a0.elapsed_time(a1) / reps

    ms64 = time_apply(0)
    ms32 = time_apply(1)

    def time_pair(reps=20):
        xs = [torch.randn(n, dtype=torch.complex64, device=dev) for _ in range(2)]
        ys = [torch.empty_like(x) for x in xs]
        pi, po = [x.data_ptr() for x in xs], [y.data_ptr() for y in ys]
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for _ in range(3):
                g2.apply_device_batch(op, pi, po, 1)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(reps):
                g2.apply_device_batch(op, pi, po, 1)
            a1.record(stream)
        torch.cuda.synchronize()
        return a0.elapsed_time(a1) / reps

    ms32_pair = time_pair()

    # the contraction alone: CUDA events on the operator's stream around its launch inside eager applies
    # (single FP64, single complex64, and the paired complex64 form the batched step runs)
    def time_contract(prec, reps=20, pair=False):
        dt = torch.complex128 if prec == 0 else torch.complex64
        xs = [torch.randn(n, dtype=dt, device=dev) for _ in range(2 if pair else 1)]
        ys = [torch.empty_like(x) for x in xs]
        op.set_kernel_timing(True)
        ts = []
        for i in range(reps + 3):
            if pair:
                g2.apply_device_batch(op, [x.data_ptr() for x in xs], [y.data_ptr() for y in ys], 1)
            else:
                op.apply_device(xs[0].data_ptr(), ys[0].data_ptr(), prec)
            if i >= 3:
                ts.append(op.last_contract_ms())
        op.set_kernel_timing(False)
        return float(np.mean(ts))

    mc64, mc32, mcp = time_contract(0), time_contract(1), time_contract(1, pair=True)
    B64 = _algorithmic_bytes(m.Nx, m.Ny, m.Nz, 16)
    B32 = _algorithmic_bytes(m.Nx, m.Ny, m.Nz, 8)
    TB64 = 16 * m.Nx * m.Ny * (2 * m.Nz * (m.Nz + 1) + 2 * m.Nz * m.Nz)  # tensor bytes per apply (FP64)
    # two vectors sharing one tensor read: S*[T + 2*(2*N_vec + NxNy*Nz)]
    B32P = 2 * B32 - 8 * m.Nx * m.Ny * (2 * m.Nz * (m.Nz + 1) + 2 * m.Nz * m.Nz)
    peaks = _peaks()
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    if not peak:
        peak = 6650.0
    ach64 = B64 / (ms64 * 1e-3) / 1e9
    ach32 = B32 / (ms32 * 1e-3) / 1e9
    # paired complex64 contraction: the tensor read once for two vectors, and its FP32 arithmetic counted as
    # 4-multiply complex multiply-adds (8 flops) -- 9 Nz x Nz blocks at 4 points per (kx, ky) pair, 2 vectors --
    # against the nominal FP32 FMA peak (148 SMs x 128 lanes x 2 flops x the maximum SM clock)
    TB32 = TB64 // 2
    flops_pair = 2 * 8 * 9 * m.Nz * m.Nz * 4 * m.Nx * m.Ny
    props = torch.cuda.get_device_properties(dev)
    fp32_peak = props.multi_processor_count * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12

    # receiver fields (the reference's "Recalculate Fields") for one line of surface receivers on this grid:
    # receiver tensor build + its spectrum (once per frequency) and one recalculation (per solution)
    def time_receivers(reps=10):
        rcop = g2.RCOperator.from_model(m, [0.0])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rcop.calc_rc_kernel(m.csigma, m.thick, m.omega)
        t1 = time.perf_counter()
        rcop.calc_fft_of_rc_kernel()
        t2 = time.perf_counter()
        rcop.set_anomaly_sigma(sig, m.freq)
        E = torch.randn(n, dtype=torch.complex128, device=dev)
        Ea = torch.empty(3 * m.Nx * m.Ny, dtype=torch.complex128, device=dev)
        Ha = torch.empty_like(Ea)
        rst = torch.cuda.ExternalStream(rcop.stream)
        for _ in range(3):
            rcop.recalculate_device(E.data_ptr(), Ea.data_ptr(), Ha.data_ptr())
        torch.cuda.synchronize()
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(rst)
        for _ in range(reps):
            rcop.recalculate_device(E.data_ptr(), Ea.data_ptr(), Ha.data_ptr())
        r1.record(rst)
        torch.cuda.synchronize()
        ms = r0.elapsed_time(r1) / reps
        rcop.delete()
        tb = 4 * m.Nx * m.Ny * 15 * m.Nz * 16  # spectral receiver tensor, read once per recalculation
        io = 16 * (n + 2 * 3 * m.Nx * m.Ny + m.Nx * m.Ny * m.Nz)  # E in, Ea and Ha out, dsig
        return {"receivers": 1, "tensor_build_s": t1 - t0, "tensor_fft_s": t2 - t1, "recalculate_ms": ms,
                "bytes_per_recalculate": tb + io, "achieved_gbs": (tb + io) / (ms * 1e-3) / 1e9}

    rcv = time_receivers() if rank == 0 else None

    # the batched multi-frequency sweep on this grid: 8 frequencies (1e-3 .. 1e2 Hz) x 2 polarisations = 16
    # lockstep instances in mixed precision, against the same 16 solved one after the other in plain FP64
    sweep = None
    if rank == 0 and not args.no_sweep:
        try:
            from giem2g_b200.sweep import run_sweep
            res = run_sweep(m, sig, list(np.logspace(-3, 2, 8)), tol=TOL, compare=True, tuned=tuned)
            sweep = {"instances": len(res["batched"]["iterations"]), "freqs_hz": res["freqs"],
                     "batched_mixed_ms": res["batched"]["device_ms"],
                     "sequential_mixed_ms": res["sequential_mixed"]["device_ms"],
                     "sequential_fp64_ms": res["sequential_fp64"]["device_ms"],
                     "speedup_vs_sequential_fp64": res["speedup_batched_vs_sequential_fp64"],
                     "outer_iterations": res["batched"]["iterations"], "stat": res["batched"]["stat"],
                     "max_field_error_vs_fp64": max(res["field_error_vs_fp64"]),
                     "setup_s_per_frequency": res["setup_s_per_frequency"]}
        except Exception as exc:  # reported, never the headline
            sweep = {"error": str(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            oracle.build()
            sh, ah = op.get_ie_kernel_spectral()
            ncores = os.cpu_count() or 1
            n_it = max(1, iy64b.iterations)
            dt, t_ap, applies, t_solve = cpu_solve_estimate(m, sig, sh, ah, n_it, ncores)
            cpu = {"value": 1.0 / t_solve, "unit": UNIT, "cores": ncores, "kind": "port",
                   "sample": f"one outer FGMRES iteration ({applies} FP64 applies incl. the initial and final "
                             f"residual) of the oracle solver at 128x128x32 on {ncores} threads = {dt:.2f} s, "
                             f"apply {t_ap:.3f} s; solve = {n_it} outer iterations (FP64, tol 1e-6): "
                             f"{n_it}*(sample - 2 apply) + 2 apply = {t_solve:.1f} s"}
        except Exception as exc:  # the CPU baseline is reported, never the target
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 inner / c128 outer",
            "data": "synthetic (seeded GRF conductivity, plane-wave sources)",
            "config": _config(world),
            "setup": {"tensor_build_s": t_tensor, "contract_variants": tuned,
                      "method": "mixed precision (c64 inner GMRES/FFTs/tensor, c128 outer), both polarisations as "
                                "one lockstep batch"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * vec_bytes,
                    "d2h_bytes_per_step": 2 * vec_bytes},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": ach64, "peak": peak, "unit": "GB/s", "frac": ach64 / peak,
                         "traffic": _profiles_traffic(), "kernel": "FP64 IE apply (5 kernels; contraction dominant)",
                         "bytes_per_launch": B64, "ms_per_launch": ms64, "peak_source": peak_src},
            "dominant_kernel": {
                "kernel": "paired complex64 Green's-tensor contraction (two vectors per tensor read; the batched "
                          "step's inner applies), autotuned shape in setup.contract_variants[2]",
                "ms": mcp, "bytes_per_launch": TB32, "achieved_gbs": TB32 / (mcp * 1e-3) / 1e9,
                "frac_hbm": TB32 / (mcp * 1e-3) / 1e9 / peak,
                "flops_per_launch": flops_pair, "achieved_tflops": flops_pair / (mcp * 1e-3) / 1e12,
                "fp32_peak_tflops_nominal": fp32_peak,
                "frac_fp32": flops_pair / (mcp * 1e-3) / 1e12 / fp32_peak,
                "single_fp64": {"ms": mc64, "bytes": TB64, "achieved_gbs": TB64 / (mc64 * 1e-3) / 1e9,
                                "frac_hbm": TB64 / (mc64 * 1e-3) / 1e9 / peak},
                "single_c64": {"ms": mc32, "bytes": TB32, "achieved_gbs": TB32 / (mc32 * 1e-3) / 1e9,
                               "frac_hbm": TB32 / (mc32 * 1e-3) / 1e9 / peak},
                "note": "algorithmic bytes = the tensor read once (T*S); the spectrum in/out is intermediate; "
                        "flops = 4-multiply complex count (the kernels use the 3-multiply form)"},
            "apply_c64": {"ms": ms32, "achieved_gbs": ach32, "frac": ach32 / peak, "bytes": B32},
            "apply_c64_pair": {"ms": ms32_pair, "bytes": B32P, "achieved_gbs": B32P / (ms32_pair * 1e-3) / 1e9,
                               "frac": B32P / (ms32_pair * 1e-3) / 1e9 / peak},
            "solve": {"mixed_batched_pair_ms": t_max / args.steps * 1e3, "mixed_sequential_pair_ms": mixed_seq_pair_ms,
                      "fp64_pair_ms": fp64_pair_ms,
                      "speedup_vs_fp64_gpu": fp64_pair_ms / (t_max / args.steps * 1e3),
                      "outer_iterations_mixed": [iy.iterations, ix.iterations],
                      "outer_iterations_mixed_sequential": [iy_s.iterations, ix_s.iterations],
                      "outer_iterations_fp64": [iy64b.iterations, ix64b.iterations],
                      "applies_mixed": [iy.applies_fp64 + iy.applies_fp32, ix.applies_fp64 + ix.applies_fp32],
                      "true_rel_residual_mixed": [iy.be, ix.be],
                      "field_error_vs_fp64_tol1e-8": [err_y, err_x]},
            "learned_preconditioner": learned,
            "receiver_fields": rcv,
            "sweep_8freq_x2pol": sweep,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    batch.delete()
    op.delete()
    if dist:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------------
def run_apply_only(args):
    """A few IE applies at one grid on the operator's stream (the workload the apply profiles capture): the
    seeded random-field model of config_grf (seed 7), the GPU Green's tensor and its spectrum, then
    `--reps` applies of one vector (or two with --nv 2, the paired complex64 form) after `--warmup` untimed
    ones.  Prints one line of CUDA-event timings."""
    import torch
    import giem2g_b200 as g2
    from giem2g_b200.synthetic import config_grf

    m, sig = config_grf(args.nx, args.ny or args.nx, args.nz, seed=7)
    t0 = time.perf_counter()
    op = g2.IEOperator.from_model(m)
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    op.calc_fft_of_ie_kernel()
    torch.cuda.synchronize()
    t_build = time.perf_counter() - t0
    op.set_anomaly_sigma(sig, m.freq)
    if args.variant is not None:
        op.set_contract_variant(2 if args.nv == 2 else args.prec, args.variant)
    if args.fft_lines is not None:
        op.set_fft_lines(args.fft_lines)
    dt = torch.complex128 if args.prec == 0 else torch.complex64
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(op.nvec, dtype=dt, device="cuda", generator=g)
    y = torch.empty_like(x)
    x2, y2 = torch.randn_like(x), torch.empty_like(x)
    stream = torch.cuda.ExternalStream(op.stream)

    def one():
        if args.nv == 2:
            g2.apply_device_batch(op, [x.data_ptr(), x2.data_ptr()], [y.data_ptr(), y2.data_ptr()], args.prec)
        else:
            op.apply_device(x.data_ptr(), y.data_ptr(), args.prec)

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            one()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.reps):
            one()
        e1.record(stream)
    torch.cuda.synchronize()
    op.check_device_error()
    form = 2 if args.nv == 2 else args.prec
    print(json.dumps({"mode": "apply-only", "grid": [m.Nx, m.Ny, m.Nz], "precision": args.prec, "nv": args.nv,
                      "variant": args.variant, "variants": op.contract_variants(form), "reps": args.reps,
                      "ms_per_apply": e0.elapsed_time(e1) / args.reps, "tensor_build_s": t_build}))
    op.delete()
    return 0


def run_learned_only(args):
    """The learned preconditioner's network (the committed weights) on one seeded input of the grid: `--reps`
    inferences after `--warmup` untimed ones, CUDA events on torch's current stream (where the convolution
    GEMMs run).  Reports ms per inference and the GEMM flops: per layer 2 x output voxels x Cout x K, with K
    the stored (padded) 27 x Cin columns the tensor cores multiply."""
    import torch
    from giem2g_b200.learned import CIN, WEIGHTS, UNet3D, _kp

    nz, ny, nx = args.nz, args.ny or args.nx, args.nx
    net = UNet3D.from_file(WEIGHTS)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(1, nz, ny, nx, CIN, device="cuda", generator=g)
    level = {"in": 0, "e0": 0, "d1": 1, "e1": 1, "d2": 2, "e2": 2, "d3": 3, "b": 3, "u2": 2, "u1": 1, "u0": 0,
             "out": 0}
    flops = 0
    for name, cin, cout, _ in UNet3D.LAYERS:
        lv = level[name]
        flops += 2 * (nz >> lv) * (ny >> lv) * (nx >> lv) * cout * _kp(cin)
    with torch.no_grad():
        for _ in range(args.warmup):
            net(x)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.reps):
            net(x)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    print(json.dumps({"mode": "learned-only", "grid": [nx, ny, nz], "reps": args.reps, "ms_per_inference": ms,
                      "gemm_gflop_per_inference": flops / 1e9, "gemm_tflops_over_inference": flops / (ms * 1e-3) / 1e12}))
    return 0


def run_receivers_only(args):
    """Receiver fields at one grid (the workload the receiver profile captures): the receiver tensor of `--nr`
    receiver depths on the config_grf model (seed 7), its spectrum, and `--reps` recalculations of a seeded
    random field after `--warmup` untimed ones.  Prints one line of timings."""
    import torch
    import giem2g_b200 as g2
    from giem2g_b200.synthetic import config_grf

    m, sig = config_grf(args.nx, args.ny or args.nx, args.nz, seed=7)
    depths = [0.0, float(m.z[-1]) + 50.0, 1000.0, 150.0][: args.nr] + [0.0] * max(0, args.nr - 4)
    rc = g2.RCOperator.from_model(m, depths)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc.calc_rc_kernel(m.csigma, m.thick, m.omega)
    t1 = time.perf_counter()
    rc.calc_fft_of_rc_kernel()
    t2 = time.perf_counter()
    rc.set_anomaly_sigma(sig, m.freq)
    nv = 3 * m.Nx * m.Ny * m.Nz
    E = torch.randn(nv, dtype=torch.complex128, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    Ea = torch.empty(3 * m.Nx * m.Ny * args.nr, dtype=torch.complex128, device="cuda")
    Ha = torch.empty_like(Ea)
    stream = torch.cuda.ExternalStream(rc.stream)
    for _ in range(args.warmup):
        rc.recalculate_device(E.data_ptr(), Ea.data_ptr(), Ha.data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.reps):
        rc.recalculate_device(E.data_ptr(), Ea.data_ptr(), Ha.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    print(json.dumps({"mode": "receivers-only", "grid": [m.Nx, m.Ny, m.Nz], "receivers": args.nr,
                      "tensor_build_s": t1 - t0, "tensor_fft_s": t2 - t1,
                      "recalculate_ms": e0.elapsed_time(e1) / max(1, args.reps)}))
    rc.delete()
    return 0


def run_step_breakdown(args):
    """Warm per-kernel device times of one batched benchmark step (the CUPTI activity trace torch.profiler
    records; every kernel of the process, this library's included), with the step's CUDA-event time taken
    without the profiler and the idle gaps between kernels.  Prints one JSON line."""
    import collections
    import torch
    import giem2g_b200 as g2
    from giem2g_b200.autotune import autotune_contraction, pin_contraction
    from torch.profiler import ProfilerActivity, profile
    g2.set_logger(lambda msg: None)
    m, sig, e_y, e_x = build_problem()
    op = g2.IEOperator.from_model(m)
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    op.calc_fft_of_ie_kernel()
    op.set_anomaly_sigma(sig, m.freq)
    tuned = pin_contraction(op, args.variants) if args.variants else autotune_contraction(op)
    dev = torch.device("cuda")
    d_in = [torch.from_numpy(np.ascontiguousarray(e).ravel()).to(dev) for e in (e_y, e_x)]
    d_out = [torch.empty_like(x) for x in d_in]
    batch = g2.Batch([op, op], outer_buf=OUTER, inner_buf=INNER, precision=1, max_restart=MAXRESTART)

    def step():
        return batch.solve_device([x.data_ptr() for x in d_in], [y.data_ptr() for y in d_out], tol=TOL)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(op.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step()
    e1.record(stream)
    torch.cuda.synchronize()
    step_ms = e0.elapsed_time(e1)
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step()
        torch.cuda.synchronize()
    tot, cnt, iv = collections.Counter(), collections.Counter(), []
    for e in prof.events():
        if e.device_type != torch.autograd.DeviceType.CUDA:
            continue
        name = e.name.replace("void ", "").replace("(anonymous namespace)::", "").replace("<unnamed>::", "")
        name = name.split("<")[0].split("(")[0].strip()
        tot[name] += e.device_time_total
        cnt[name] += 1
        iv.append((e.time_range.start, e.time_range.end))
    iv.sort()
    gaps = [b[0] - a[1] for a, b in zip(iv, iv[1:]) if b[0] > a[1]]
    print(json.dumps({"mode": "step-breakdown", "step_ms": step_ms, "kernels": sum(cnt.values()),
                      "busy_ms": sum(tot.values()) / 1e3, "idle_gap_ms": sum(gaps) / 1e3,
                      "per_kernel_ms": {k: [round(v / 1e3, 4), cnt[k]] for k, v in tot.most_common()},
                      "contract_variants": {k: v.get("variant", v.get("lines")) for k, v in tuned.items()}}))
    batch.delete()
    op.delete()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the 16-instance multi-frequency sweep")
    ap.add_argument("--variants", default=None,
                    help="pin the tile shapes instead of autotuning: v64,v32,vpair[,fft_lines[,fft_lines64]] "
                         "(for profilers)")
    prof = ap.add_argument_group("profiler workloads (--apply-only, --receivers-only, --learned-only)")
    prof.add_argument("--apply-only", action="store_true", help="a few IE applies at one grid")
    prof.add_argument("--receivers-only", action="store_true", help="receiver tensor and recalculations")
    prof.add_argument("--learned-only", action="store_true", help="inferences of the learned preconditioner's net")
    prof.add_argument("--nx", type=int, default=128)
    prof.add_argument("--ny", type=int, default=None)
    prof.add_argument("--nz", type=int, default=32)
    prof.add_argument("--prec", type=int, default=0, choices=[0, 1])
    prof.add_argument("--reps", type=int, default=3)
    prof.add_argument("--variant", type=int, default=None)
    prof.add_argument("--nv", type=int, default=1, choices=[1, 2], help="vectors per apply (2: paired complex64)")
    prof.add_argument("--fft-lines", type=int, default=None, choices=[4, 8, 16, 32])
    prof.add_argument("--nr", type=int, default=1, help="receiver depths")
    prof.add_argument("--step-breakdown", action="store_true",
                      help="warm per-kernel device times of one batched step (CUPTI trace)")
    args = ap.parse_args()
    if args.apply_only:
        return run_apply_only(args)
    if args.step_breakdown:
        return run_step_breakdown(args)
    if args.receivers_only:
        if args.warmup == ap.get_default("warmup"):
            args.warmup = 1
        return run_receivers_only(args)
    if args.learned_only:
        return run_learned_only(args)
    rank, world, local = _env_int("RANK", 0), _env_int("WORLD_SIZE", 1), _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_b200(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
