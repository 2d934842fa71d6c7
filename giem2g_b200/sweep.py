"""Frequency x polarisation sweep of IE solves on one GPU.

This is the reference's main loop for the solve path (giem2g.F90:320-373: for every frequency build
the Green's tensor, transform it, set the anomaly, solve EY then EX), with the instances solved as one
batch (giem2g_batch_*): every (frequency, polarisation) instance runs its own nested FGMRES, in
lockstep with the others, and the two polarisations of one frequency share each complex64 tensor read.

    python -m giem2g_b200.sweep --config c1 --precision 0 --tol 1e-8   # 32x32x8 block model, FP64
    python -m giem2g_b200.sweep --config c3            # 128x128x32, 8 frequencies x 2 polarisations
    python -m giem2g_b200.sweep --config c5 --compare  # 256x256x48 + ellipsoids, 4 x 2, vs sequential

Prints one JSON object: set-up time per frequency, per-instance iterations, status and true residual,
the batched solve time (device), and with --compare the same instances solved one after the other in
mixed precision and in plain FP64, with the field error of the batched solution against FP64.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def sweep_config(name: str):
    from .synthetic import config_c2, config_c5, config_small_block
    if name == "c1":
        m, sig = config_small_block()
        return m, sig, [1.0]
    if name == "c3":
        m, sig = config_c2(seed=2024)
        return m, sig, list(np.logspace(-3, 2, 8))
    if name == "c5":
        m, sig = config_c5(seed=5)
        return m, sig, [0.01, 0.1, 1.0, 10.0]
    if name == "c2":
        m, sig = config_c2(seed=2024)
        return m, sig, [0.1]
    raise ValueError(f"unknown sweep config {name}")


def run_sweep(m, sig, freqs, pols=(1, 0), tol=1e-6, precision=1, outer=30, inner=10, max_restart=100,
              compare=False, fp64_tol=1e-8, tuned=None):
    """`tuned`: tile shapes to pin on every operator (an autotune_contraction result of the same grid);
    without it the shapes are timed on the first operator."""
    import torch
    import giem2g_b200 as g2
    from .sources import plane_wave_integral

    out = {"grid": [m.Nx, m.Ny, m.Nz], "freqs": [float(f) for f in freqs], "pols": list(pols), "tol": tol}
    ops, setup_s = [], []
    for f in freqs:
        mf = m.with_freq(float(f))
        t0 = time.perf_counter()
        op = g2.IEOperator.from_model(mf)
        op.calc_ie_kernel(mf.csigma, mf.thick, mf.omega)
        op.calc_fft_of_ie_kernel()
        op.set_anomaly_sigma(sig, mf.freq)
        torch.cuda.synchronize()
        setup_s.append(time.perf_counter() - t0)
        ops.append((mf, op))
    out["setup_s_per_frequency"] = setup_s
    # tile shapes: time the variants on the first operator; the others have the same grid
    from .autotune import autotune_contraction
    pinned = tuned is not None
    if not pinned:
        tuned = autotune_contraction(ops[0][1])
    for _, op in (ops if pinned else ops[1:]):
        for prec in (0, 1, 2):
            if str(prec) in tuned and op.contract_variants(prec) > 1:
                op.set_contract_variant(prec, tuned[str(prec)]["variant"])
        op.set_fft_lines(tuned["fft_lines"]["lines"], precision=1)
        op.set_fft_lines(tuned["fft_lines64"]["lines"], precision=0)
    out["tuned"] = tuned
    inst_ops, d_rhs = [], []
    for mf, op in ops:
        for p in pols:
            inst_ops.append(op)
            d_rhs.append(torch.from_numpy(np.ascontiguousarray(plane_wave_integral(mf, p)).ravel()).to("cuda"))
    d_sol = [torch.empty_like(x) for x in d_rhs]
    batch = g2.Batch(inst_ops, outer_buf=outer, inner_buf=inner, precision=precision, max_restart=max_restart)
    batch.solve_device([x.data_ptr() for x in d_rhs], [y.data_ptr() for y in d_sol], tol=tol)  # warm-up
    infos = batch.solve_device([x.data_ptr() for x in d_rhs], [y.data_ptr() for y in d_sol], tol=tol)
    out["batched"] = {"device_ms": infos[0].device_ms,
                      "iterations": [i.iterations for i in infos], "stat": [i.stat for i in infos],
                      "true_rel_residual": [i.be for i in infos],
                      "applies": [i.applies_fp64 + i.applies_fp32 for i in infos]}
    batch.delete()  # its work space goes before the sequential solves allocate theirs
    if compare:
        for label, prec, t in (("sequential_mixed", 1, tol), ("sequential_fp64", 0, tol)):
            ms, its = 0.0, []
            for op, x in zip(inst_ops, d_rhs):
                y = torch.empty_like(x)
                op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=t, max_restart=max_restart,
                                outer_buf=outer, inner_buf=inner, precision=prec)  # warm-up
                info = op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=t, max_restart=max_restart,
                                       outer_buf=outer, inner_buf=inner, precision=prec)
                ms += info.device_ms
                its.append(info.iterations)
            out[label] = {"device_ms": ms, "iterations": its}
        errs = []
        for op, x, ys in zip(inst_ops, d_rhs, d_sol):
            y = torch.empty_like(x)
            op.solve_device(x.data_ptr(), y.data_ptr(), None, tol=fp64_tol, max_restart=max_restart,
                            outer_buf=outer, inner_buf=inner, precision=0)
            errs.append((torch.linalg.vector_norm(ys - y) / torch.linalg.vector_norm(y)).item())
        out["field_error_vs_fp64"] = errs
        out["speedup_batched_vs_sequential_fp64"] = out["sequential_fp64"]["device_ms"] / out["batched"]["device_ms"]
        out["speedup_batched_vs_sequential_mixed"] = out["sequential_mixed"]["device_ms"] / out["batched"]["device_ms"]
    for _, op in ops:
        op.delete()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c5"])
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1])
    ap.add_argument("--compare", action="store_true")
    args = ap.parse_args(argv)
    import giem2g_b200 as g2
    import sys
    g2.set_logger(lambda msg: None)
    m, sig, freqs = sweep_config(args.config)
    res = run_sweep(m, sig, freqs, tol=args.tol, precision=args.precision, compare=args.compare)
    res["config"] = args.config
    print(json.dumps(res))
    sys.stdout.flush()


if __name__ == "__main__":
    main()
