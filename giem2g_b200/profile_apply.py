"""Run a few IE-operator applies at a given grid, for profilers.

    python -m giem2g_b200.profile_apply --nx 128 --nz 32 --prec 0 --reps 3

Builds the operator on the GPU (Green's tensor over the 3-layer background, spectral transform),
sets a seeded Gaussian-random-field anomaly and runs `--reps` applies in the requested precision
(0 = complex128, 1 = complex64) on the operator's stream, then prints the CUDA-event time per apply.
A profiler selects the apply kernels by name (k_fx, k_fy, k_contract_tma or k_contract_wl, k_by, k_bx).
"""
from __future__ import annotations

import argparse
import json
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=None)
    ap.add_argument("--nz", type=int, default=32)
    ap.add_argument("--prec", type=int, default=0, choices=[0, 1])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=0, help="untimed applies before the timed ones")
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--nv", type=int, default=1, choices=[1, 2], help="vectors per apply (2: paired complex64)")
    ap.add_argument("--fft-lines", type=int, default=None, choices=[4, 8, 16, 32], help="lines per CTA of the FFTs")
    args = ap.parse_args(argv)
    import torch
    import giem2g_b200 as g2
    from giem2g_b200.synthetic import config_grf

    m, sig = config_grf(args.nx, args.ny or args.nx, args.nz, seed=7)
    Nx, Ny, Nz = m.Nx, m.Ny, m.Nz
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
    stream = torch.cuda.ExternalStream(op.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x2, y2 = torch.randn_like(x), torch.empty_like(x)

    def one():
        if args.nv == 2:
            g2.apply_device_batch(op, [x.data_ptr(), x2.data_ptr()], [y.data_ptr(), y2.data_ptr()], args.prec)
        else:
            op.apply_device(x.data_ptr(), y.data_ptr(), args.prec)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.reps):
        one()
    e1.record(stream)
    torch.cuda.synchronize()
    op.check_device_error()
    print(json.dumps({"grid": [Nx, Ny, Nz], "precision": args.prec, "nv": args.nv, "reps": args.reps,
                      "ms_per_apply": e0.elapsed_time(e1) / args.reps, "tensor_build_s": t_build}))
    op.delete()


if __name__ == "__main__":
    main()
