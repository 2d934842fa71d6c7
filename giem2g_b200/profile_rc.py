"""Receiver-field workload for profilers: build the receiver tensor and run recalculations.

    python -m giem2g_b200.profile_rc --nx 128 --nz 32 --nr 1 --reps 3

Builds the receiver tensor for Nr surface-and-below receivers on a seeded random-field model, transforms
it, and runs `reps` recalculations on device buffers; prints one JSON line with CUDA-event timings.
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
    ap.add_argument("--nr", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    args = ap.parse_args(argv)
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
    n = 3 * m.Nx * m.Ny * m.Nz
    E = torch.randn(n, dtype=torch.complex128, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
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
    print(json.dumps({"grid": [m.Nx, m.Ny, m.Nz], "receivers": args.nr, "tensor_build_s": t1 - t0,
                      "tensor_fft_s": t2 - t1, "recalculate_ms": e0.elapsed_time(e1) / max(1, args.reps)}))
    rc.delete()


if __name__ == "__main__":
    main()
