"""Driver for the IE solve path with the reference's input and output files.

    python -m giem2g_b200.driver input.json [--precision 0|1] [--outdir DIR]

Restates the solve part of the reference's main program (giem2g.F90:336-373, 430-470): read the JSON
input (background, anomaly grid and conductivity file, frequencies, FGMRES settings), then for every
frequency in order build the Green's tensor on the GPU, transform it, set the anomaly conductivity and
solve the plane-wave problem for EY and EX (as one lockstep batch of the two polarisations by default, or
one after the other with --sequential, as the reference does).  The initial guess of each solve follows the reference:
a solution file of the same frequency and polarisation if one exists in the output directory, else
nothing for the first frequency, else the previous frequency's solution of that polarisation.  With
"Save Solution" true every solution is written as SOL_P{Y,X}_F<freq>.bin.  With "Recalculate Fields"
true (giem2g.F90:276-310, 338-343, 380-430) the receiver tensor is built and transformed on the GPU per
frequency, the anomalous E and H at the receivers ("Recievers") come from each solution, the normal
field of the background is added, and both are written as P{Y,X}_F<freq>.dat.  With "Solve Equation"
false the solutions are read from the SOL files; a frequency whose file is missing is skipped, as in
the reference.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from .solution_io import (EX, EY, load_input, load_solution, read_sigma_text, receiver_output_name,
                          receivers_from_input, save_receiver_fields, save_solution, solution_name)


def model_from_input(inp: dict, base_dir: str):
    """(IEModel at the first frequency, conductivity [Ny, Nx, Nz], frequencies, FGMRES settings)."""
    from .synthetic import IEModel
    bkg, an = inp["Background"], inp["Anomaly"]
    sigma = np.asarray(bkg["Conductivity"], dtype=np.float64)
    thick = np.asarray(bkg.get("Thickness", []), dtype=np.float64)[: len(sigma) - 1]
    Nx, Ny, Nz = int(an["Nx"]), int(an["Ny"]), int(an["Nz"])
    z = np.asarray(an["zborders"], dtype=np.float64)[: Nz + 1]
    freqs = [float(f) for f in inp["Frequencies"]]
    m = IEModel(Nx, Ny, Nz, float(an["dx"]), float(an["dy"]), z, sigma, thick, freqs[0])
    cpath = an["Conductivity"]
    if not os.path.isabs(cpath) and not os.path.exists(cpath):
        cpath = os.path.join(base_dir, cpath)
    sig = read_sigma_text(cpath, Nx, Ny, Nz)
    fg = inp.get("FGMRES", {})
    ctl = {"outer_buf": int(fg.get("OuterBufferSize", 30)), "inner_buf": int(fg.get("InnerBufferSize", 10)),
           "max_restart": int(fg.get("MaxRestart", 100)), "tol": float(fg.get("Tolerance", 1e-8))}
    return m, sig, freqs, ctl


def run(input_path: str, precision: int = 0, outdir: str | None = None, log=print, warm_start: bool = True,
        batched: bool = True) -> dict:
    """batched: solve the two polarisations of each frequency as one lockstep batch (the same iterates as
    two single solves; in mixed precision their complex64 applies share every tensor read)."""
    from . import Batch, IEOperator, RCOperator
    from .sources import plane_wave_integral, plane_wave_points
    inp = load_input(input_path)
    base = os.path.dirname(os.path.abspath(input_path))
    outdir = outdir or os.getcwd()
    m0, sig, freqs, ctl = model_from_input(inp, base)
    solve = bool(inp.get("Solve Equation", True))
    save = bool(inp.get("Save Solution", False))
    recalc = bool(inp.get("Recalculate Fields", False))
    out = {"grid": [m0.Nx, m0.Ny, m0.Nz], "frequencies": freqs, "precision": precision, "solves": []}
    if not solve and not recalc:
        return out
    rc = None
    if recalc:
        zr, xs, ys = receivers_from_input(inp)
        if not zr:
            raise ValueError("Recalculate Fields needs a non-empty Recievers list")
        rc = RCOperator.from_model(m0, zr, xs, ys)
        zr_used, _, _ = rc.receivers()
        out["receivers"] = {"depth": zr_used.tolist(), "xshift": xs, "yshift": ys}
    op = IEOperator.from_model(m0) if solve else None
    prev = {EY: None, EX: None}
    pols = (EY, EX)
    try:
        for i, f in enumerate(freqs):
            m = m0.with_freq(f)
            t0 = time.perf_counter()
            if solve:
                op.calc_ie_kernel(m.csigma, m.thick, m.omega)
                op.calc_fft_of_ie_kernel()
                op.set_anomaly_sigma(sig, f)
            if rc is not None:
                rc.calc_rc_kernel(m.csigma, m.thick, m.omega)
                rc.calc_fft_of_rc_kernel()
                rc.set_anomaly_sigma(sig, f)
            t_setup = time.perf_counter() - t0
            names = {pol: os.path.join(outdir, solution_name(pol, f)) for pol in pols}
            rows = {pol: {"freq": f, "pol": "EY" if pol == EY else "EX", "setup_s": t_setup} for pol in pols}
            fields = {}
            if solve:
                # initial guesses (giem2g.F90:356-373): the file of this frequency, else the previous frequency
                guesses, sources = {}, {}
                for pol in pols:
                    g = load_solution(names[pol], m.Nx, m.Ny, m.Nz)
                    src = "file" if g is not None else ("previous frequency" if i > 0 and warm_start else "none")
                    if g is None and i > 0 and warm_start:
                        g = prev[pol]
                    guesses[pol], sources[pol] = g, src
                E_bkg = {pol: plane_wave_integral(m, pol) for pol in pols}
                if batched:
                    b = Batch([op, op], outer_buf=ctl["outer_buf"], inner_buf=ctl["inner_buf"], precision=precision,
                              max_restart=ctl["max_restart"])
                    try:
                        sols, infos = b.solve([E_bkg[p] for p in pols], E0=[guesses[p] for p in pols], tol=ctl["tol"])
                    finally:
                        b.delete()
                    results = dict(zip(pols, zip(sols, infos)))
                else:
                    results = {pol: op.solve_equation(E_bkg[pol], E0=guesses[pol], tol=ctl["tol"],
                                                      max_restart=ctl["max_restart"], outer_buf=ctl["outer_buf"],
                                                      inner_buf=ctl["inner_buf"], precision=precision)
                               for pol in pols}
                for pol in pols:
                    E, info = results[pol]
                    prev[pol] = fields[pol] = E
                    if save:
                        save_solution(names[pol], E)
                    rows[pol].update({"guess": sources[pol], "iterations": info.iterations, "stat": info.stat,
                                      "true_rel_residual": info.be, "device_ms": info.device_ms,
                                      "batched": bool(batched)})
            else:
                for pol in pols:
                    g = load_solution(names[pol], m.Nx, m.Ny, m.Nz)
                    if g is None:  # giem2g.F90:398-412: "Solution not found", next frequency
                        rows[pol]["solution"] = "not found"
                        break
                    fields[pol] = g
                    rows[pol]["solution"] = "file"
            for pol in pols:
                if pol not in fields:
                    if "solution" in rows[pol]:
                        out["solves"].append(rows[pol])
                        if log:
                            log(json.dumps(rows[pol]))
                    break
                if rc is not None:
                    t1 = time.perf_counter()
                    Ea, Ha = rc.recalculate(fields[pol])
                    F = plane_wave_points(m, pol, zr_used)  # [Nr, 6]: Ex Ey Ez Hx Hy Hz
                    Et = Ea + F[:, :3].T[None, None]
                    Ht = Ha + F[:, 3:].T[None, None]
                    save_receiver_fields(os.path.join(outdir, receiver_output_name(pol, f)), m.dx, m.dy, zr_used, xs,
                                         ys, f, Ea, Ha, Et, Ht)
                    rows[pol]["recalc_s"] = time.perf_counter() - t1
                out["solves"].append(rows[pol])
                if log:
                    log(json.dumps(rows[pol]))
    finally:
        if op is not None:
            op.delete()
        if rc is not None:
            rc.delete()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="IE solves of a GIEM2G input file on one GPU")
    ap.add_argument("input")
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1], help="0: FP64, 1: mixed")
    ap.add_argument("--outdir", default=None, help="directory of the SOL_*.bin files (default: cwd)")
    ap.add_argument("--cold", action="store_true", help="no previous-frequency guess (for comparison)")
    ap.add_argument("--sequential", action="store_true", help="solve EY then EX one at a time, as the reference does")
    args = ap.parse_args(argv)
    res = run(args.input, args.precision, args.outdir, warm_start=not args.cold, batched=not args.sequential)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
