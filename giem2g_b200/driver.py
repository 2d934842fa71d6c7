"""Driver for the IE solve path with the reference's input and output files.

    python -m giem2g_b200.driver input.json [--precision 0|1] [--outdir DIR]

Restates the solve part of the reference's main program (giem2g.F90:336-373, 430-470): read the JSON
input (background, anomaly grid and conductivity file, frequencies, FGMRES settings), then for every
frequency in order build the Green's tensor on the GPU, transform it, set the anomaly conductivity and
solve the plane-wave problem for EY, then EX.  The initial guess of each solve follows the reference:
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


def run(input_path: str, precision: int = 0, outdir: str | None = None, log=print, warm_start: bool = True) -> dict:
    from . import IEOperator, RCOperator
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
            for pol in (EY, EX):
                name = os.path.join(outdir, solution_name(pol, f))
                guess = load_solution(name, m.Nx, m.Ny, m.Nz)
                row = {"freq": f, "pol": "EY" if pol == EY else "EX", "setup_s": t_setup}
                if solve:
                    source = "file" if guess is not None else ("previous frequency" if i > 0 else "none")
                    if guess is None and i > 0 and warm_start:
                        guess = prev[pol]
                    elif guess is None:
                        source = "none"
                    E_bkg = plane_wave_integral(m, pol)
                    E, info = op.solve_equation(E_bkg, E0=guess, tol=ctl["tol"], max_restart=ctl["max_restart"],
                                                outer_buf=ctl["outer_buf"], inner_buf=ctl["inner_buf"],
                                                precision=precision)
                    prev[pol] = E
                    if save:
                        save_solution(name, E)
                    row.update({"guess": source, "iterations": info.iterations, "stat": info.stat,
                                "true_rel_residual": info.be, "device_ms": info.device_ms})
                else:
                    if guess is None:  # giem2g.F90:398-412: "Solution not found", next frequency
                        row["solution"] = "not found"
                        out["solves"].append(row)
                        if log:
                            log(json.dumps(row))
                        break
                    E = guess
                    row["solution"] = "file"
                if rc is not None:
                    t1 = time.perf_counter()
                    Ea, Ha = rc.recalculate(E)
                    F = plane_wave_points(m, pol, zr_used)  # [Nr, 6]: Ex Ey Ez Hx Hy Hz
                    Et = Ea + F[:, :3].T[None, None]
                    Ht = Ha + F[:, 3:].T[None, None]
                    save_receiver_fields(os.path.join(outdir, receiver_output_name(pol, f)), m.dx, m.dy, zr_used, xs,
                                         ys, f, Ea, Ha, Et, Ht)
                    row["recalc_s"] = time.perf_counter() - t1
                out["solves"].append(row)
                if log:
                    log(json.dumps(row))
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
    args = ap.parse_args(argv)
    res = run(args.input, args.precision, args.outdir, warm_start=not args.cold)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
