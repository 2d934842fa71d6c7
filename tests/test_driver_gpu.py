"""The input-file driver on a small model: the reference's frequency loop, solution files and warm starts."""
import json
import os

import numpy as np
import pytest

from giem2g_b200.solution_io import EX, EY, load_solution, solution_name

pytestmark = pytest.mark.gpu


def _write_case(tmp_path, freqs):
    Nx, Ny, Nz = 16, 16, 8
    sig = np.full((Ny, Nx, Nz), 0.01)
    sig[5:11, 4:12, 2:6] = 0.5
    with open(tmp_path / "sigma.dat", "w") as f:
        for v in sig.ravel():   # siga(Nz, Nx, Ny), z fastest
            f.write(f"{v:.6e}\n")
    inp = {"Save Solution": True, "Solve Equation": True, "Recalculate Fields": False,
           "Background": {"Conductivity": [0.01, 0.001, 0.1], "Permittivity": [], "Thickness": [500, 1500]},
           "Anomaly": {"Nx": Nx, "Ny": Ny, "Nz": Nz, "dx": 100.0, "dy": 100.0,
                       "zborders": [50.0 * k for k in range(Nz + 1)], "Conductivity": "sigma.dat"},
           "Frequencies": freqs,
           "FGMRES": {"OuterBufferSize": 30, "InnerBufferSize": 10, "MaxRestart": 100, "Tolerance": 1e-8}}
    p = tmp_path / "input.json"
    p.write_text(json.dumps(inp))
    return str(p), sig


def test_driver_frequency_loop_files_and_warm_start(g2lib, tmp_path):
    from giem2g_b200.driver import run
    from giem2g_b200.sources import plane_wave_integral
    from giem2g_b200.synthetic import IEModel
    freqs = [1.0, 3.0]
    path, sig = _write_case(tmp_path, freqs)
    out = run(path, precision=0, outdir=str(tmp_path), log=None)
    rows = out["solves"]
    assert [(r["freq"], r["pol"], r["guess"]) for r in rows] == [
        (1.0, "EY", "none"), (1.0, "EX", "none"), (3.0, "EY", "previous frequency"), (3.0, "EX", "previous frequency")]
    assert all(r["stat"] == 1 and r["true_rel_residual"] < 1e-8 for r in rows)
    for f in freqs:
        for pol in (EY, EX):
            assert os.path.exists(tmp_path / solution_name(pol, f))
    # the warm-started 3 Hz solution equals a cold solve of the same problem
    m = IEModel(16, 16, 8, 100.0, 100.0, np.arange(9) * 50.0, np.array([0.01, 0.001, 0.1]),
                np.array([500.0, 1500.0]), 3.0)
    op = g2lib.IEOperator.from_model(m)
    op.calc_ie_kernel(m.csigma, m.thick, m.omega)
    op.calc_fft_of_ie_kernel()
    op.set_anomaly_sigma(sig, m.freq)
    E_cold, _ = op.solve_equation(plane_wave_integral(m, EX), tol=1e-10, precision=0)
    op.delete()
    E_file = load_solution(str(tmp_path / solution_name(EX, 3.0)), 16, 16, 8)
    assert np.linalg.norm(E_file - E_cold) / np.linalg.norm(E_cold) < 1e-6
    # a second run starts every solve from its own solution file: nothing left to iterate
    again = run(path, precision=0, outdir=str(tmp_path), log=None)
    assert all(r["guess"] == "file" and r["stat"] == 1 and r["iterations"] <= 1 for r in again["solves"])
