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
    # the reference's order (EY, then EX, one at a time) gives the same solutions as the batched default
    seq_dir = tmp_path / "sequential"
    seq_dir.mkdir()
    seq = run(path, precision=0, outdir=str(seq_dir), log=None, batched=False)
    assert [r["iterations"] for r in seq["solves"]] == [r["iterations"] for r in rows]
    for f in freqs:
        for pol in (EY, EX):
            a = load_solution(str(seq_dir / solution_name(pol, f)), 16, 16, 8)
            b = load_solution(str(tmp_path / solution_name(pol, f)), 16, 16, 8)
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-10
    # a second run starts every solve from its own solution file: nothing left to iterate
    again = run(path, precision=0, outdir=str(tmp_path), log=None)
    assert all(r["guess"] == "file" and r["stat"] == 1 and r["iterations"] <= 1 for r in again["solves"])


def test_driver_receiver_fields(g2lib, orc, tmp_path):
    """"Recalculate Fields": the P{Y,X}_F files hold the anomalous fields of each solution at the
    receivers (checked against the oracle's ReCalculation of the same solution with the oracle's own
    receiver tensor) plus the background's PlaneWave; with "Solve Equation" false the same files come
    from the saved solutions."""
    from giem2g_b200.driver import run
    from giem2g_b200.solution_io import load_receiver_fields, receiver_output_name
    from giem2g_b200.synthetic import IEModel, csiga_from_sigma
    path, sig = _write_case(tmp_path, [2.0])
    inp = json.loads(open(path).read())
    inp["Recalculate Fields"] = True
    inp["Recievers"] = [{"depth": 0.0, "xshift": 0.0, "yshift": 0.0},
                        {"depth": 175.0, "xshift": 10.0, "yshift": -20.0}]   # inside a cell: moved to 150
    open(path, "w").write(json.dumps(inp))
    out = run(path, precision=0, outdir=str(tmp_path), log=None)
    assert out["receivers"]["depth"] == [0.0, 150.0]
    assert all("recalc_s" in r for r in out["solves"])
    m = IEModel(16, 16, 8, 100.0, 100.0, np.arange(9) * 50.0, np.array([0.01, 0.001, 0.1]),
                np.array([500.0, 1500.0]), 2.0)
    rv = orc.prepare_receivers(m, [0.0, 175.0], [0.0, 10.0], [0.0, -20.0])
    G = orc.rc_tensor(m, rv)
    csigb, _ = orc.background_cells(m)
    csiga = csiga_from_sigma(sig, m.freq)
    for pol in (EY, EX):
        E = load_solution(str(tmp_path / solution_name(pol, 2.0)), 16, 16, 8)
        Ea, Ha = orc.rc_apply(16, 16, 8, G, csiga, csigb, E)
        F = orc.plane_wave_points(m, pol, rv.zrecv)
        T = load_receiver_fields(str(tmp_path / receiver_output_name(pol, 2.0)))
        assert T.shape == (2 * 16 * 16, 28)
        vals = T[:, 4:].reshape(2, 16, 16, 4, 3, 2)             # [r][y][x][Ea Ha Et Ht][c][re im]
        got = vals[..., 0] + 1j * vals[..., 1]
        ref_a = np.stack([np.transpose(Ea, (3, 0, 1, 2)), np.transpose(Ha, (3, 0, 1, 2))], axis=3)
        ref_t = ref_a + np.stack([F[:, :3], F[:, 3:]], axis=1)[:, None, None]
        assert np.abs(got[:, :, :, :2] - ref_a).max() < 1e-9 * np.abs(ref_a).max()   # 10 significant digits
        assert np.abs(got[:, :, :, 2:] - ref_t).max() < 1e-9 * np.abs(ref_t).max()
    # recalculation only, from the saved solutions
    first = {pol: (tmp_path / receiver_output_name(pol, 2.0)).read_text() for pol in (EY, EX)}
    inp["Solve Equation"] = False
    open(path, "w").write(json.dumps(inp))
    out2 = run(path, precision=0, outdir=str(tmp_path), log=None)
    assert [r["solution"] for r in out2["solves"]] == ["file", "file"]
    for pol in (EY, EX):
        assert (tmp_path / receiver_output_name(pol, 2.0)).read_text() == first[pol]
