"""File formats of the reference's driver (solution files, conductivity text, input JSON) on the CPU."""
import json
import os

import numpy as np

from giem2g_b200.solution_io import (EX, EY, freq_string, load_input, load_solution, read_sigma_text,
                                     save_solution, solution_name)


def test_frequency_tag_matches_f22_10_with_leading_zeros():
    assert freq_string(0.1) == "00000000000.1000000000"
    assert freq_string(100.0) == "00000000100.0000000000"
    assert freq_string(0.001) == "00000000000.0010000000"
    assert len(freq_string(3.7275937203149416)) == 22
    assert solution_name(EY, 1.0) == "SOL_PY_F00000000001.0000000000.bin"
    assert solution_name(EX, 1.0) == "SOL_PX_F00000000001.0000000000.bin"


def test_solution_file_order_is_z_c_x_y(tmp_path):
    Nx, Ny, Nz = 4, 3, 2
    rng = np.random.default_rng(1)
    E = rng.standard_normal((3, Nz, Ny, Nx)) + 1j * rng.standard_normal((3, Nz, Ny, Nx))
    p = tmp_path / "s.bin"
    save_solution(str(p), E)
    raw = np.fromfile(p, dtype="<c16")
    assert raw.size == E.size
    # element (z, c, x, y) of the file sits at z + Nz*(c + 3*(x + Nx*y))
    for (z, c, x, y) in [(0, 0, 0, 0), (1, 2, 3, 2), (0, 1, 2, 1), (1, 0, 1, 0)]:
        assert raw[z + Nz * (c + 3 * (x + Nx * y))] == E[c, z, y, x]
    back = load_solution(str(p), Nx, Ny, Nz)
    assert np.array_equal(back, E)
    assert load_solution(str(tmp_path / "missing.bin"), Nx, Ny, Nz) is None


def test_sigma_text_list_directed(tmp_path):
    Nx, Ny, Nz = 3, 2, 2
    vals = np.arange(1, Nx * Ny * Nz + 1, dtype=float) * 1e-3
    p = tmp_path / "sig.dat"
    # blanks, commas, new lines, a repeat count and D exponents, as a list-directed READ accepts
    toks = [f"{v:.3E}".replace("E", "D") for v in vals[:6]] + ["2*7.000E-03"]
    body = " ".join(toks[:3]) + ",\n" + ", ".join(toks[3:]) + "\n" + "\n".join(f"{v}" for v in vals[8:])
    p.write_text(body)
    vals2 = vals.copy()
    vals2[6:8] = 7e-3
    s = read_sigma_text(str(p), Nx, Ny, Nz)
    assert s.shape == (Ny, Nx, Nz)
    assert np.allclose(s.ravel(), vals2)
    assert s[1, 2, 0] == vals2[0 + Nz * (2 + Nx * 1)]  # siga(z, x, y) with z fastest


def test_input_json_with_trailing_commas(tmp_path):
    p = tmp_path / "in.json"
    p.write_text('{"Frequencies": [0.1, 1.0,], "FGMRES": {"Tolerance": 1e-8,}, "Recievers": [{"depth": 0},],}')
    d = load_input(str(p))
    assert d["Frequencies"] == [0.1, 1.0] and d["FGMRES"]["Tolerance"] == 1e-8


def test_receiver_output_table_layout(tmp_path):
    from giem2g_b200.solution_io import load_receiver_fields, receiver_output_name, save_receiver_fields
    assert receiver_output_name(EY, 0.1) == "PY_F00000000000.1000000000.dat"
    assert receiver_output_name(EX, 10.0) == "PX_F00000000010.0000000000.dat"
    Ny, Nx, Nr = 2, 3, 2
    rng = np.random.default_rng(4)
    F = [rng.standard_normal((Ny, Nx, 3, Nr)) + 1j * rng.standard_normal((Ny, Nx, 3, Nr)) for _ in range(4)]
    p = tmp_path / "PY.dat"
    save_receiver_fields(str(p), 50.0, 40.0, [0.0, 120.0], [0.0, 5.0], [0.0, -5.0], 0.1, *F)
    lines = p.read_text().splitlines()
    assert lines[0].startswith("%") and len(lines[0]) == 1 + 28 * 20 and lines[0][1:21].strip() == "x_recv"
    assert all(len(l) == 1 + 28 * 20 and l[0] == " " for l in lines[1:])
    assert "E+000" in lines[1] or "E-0" in lines[1]
    T = load_receiver_fields(str(p))
    assert T.shape == (Nr * Ny * Nx, 28)
    # receiver outer, then y, then x; x = (ix + 1/2) dx + xshift
    k = 1 * Ny * Nx + 1 * Nx + 2   # r = 1, iy = 1, ix = 2
    assert np.allclose(T[k, :4], [2.5 * 50.0 + 5.0, 1.5 * 40.0 - 5.0, 120.0, 0.1])
    for j, Fa in enumerate(F):
        got = T[k, 4 + 6 * j: 10 + 6 * j].reshape(3, 2)
        assert np.allclose(got[:, 0] + 1j * got[:, 1], Fa[1, 2, :, 1], rtol=1e-10)


def test_receivers_from_input():
    from giem2g_b200.solution_io import receivers_from_input
    z, xs, ys = receivers_from_input({"Recievers": [{"depth": 0, "xshift": 1.5, "yshift": 0}, {"depth": 200.0}]})
    assert z == [0.0, 200.0] and xs == [1.5, 0.0] and ys == [0.0, 0.0]


def test_model_from_input(tmp_path):
    """The driver's model: grid, borders, background truncated to the layer count, frequencies, FGMRES
    defaults, and a conductivity file named relative to the input's directory."""
    from giem2g_b200.driver import model_from_input
    Nx, Ny, Nz = 4, 2, 3
    (tmp_path / "sig.txt").write_text(" ".join(["1.0D-2"] * (Nx * Ny * Nz)))
    inp = {
        "Background": {"Conductivity": [0.0, 0.01, 0.001, 0.1], "Thickness": [500.0, 1500.0, 99.0]},
        "Anomaly": {"Nx": Nx, "Ny": Ny, "Nz": Nz, "dx": 50.0, "dy": 60.0,
                    "zborders": [0.0, 25.0, 50.0, 100.0, 999.0], "Conductivity": "sig.txt"},
        "Frequencies": [0.1, 1, "10"],
        "FGMRES": {"Tolerance": 1e-6, "OuterBufferSize": 20},
    }
    m, sig, freqs, ctl = model_from_input(inp, str(tmp_path))
    assert (m.Nx, m.Ny, m.Nz) == (Nx, Ny, Nz) and (m.dx, m.dy) == (50.0, 60.0)
    assert list(m.z) == [0.0, 25.0, 50.0, 100.0]  # Nz + 1 borders
    assert list(m.thick) == [500.0, 1500.0, 99.0][: len(inp["Background"]["Conductivity"]) - 1]
    assert freqs == [0.1, 1.0, 10.0] and m.freq == 0.1
    assert sig.shape == (Ny, Nx, Nz) and np.all(sig == 1e-2)
    assert ctl == {"outer_buf": 20, "inner_buf": 10, "max_restart": 100, "tol": 1e-6}
