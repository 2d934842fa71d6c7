"""File formats of the reference's driver for the IE solve path.

* Solution files (mpi_saveload_module.F90:568-653): ``SOL_PY_F<freq>.bin`` / ``SOL_PX_F<freq>.bin`` hold
  the anomalous-domain field of one polarisation as raw little-endian complex(8) in the reference's
  internal order E(z, c, x, y) (z fastest; ConvertNaIn, :655-676).  The frequency string is Fortran
  F22.10 with the leading blanks of its first 11 characters turned into zeros (giem2g.F90:324-328), so
  0.1 Hz gives ``00000000000.1000000000``.  Fields here are complex [3, Nz, Ny, Nx] arrays, the memory
  order of the reference's "naive" E(x, y, z, c).
* Conductivity text file (mpi_saveload_module.F90:113-146): a Fortran list-directed READ of
  siga(Nz, Nx, Ny), z fastest; numbers separated by blanks, commas or new lines, with optional
  ``r*value`` repeat counts and D exponents.  Returned as numpy [Ny, Nx, Nz].
* Input JSON (mpi_saveload_module.F90:30-239): the reference's keys, read leniently (trailing commas,
  which the reference's own parser accepts, are allowed).  Receivers come from "Recievers" (the
  reference's spelling): a list of {"depth", "xshift", "yshift"} (LoadRecievers, :174-213).
* Receiver output (SaveOutputOneFile, mpi_saveload_module.F90:391-483): ``P{Y,X}_F<freq>.dat``, a title
  line "%" + 28 A20 titles, then one line per receiver and cell (receiver outer, then y, then x) of
  " " + 28 ES20.10E3 numbers: x, y, z of the receiver, frequency, then Re/Im of Ea (Ex Ey Ez),
  Ha (Hx Hy Hz), Et, Ht.  The receiver at cell (ix, iy) (0-based) is at x = (ix + 1/2) dx + xshift,
  y = (iy + 1/2) dy + yshift.
"""
from __future__ import annotations

import json
import os
import re

import numpy as np

EX, EY = 0, 1


def freq_string(freq: float) -> str:
    """The reference's frequency tag: F22.10 with blanks in the first 11 characters set to '0'."""
    s = f"{freq:22.10f}"
    return "".join("0" if (i < 11 and ch == " ") else ch for i, ch in enumerate(s)).rstrip()


def solution_name(pol: int, freq: float) -> str:
    """SOL_PY_F<freq>.bin for pol EY, SOL_PX_F<freq>.bin for pol EX (giem2g.F90:356, :379, :439)."""
    return ("SOL_PY_F" if pol == EY else "SOL_PX_F") + freq_string(freq) + ".bin"


def save_solution(path: str, E: np.ndarray) -> None:
    """E: complex [3, Nz, Ny, Nx] -> file in the order E(z, c, x, y), z fastest."""
    E = np.asarray(E, dtype=np.complex128)
    if E.ndim != 4 or E.shape[0] != 3:
        raise ValueError(f"field must be [3, Nz, Ny, Nx], got {E.shape}")
    np.ascontiguousarray(np.transpose(E, (2, 3, 0, 1))).astype("<c16").tofile(path)  # [y][x][c][z]


def load_solution(path: str, Nx: int, Ny: int, Nz: int) -> np.ndarray | None:
    """The field stored by save_solution (or by the reference), or None if the file does not exist."""
    if not os.path.exists(path):
        return None
    a = np.fromfile(path, dtype="<c16")
    if a.size != 3 * Nx * Ny * Nz:
        raise ValueError(f"{path}: {a.size} values, expected {3 * Nx * Ny * Nz}")
    return np.ascontiguousarray(np.transpose(a.reshape(Ny, Nx, 3, Nz), (2, 3, 0, 1)))


_REPEAT = re.compile(r"^(\d+)\*(.*)$")


def read_sigma_text(path: str, Nx: int, Ny: int, Nz: int) -> np.ndarray:
    """List-directed read of siga(Nz, Nx, Ny) -> numpy [Ny, Nx, Nz] (file order, z fastest)."""
    vals: list[float] = []
    need = Nx * Ny * Nz
    with open(path) as f:
        for line in f:
            for tok in re.split(r"[\s,]+", line.strip()):
                if not tok:
                    continue
                m = _REPEAT.match(tok)
                count, tok = (int(m.group(1)), m.group(2)) if m else (1, tok)
                v = float(tok.replace("D", "E").replace("d", "e"))
                vals.extend([v] * count)
            if len(vals) >= need:
                break
    if len(vals) < need:
        raise ValueError(f"{path}: {len(vals)} conductivities, expected {need}")
    return np.asarray(vals[:need], dtype=np.float64).reshape(Ny, Nx, Nz)


def load_input(path: str) -> dict:
    """The driver's JSON input, with trailing commas before ] or } tolerated."""
    text = open(path).read()
    text = re.sub(r",(\s*[\]}])", r"\1", text)
    return json.loads(text)


def receiver_output_name(pol: int, freq: float) -> str:
    """PY_F<freq>.dat for pol EY, PX_F<freq>.dat for pol EX (giem2g.F90:427-428, :501-502)."""
    return ("PY_F" if pol == EY else "PX_F") + freq_string(freq) + ".dat"


_TITLES = ["x_recv", "y_recv", "z_recv", "frequency",
           "Re Ex^a", "Im Ex^a", "Re Ey^a", "Im Ey^a", "Re Ez^a", "Im Ez^a",
           "Re Hx^a", "Im Hx^a", "Re Hy^a", "Im Hy^a", "Re Hz^a", "Im Hz^a",
           "Re Ex^t", "Im Ex^t", "Re Ey^t", "Im Ey^t", "Re Ez^t", "Im Ez^t",
           "Re Hx^t", "Im Hx^t", "Re Hy^t", "Im Hy^t", "Re Hz^t", "Im Hz^t"]


def _es20_10e3(v: float) -> str:
    """Fortran ES20.10E3: one digit before the point, ten after, a three-digit exponent."""
    mant, exp = f"{float(v):.10E}".split("E")
    return f"{mant}E{int(exp):+04d}".rjust(20)


def save_receiver_fields(path: str, dx: float, dy: float, zrecv, x_shift, y_shift, freq: float,
                         Ea: np.ndarray, Ha: np.ndarray, Et: np.ndarray, Ht: np.ndarray) -> None:
    """Fields [Ny, Nx, 3, Nr] (the reference's (Nr,3,Nx,Ny)) -> the reference's text table."""
    Ny, Nx, _, Nr = Ea.shape
    lines = ["%" + "".join(t.rjust(20) for t in _TITLES)]
    for r in range(Nr):
        for iy in range(Ny):
            y = (iy + 1) * dy - dy / 2.0 + y_shift[r]
            for ix in range(Nx):
                x = (ix + 1) * dx - dx / 2.0 + x_shift[r]
                vals = [x, y, zrecv[r], freq]
                for F in (Ea, Ha, Et, Ht):
                    for c in range(3):
                        v = F[iy, ix, c, r]
                        vals += [v.real, v.imag]
                lines.append(" " + "".join(_es20_10e3(v) for v in vals))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def load_receiver_fields(path: str) -> np.ndarray:
    """The numeric table of a receiver output file: [rows, 28] (x, y, z, f, then 24 Re/Im values)."""
    return np.loadtxt(path, comments="%", ndmin=2)


def receivers_from_input(inp: dict):
    """(depths, xshifts, yshifts) from the "Recievers" list of the input JSON."""
    rs = inp.get("Recievers", [])
    return ([float(r["depth"]) for r in rs], [float(r.get("xshift", 0.0)) for r in rs],
            [float(r.get("yshift", 0.0)) for r in rs])
