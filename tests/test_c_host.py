"""A plain C host (tests/c_host/host_solve.c) against the library: the header is valid C and the program
links against the .so on any machine; on a B200 it runs the reference's call sequence and a solve, and
its own FP64 residual check must pass."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    from giem2g_b200 import build as b
    lib = b.build()
    exe = str(tmp_path / "host_solve")
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Werror", os.path.join(ROOT, "tests", "c_host", "host_solve.c"),
           "-I", os.path.join(ROOT, "include"), "-L", os.path.dirname(lib), "-lgiem2g_b200",
           "-Wl,-rpath," + os.path.dirname(lib), "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_c_host_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_c_host_solves(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    it, stat, be, rres, rmax = r.stdout.split()[-5:]
    assert int(stat) == 1 and float(be) < 1e-8 and float(rres) < 1.5e-8 and float(rmax) > 0
