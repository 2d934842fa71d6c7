"""The Fortran ISO_C_BINDING module (include/giem2g_cuda_bind.F90) against the C header.

No Fortran compiler exists in this image, so the module is checked as text: every BIND(C) derived type
lists the same fields, in the same order and with the same C kinds, as the struct of the same name in
include/giem2g.h, and every bound procedure names a function the header declares.  Where gfortran is on
PATH the module is also compiled (syntax and semantics only)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "giem2g_cuda_bind.F90")
HDR = os.path.join(ROOT, "include", "giem2g.h")

C_OF_F = {"INTEGER(C_INT)": "int", "INTEGER(C_LONG_LONG)": "long long", "REAL(C_DOUBLE)": "double",
          "TYPE(C_PTR)": "void *"}


def _fortran_types():
    src = open(F90).read()
    out = {}
    for name, body in re.findall(r"TYPE, BIND\(C\) :: (\w+)\n(.*?)END TYPE", src, re.S):
        fields = []
        for line in body.splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            kind, names = [x.strip() for x in line.split("::")]
            fields += [(C_OF_F[kind], n.strip()) for n in names.split(",")]
        out[name] = fields
    return out


def _c_structs():
    src = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    out = {}
    for body, name in re.findall(r"typedef struct \{(.*?)\} (\w+);", src, re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            m = re.match(r"(long long|int|double|void)\s*(\*?)\s*(.*)", decl)
            ctype = m.group(1) + (" *" if m.group(2) else "")
            for n in m.group(3).split(","):
                n = n.strip()
                if n.startswith("*"):
                    ctype, n = m.group(1) + " *", n[1:].strip()
                fields.append((ctype, n))
        out[name] = fields
    return out


def test_derived_types_match_the_c_structs():
    ft, cs = _fortran_types(), _c_structs()
    assert set(ft) == {"GIEM2G_BACKGROUND_TYPE", "GIEM2G_ANOMALY_TYPE", "GIEM2G_DATA_TYPE", "GIEM2G_FGMRES_CTL",
                       "GIEM2G_RESULT"}
    for name, fields in ft.items():
        want = [(t, n.lower()) for t, n in cs[name]]
        got = [(t, n.lower()) for t, n in fields]
        assert got == want, name


def test_bound_procedures_are_declared_in_the_header():
    src = open(F90).read()
    hdr = open(HDR).read()
    names = re.findall(r"BIND\(C, NAME='(\w+)'\)", src)
    assert "giem2g_apply_ie_operator" in names and "giem2g_solve" in names
    for n in names:
        if n == "strlen":
            continue
        assert re.search(r"\b%s\s*\(" % n, hdr), n


@pytest.mark.skipif(shutil.which("gfortran") is None, reason="no Fortran compiler in this image")
def test_module_compiles(tmp_path):
    r = subprocess.run(["gfortran", "-std=f2008", "-fsyntax-only", "-J", str(tmp_path), F90], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
