"""CPU checks of the product library: it loads without a GPU, exports every
entry point declared in include/*.h, and its host set-up routines reproduce
the oracle's (RcutToAlpha, the pair table)."""
import ctypes as C
import os
import re

import numpy as np

import helpers as Hp
import pyoracle as O
from molsim_b200 import _lib, pot_tab, rcut_to_alpha
from molsim_b200 import systems as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(msg_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    L = C.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert names <= set(_lib.SIGNATURES)


def test_rcut_to_alpha_matches_oracle():
    for L_, rc, tol in ((100.0, 30.0, 1e-5), (250.0, 25.0, 1e-5), (1200.0, 30.0, 1e-5), (40.0, 18.0, 1e-4)):
        epsfp = S.EPSI0_FOUR_PI / 78.4
        a = rcut_to_alpha(tol, 1.0, epsfp, L_, rc)
        b = O.rcut_to_alpha(tol, 1.0, epsfp, L_, rc)
        assert a == b
        # the Kolafa-Perram estimate at that alpha gives back the tolerance
        est = O.lib().or_ewald_error_ureal(1.0, L_, a, rc, epsfp)
        assert abs(est / tol - 1) < 1e-4


def test_pot_tab_matches_oracle_bitwise():
    for s in (Hp.config0(), Hp.colloid_small(), Hp.electrolyte_small()):
        t = Hp.oracle_table(s)
        p = pot_tab(s, t["ualpha"])
        assert np.array_equal(p["iubuflow"], t["iubuflow"])
        assert np.array_equal(p["nugrid"], t["nugrid"])
        assert np.array_equal(p["ubuf"], t["ubuf"])
        assert np.array_equal(p["r2umin"], t["r2umin"])


def test_engine_fails_loudly_without_library(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    try:
        _lib.lib()
    except RuntimeError as e:
        assert "not built" in str(e)
    else:
        raise AssertionError("loading a missing library must fail")


def test_fortran_module_binds_every_entry_point():
    """The ISO_C_BINDING module declares every entry point of include/*.h under its C name."""
    f = open(os.path.join(ROOT, "molsim_b200", "fortran", "molsim_gpu_iface.F90")).read()
    bound = set(re.findall(r"name='(msg_[a-z0-9_]+)'", f))
    missing = declared_symbols() - bound
    assert not missing, sorted(missing)


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """Every struct of include/molsim_gpu.h has the same size and field offsets in the ctypes
    mirror as gcc gives it (a small C program compiled against the header prints them)."""
    import shutil
    import subprocess

    import pytest

    if not shutil.which("gcc"):
        pytest.skip("gcc is not installed")
    structs = {"msg_params": _lib.MsgParams, "msg_energy": _lib.MsgEnergy, "msg_mc_params": _lib.MsgMcParams,
               "msg_mcall_params": _lib.MsgMcAllParams, "msg_site_ewald": _lib.MsgSiteEwald,
               "msg_tab_params": _lib.MsgTabParams}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "molsim_gpu.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in cls._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines += ["return 0; }"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in structs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_oracle_params_match_the_c_layout(tmp_path):
    """The oracle's or_params and its ctypes mirror (pyoracle.Params) agree field by field."""
    import shutil
    import subprocess

    import pytest

    if not shutil.which("gcc"):
        pytest.skip("gcc is not installed")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "oracle.h"', "int main(void) {",
             'printf("size %zu\\n", sizeof(or_params));']
    for fname, _ in O.Params._fields_:
        lines.append('printf("%s %%zu\\n", offsetof(or_params, %s));' % (fname, fname))
    lines += ["return 0; }"]
    src = tmp_path / "olayout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "olayout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "oracle"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {l.split()[0]: int(l.split()[1]) for l in out if l.strip()}
    assert got["size"] == C.sizeof(O.Params)
    for fname, _ in O.Params._fields_:
        assert got[fname] == getattr(O.Params, fname).offset, fname


def test_fortran_types_follow_the_c_structs():
    """Each bind(c) type of the Fortran module lists the fields of its C struct in the same order
    (no Fortran compiler here: the declarations are compared as text)."""
    f = open(os.path.join(ROOT, "molsim_b200", "fortran", "molsim_gpu_iface.F90")).read()
    h = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "molsim_gpu.h")).read(), flags=re.S)
    ftypes = re.findall(r"type, bind\(c\) :: (\w+)\n(.*?)end type \1", f, flags=re.S)
    assert len(ftypes) >= 5
    for name, body in ftypes:
        fnames = []
        for line in body.split("\n"):
            line = line.split("!")[0]
            if "::" not in line:
                continue
            decl = re.sub(r"\([^)]*\)", "", line.split("::", 1)[1])
            fnames += [x.strip() for x in decl.split(",") if x.strip()]
        m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), h, flags=re.S)
        assert m, name
        cnames = []
        for stmt in m.group(1).split(";"):
            stmt = re.sub(r"\[[^\]]*\]", "", stmt).strip()
            if not stmt:
                continue
            parts = [p.strip() for p in stmt.split(",")]
            first = parts[0].replace("*", " ").split()[-1]
            cnames += [first] + [p.replace("*", "").strip() for p in parts[1:]]
        assert fnames == cnames, (name, fnames, cnames)
