"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the
FP64 oracle): the oracle must reproduce them bit for bit (CPU), and the CUDA path
must match them within the parity bars (GPU)."""
import glob
import os
import sys

import numpy as np
import pytest

import helpers as Hp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as G  # noqa: E402

FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def test_fixtures_exist():
    assert len(FIXTURES) >= 2


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_reproduces_fixture(path):
    s, t, want = G.load(path)
    # the table itself: PotTwoBodyTab from the stored potential parameters
    t2 = Hp.oracle_table(s)
    assert t2["ualpha"] == t["ualpha"]
    assert np.array_equal(t2["ubuf"], t["ubuf"]) and np.array_equal(t2["iubuflow"], t["iubuflow"])
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    nn, jp = o.get_vlist()
    assert np.array_equal(nn, want["nneighpn"]) and np.array_equal(jp, want["jpnlist"])
    u = o.utotal()
    assert np.array_equal(u["force"], want["force"])
    for k in ("utot", "urec", "ubond", "virial"):
        assert u[k] == want[k], k
    st = o.get_state()
    o.set_state(st["ro"], st["rod"], u["forceo"] / np.asarray(s["masspt"])[np.asarray(s["iptpn"]) - 1][:, None])
    for _ in range(3):
        o.velver_step()
    st3 = o.get_state()
    assert np.array_equal(st3["ro"], want["ro3"]) and np.array_equal(st3["rod"], want["rod3"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_cuda_path_matches_fixture(path, precision):
    from molsim_b200 import Engine

    s, t, want = G.load(path)
    g = Engine(s, t, precision=precision)
    nn, jp, npair = g.SetVList(0, export=True, maxnneigh=want["jpnlist"].shape[1])
    assert np.array_equal(nn, want["nneighpn"])
    for ip in range(s["np"]):
        assert np.array_equal(jp[ip, :nn[ip]], want["jpnlist"][ip, :nn[ip]])
    r = g.UTotal()
    assert Hp.rel_rms(r["force"], want["force"]) <= 1e-5
    etol = 1e-7 if precision == "fp64" else 1e-6
    scale = abs(want["utot"]) + abs(want["urec"]) + abs(want["utwob"][0])
    for k in ("utot", "urec", "virial"):
        assert abs(r[k] - want[k]) <= etol * max(abs(want[k]), scale if precision == "mixed" else 0.0), k
    g.GetLinAcc()
    g.VelVer(3, energies=False)
    st = g.get_state(0)
    L = s["boxlen"][0]
    d = st["ro"] - want["ro3"]
    d -= L * np.round(d / L)
    assert np.abs(d).max() <= (1e-9 if precision == "fp64" else 1e-5) * L
