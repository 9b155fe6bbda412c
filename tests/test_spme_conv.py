"""The SPME convolution kernel (own mixed-radix FFT and influence multiply in one
persistent launch, switched on with MSG_SPME_CONV=1 at handle creation) against the
cuFFT chain it replaces (the default) and against the FP64 oracle.

Grid edges cover every radix of the kernel's transform (8, 5, 4, 3, 2; two to three
passes) and one edge it leaves to cuFFT (14 = 2 * 7), alone and in one handle with
edges that it takes.
"""
import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine

pytestmark = pytest.mark.gpu

EDGES = [16, 20, 24, 30, 40, 48, 64, 96]


def _system(edge, seed=1):
    s = dict(Hp.electrolyte_small(seed=seed))
    s["nmesh"] = edge
    return s


def _conv_engine(monkeypatch, *args, **kw):
    """A handle created with the convolution kernel switched on (MSG_SPME_CONV=1)."""
    monkeypatch.setenv("MSG_SPME_CONV", "1")
    try:
        return Engine(*args, **kw)
    finally:
        monkeypatch.delenv("MSG_SPME_CONV")


def _pair_of_engines(s, t, precision, monkeypatch):
    return _conv_engine(monkeypatch, s, t, precision=precision), Engine(s, t, precision=precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("edge", EDGES)
def test_conv_matches_cufft(edge, precision, monkeypatch):
    """Same reciprocal energy and virial as the cuFFT chain to the resolution of their
    sums (each path adds its partial sums as 2^-32 fixed point, the convolution kernel one
    per z slab, the cuFFT chain's multiply one per 512 spectrum entries, so the totals
    differ by a few quanta times EpsiFourPi); same forces to FP64 rounding on the FP64 path
    and to FP32 rounding on the mixed path (FP32 backward transforms)."""
    s = _system(edge)
    t = Hp.oracle_table(s)
    g, c = _pair_of_engines(s, t, precision, monkeypatch)
    rg, rc = g.UTotal(), c.UTotal()
    for k in ("urec", "virial", "utot"):
        assert Hp.rel(rg[k], rc[k]) < 2e-8, (k, rg[k], rc[k])
    ftol = 1e-11 if precision == "fp64" else 2e-6
    assert Hp.rel_rms(rg["force"], rc["force"]) < ftol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("edge", [24, 40, 64])
def test_conv_matches_oracle(edge, precision, monkeypatch):
    """UTotal through the convolution kernel against the FP64 oracle at the parity bars
    (forces 1e-5 relative RMS, energies and virial 1e-7 relative)."""
    s = _system(edge, seed=2)
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    ro, rg = o.utotal(), _conv_engine(monkeypatch, s, t, precision=precision).UTotal()
    assert Hp.rel_rms(rg["force"], ro["force"]) < 1e-5
    for k in ("utot", "urec", "virial"):
        assert Hp.rel(rg[k], ro[k]) < 1e-7, (k, rg[k], ro[k])
    if precision == "fp64":
        assert Hp.rel_rms(rg["force"], ro["force"]) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mixed_edges_in_one_handle_equal_alone(precision, monkeypatch):
    """Edges the kernel takes and an edge left to cuFFT in one handle: each system's
    result equals its result alone, bit for bit, and repeats bit for bit."""
    sys_list = [_system(64, seed=3), _system(14, seed=4), _system(24, seed=5), _system(64, seed=6)]
    tabs = [Hp.oracle_table(s) for s in sys_list]
    gb = _conv_engine(monkeypatch, sys_list, tabs, precision=precision)
    first = [gb.UTotal(k) for k in range(len(sys_list))]
    again = [gb.UTotal(k) for k in range(len(sys_list))]
    for k, (s, t) in enumerate(zip(sys_list, tabs)):
        ra = _conv_engine(monkeypatch, s, t, precision=precision).UTotal()
        for rb in (first[k], again[k]):
            assert np.array_equal(rb["force"], ra["force"]), k
            assert rb["urec"] == ra["urec"] and rb["virial"] == ra["virial"] and rb["utot"] == ra["utot"], k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_conv_trajectory_matches_cufft(precision, monkeypatch):
    """Twenty velocity-Verlet steps (the convolution kernel inside the step graph, with
    list rebuilds) stay on the cuFFT chain's trajectory."""
    s = dict(Hp.pe_small())
    s["tstep"] = 0.02
    s["drnlist"] = 0.6
    t = Hp.oracle_table(s)
    g, c = _pair_of_engines(s, t, precision, monkeypatch)
    for e in (g, c):
        e.UTotal()
        e.GetLinAcc()
    eg, ec = g.VelVer(20), c.VelVer(20)
    tol = 1e-10 if precision == "fp64" else 1e-6
    for x, y in zip(eg, ec):
        assert Hp.rel(x["utot"], y["utot"]) < tol
    assert np.abs(g.get_state()["ro"] - c.get_state()["ro"]).max() < (1e-8 if precision == "fp64" else 1e-4)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_conv_blocks_do_not_change_results(precision, monkeypatch):
    """Blocks per SM of the convolution kernel (MSG_TUNE_CONV_BLOCKS) move work between
    blocks only: forces and energies stay bit for bit the same."""
    from molsim_b200 import _lib

    sys_list = [_system(64, seed=7), _system(24, seed=8)]
    tabs = [Hp.oracle_table(s) for s in sys_list]
    g = _conv_engine(monkeypatch, sys_list, tabs, precision=precision)
    ref = [g.UTotal(k) for k in range(2)]
    for blocks in (1, 3, 0):
        assert _lib.lib().msg_tune(g.h, _lib.MSG_TUNE_CONV_BLOCKS, blocks) == 0
        for k in range(2):
            r = g.UTotal(k)
            assert np.array_equal(r["force"], ref[k]["force"])
            assert r["urec"] == ref[k]["urec"] and r["virial"] == ref[k]["virial"]
    assert _lib.lib().msg_tune(g.h, _lib.MSG_TUNE_CONV_BLOCKS, -1) != 0
