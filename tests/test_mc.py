"""Monte Carlo single-particle translations (MCPass with SPartMove, Src/mc.F90:1470-1755;
DUTotal, Src/denergy.F90:110-230; Metropolis and MCUpdate, Src/mc.F90:5135-5236) on
the GPU against the oracle.

The device draws the reference's random numbers (Random, Src/mollib.F90:2689-2708)
in the reference's order, so the chains agree move for move: the same moves are
accepted and the final positions are bit-identical; the energies carried by the
accepted moves agree within 1e-9 of the energy scale (the sums differ in rounding
order only)."""
import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine, MolsimGpuError
from molsim_b200 import systems as S

pytestmark = pytest.mark.gpu

ETOL = 1e-9


def _systems():
    a = Hp.std_ewald(Hp.electrolyte_small())
    b = Hp.std_ewald(Hp.electrolyte_small(lsurf=True))
    c = Hp.std_ewald(Hp.pe_small())
    d = dict(Hp.electrolyte_small())
    d["lewald"] = False
    return {"std": a, "std_surf": b, "std_bonds": c, "noewald": d}


def _oracle_run(s, t, npass, dtran, beta, isamp, seed):
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    u = o.utotal()
    o.mc_seed(seed)
    acc, hs = o.mc_pass(npass, dtran, beta, u, isamp=isamp)
    return o, u, acc, hs


def _scale(u):
    return abs(u["utwob"][0]) + abs(u["urec"]) + abs(u["ubond"]) + 1.0


@pytest.mark.parametrize("isamp", [0, 1])
@pytest.mark.parametrize("which", ["std", "std_surf", "std_bonds", "noewald"])
def test_chain_matches_oracle(which, isamp):
    s = _systems()[which]
    t = Hp.oracle_table(s)
    beta = 1.0 / S.kT(s["temp"])
    dtran = [2.0] * s["npt"] if isamp == 0 else [-3.0] * s["npt"]
    o, u, acc, hs = _oracle_run(s, t, 2, dtran, beta, isamp, 7)
    g = Engine(s, t, precision="fp64")
    g.mc_seed(7)
    ag, hg, eg = g.MCPass(2, dtran, beta, isamp)
    assert (int(ag[0]), int(hg[0])) == (acc, hs)
    assert np.array_equal(g.get_state()["ro"], o.get_state()["ro"])
    sc = _scale(u)
    for k in ("utot", "urec", "ubond"):
        assert abs(eg[k] - u[k]) <= ETOL * sc, (k, eg[k], u[k])
    assert np.abs(np.asarray(eg["utwob"]) - np.asarray(u["utwob"])).max() <= ETOL * sc


def test_carried_energy_equals_fresh_utotal_and_continues():
    """The energies after the sweeps equal a fresh UTotal of the final configuration,
    and a second call continues the same random stream (its chain equals the oracle's
    two-call chain)."""
    s = _systems()["std_surf"]
    t = Hp.oracle_table(s)
    beta = 1.0 / S.kT(s["temp"])
    g = Engine(s, t, precision="fp64")
    g.mc_seed(3)
    _, _, e1 = g.MCPass(1, [2.5] * s["npt"], beta)
    fresh = g.UTotal()
    sc = _scale(fresh)
    for k in ("utot", "urec"):
        assert abs(e1[k] - fresh[k]) <= ETOL * sc
    a2, _, _ = g.MCPass(1, [2.5] * s["npt"], beta)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    u = o.utotal()
    o.mc_seed(3)
    o.mc_pass(1, [2.5] * s["npt"], beta, u)
    o.set_vlist()
    u = o.utotal()
    acc2, _ = o.mc_pass(1, [2.5] * s["npt"], beta, u)
    assert int(a2[0]) == acc2
    assert np.array_equal(g.get_state()["ro"], o.get_state()["ro"])


def test_batch_equals_alone():
    sy = _systems()
    names = ["std", "std_bonds", "noewald"]
    ss = [sy[k] for k in names]
    ts = [Hp.oracle_table(s) for s in ss]
    beta = [1.0 / S.kT(s["temp"]) for s in ss]
    dtran = [[2.0] * s["npt"] for s in ss]
    both = Engine(ss, ts, precision="fp64")
    for k in range(len(ss)):
        both.mc_seed(20 + k, isys=k)
    acc, _, _ = both.MCPass(2, dtran, beta)
    for k, (s, t) in enumerate(zip(ss, ts)):
        one = Engine(s, t, precision="fp64")
        one.mc_seed(20 + k)
        a1, _, _ = one.MCPass(2, dtran[k], beta[k])
        assert int(a1[0]) == int(acc[k])
        assert np.array_equal(one.get_state()["ro"], both.get_state(k)["ro"])


def test_mixed_handle_runs_the_same_chain():
    """The chain is FP64 in both precision modes: a mixed-precision handle makes the
    same moves; only its starting energies carry the FP32 pair terms."""
    s = _systems()["std"]
    t = Hp.oracle_table(s)
    beta = 1.0 / S.kT(s["temp"])
    gd = Engine(s, t, precision="fp64")
    gm = Engine(s, t, precision="mixed")
    for g in (gd, gm):
        g.mc_seed(5)
    ad, _, ed = gd.MCPass(2, [2.0] * s["npt"], beta)
    am, _, em = gm.MCPass(2, [2.0] * s["npt"], beta)
    assert int(ad[0]) == int(am[0])
    assert np.array_equal(gd.get_state()["ro"], gm.get_state()["ro"])
    assert abs(ed["utot"] - em["utot"]) <= 1e-6 * _scale(ed)


def test_zero_sweeps_and_bad_arguments():
    """npass = 0 returns the current energies (a UTotal) and moves nothing; an isamp
    other than 0 or 1 and a missing dtran are refused with MSG_ERR_ARG."""
    import ctypes as C

    from molsim_b200 import _lib

    s = _systems()["std"]
    t = Hp.oracle_table(s)
    g = Engine(s, t, precision="fp64")
    ro0 = g.get_state()["ro"]
    acc, hs, e = g.MCPass(0, [2.0] * s["npt"], 1.0)
    assert int(acc[0]) == 0 and int(hs[0]) == 0
    assert np.array_equal(g.get_state()["ro"], ro0)
    u = g.UTotal()
    assert abs(e["utot"] - u["utot"]) <= 1e-12 * abs(u["utot"])
    with pytest.raises(MolsimGpuError) as ei:
        g.MCPass(1, [2.0] * s["npt"], 1.0, isamp=2)
    assert ei.value.code == 6
    par = (_lib.MsgMcParams * 1)()
    par[0] = _lib.MsgMcParams(1.0, C.POINTER(C.c_double)(), 0, 0)
    assert _lib.lib().msg_mc_pass(g.h, 1, par, None, None, 0, None) == 6
