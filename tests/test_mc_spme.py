"""Monte Carlo with SPME reciprocal space (DUTwoBodyEwaldRecSPM, Src/denergy.F90:1413-1495:
the trial's charge mesh re-transformed, u%rec(trial) - u%rec(current) with the energy
weights of UEwaldRecSPM) on the GPU against the oracle.

The oracle restates the reference's way: it re-spreads the moved particle's stencil and
transforms the whole mesh for every trial.  The GPU forms the same difference from the
pass's starting spectrum and the transforms of the two stencils (separable along x, y, z),
so the two agree to rounding: the same moves, bit-identical positions, energies within
1e-9 of the energy scale."""
import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine
from molsim_b200 import systems as S


def _oracle(s, t):
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    return o


@pytest.mark.parametrize("lsurf", [False, True])
def test_oracle_carried_energy_equals_fresh_utotal(lsurf):
    s = dict(Hp.electrolyte_small(lsurf=lsurf))
    t = Hp.oracle_table(s)
    o = _oracle(s, t)
    u = o.utotal()
    o.mc_seed(5)
    acc, _ = o.mc_pass(2, [2.0] * s["npt"], 1.0 / S.kT(s["temp"]), u)
    assert acc > 0
    o.set_vlist()
    fresh = o.utotal()
    sc = abs(fresh["utwob"][0]) + abs(fresh["urec"]) + 1.0
    for k in ("utot", "urec"):
        assert abs(u[k] - fresh[k]) <= 1e-9 * sc, (k, u[k], fresh[k])


def _scale(u):
    return abs(u["utwob"][0]) + abs(u["urec"]) + abs(u["ubond"]) + 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("isamp", [0, 1])
@pytest.mark.parametrize("which", ["electrolyte", "electrolyte_surf", "polyelectrolyte"])
def test_gpu_chain_matches_oracle(which, isamp):
    s = {"electrolyte": lambda: Hp.electrolyte_small(),
         "electrolyte_surf": lambda: Hp.electrolyte_small(lsurf=True),
         "polyelectrolyte": lambda: Hp.pe_small()}[which]()
    s = dict(s)
    t = Hp.oracle_table(s)
    beta = 1.0 / S.kT(s["temp"])
    dtran = [2.0] * s["npt"] if isamp == 0 else [-3.0] * s["npt"]
    o = _oracle(s, t)
    u = o.utotal()
    o.mc_seed(7)
    acc, hs = o.mc_pass(2, dtran, beta, u, isamp=isamp)
    g = Engine(s, t, precision="fp64")
    g.mc_seed(7)
    ag, hg, eg = g.MCPass(2, dtran, beta, isamp)
    assert (int(ag[0]), int(hg[0])) == (acc, hs)
    assert np.array_equal(g.get_state()["ro"], o.get_state()["ro"])
    sc = _scale(u)
    for k in ("utot", "urec", "ubond"):
        assert abs(eg[k] - u[k]) <= 1e-9 * sc, (k, eg[k], u[k])


@pytest.mark.gpu
def test_gpu_carried_energy_equals_fresh_utotal_mixed():
    """A mixed-precision handle runs the same FP64 chain; its carried energy matches a fresh
    UTotal to the FP32 pair terms' precision."""
    s = dict(Hp.electrolyte_small(lsurf=True))
    t = Hp.oracle_table(s)
    g = Engine(s, t, precision="mixed")
    g.mc_seed(3)
    _, _, e = g.MCPass(2, [2.0] * s["npt"], 1.0 / S.kT(s["temp"]))
    fresh = g.UTotal()
    assert abs(e["utot"] - fresh["utot"]) <= 1e-6 * _scale(fresh)
    assert abs(e["urec"] - fresh["urec"]) <= 1e-6 * _scale(fresh)


@pytest.mark.gpu
def test_gpu_spme_and_std_systems_in_one_handle():
    """An SPME system and a standard-Ewald system in one handle run the chains they run alone."""
    a = dict(Hp.electrolyte_small())
    b = Hp.std_ewald(Hp.electrolyte_small(n_pairs=50, L=36.0, seed=4))
    ta, tb = Hp.oracle_table(a), Hp.oracle_table(b)
    beta = [1.0 / S.kT(a["temp"]), 1.0 / S.kT(b["temp"])]
    both = Engine([a, b], [ta, tb], precision="fp64")
    for k in range(2):
        both.mc_seed(30 + k, isys=k)
    acc, _, _ = both.MCPass(2, [[2.0] * a["npt"], [2.0] * b["npt"]], beta)
    for k, (s, t) in enumerate(((a, ta), (b, tb))):
        one = Engine(s, t, precision="fp64")
        one.mc_seed(30 + k)
        a1, _, _ = one.MCPass(2, [2.0] * s["npt"], beta[k])
        assert int(a1[0]) == int(acc[k])
        assert np.array_equal(one.get_state()["ro"], both.get_state(k)["ro"])
