"""The 2D layer correction of the standard Ewald sum (lewald2dlc: UEwaldRecStd2dlc with
EwaldSetArray2d, Src/energy.F90:1106-1203, 1435-1463; kfac2d from EwaldSetup,
:6785-6851; UEwaldSurf's 2d-periodic form, :1362-1369) on the GPU against the oracle.

The oracle's restatement is pinned two ways: its forces are -grad u%tot (central
differences), and on a slab of ions the corrected energy does not depend on the box
height, while the uncorrected 3D sum moves by kJ/mol.  GPU bars as for the standard
sum: forces within 1e-10 relative RMS and u%rec within 1e-9 (FP64 chain)."""
import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine, MolsimGpuError


def _oracle(s):
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    return t, o


def test_oracle_forces_are_the_energy_gradient():
    s = Hp.slab_small()
    t, o = _oracle(s)
    u = o.utotal()
    ro = np.array(s["ro"])
    h = 1e-5
    fmax = np.abs(u["force"]).max()
    for i in (0, 7, 63):
        for c in range(3):
            up, dn = ro.copy(), ro.copy()
            up[i, c] += h
            dn[i, c] -= h
            o.set_state(up, s["rod"])
            eu = o.utotal()["utot"]
            o.set_state(dn, s["rod"])
            ed = o.utotal()["utot"]
            assert abs(-(eu - ed) / (2 * h) - u["force"][i, c]) < 1e-6 * fmax, (i, c)


def test_oracle_energy_does_not_depend_on_the_box_height():
    """With the correction the slab's u%tot at Lz = 80, 120 and 200 A agrees within 2e-3
    kJ/mol (ncut grown with Lz); the uncorrected sum (3D surface term) moves by over 1 kJ/mol."""
    for elc, ok in ((True, lambda d: d < 2e-3), (False, lambda d: d > 1.0)):
        us = []
        for Lz in (80.0, 120.0, 200.0):
            s = Hp.slab_small(Lz=Lz, ncut=int(16 * Lz / 120) + 1, elc=elc)
            us.append(_oracle(s)[1].utotal()["utot"])
        assert ok(max(us) - min(us)), (elc, us)


@pytest.mark.gpu
@pytest.mark.parametrize("region,lsurf", [("sphere", True), ("cube", False), ("sphere", False)])
def test_gpu_utotal_against_oracle(region, lsurf):
    s = Hp.slab_small(lsurf=lsurf, ncut=10 if region == "cube" else 12, region=region)
    t, o = _oracle(s)
    ro = o.utotal()
    rg = Engine(s, t, precision="fp64").UTotal()
    assert Hp.rel_rms(rg["force"], ro["force"]) < 1e-10
    assert Hp.rel(rg["urec"], ro["urec"]) < 1e-9, (rg["urec"], ro["urec"])
    for k in ("utot", "virial"):
        assert Hp.rel(rg[k], ro[k]) < 1e-7, (k, rg[k], ro[k])


@pytest.mark.gpu
def test_gpu_spme_takes_the_2d_surface_term():
    """With SPME the flag changes only UEwaldSurf to its 2d-periodic form."""
    s = Hp.slab_small()
    s["ewaldrec"] = "spm"
    t, o = _oracle(s)
    ro = o.utotal()
    rg = Engine(s, t, precision="fp64").UTotal()
    assert Hp.rel_rms(rg["force"], ro["force"]) < 1e-10
    assert Hp.rel(rg["urec"], ro["urec"]) < 1e-9


@pytest.mark.gpu
def test_gpu_velver_short_trajectory():
    """Ten velocity-Verlet steps of the slab with the correction against the oracle."""
    s = Hp.slab_small()
    s["tstep"] = 0.01
    t, o = _oracle(s)
    g = Engine(s, t, precision="fp64")
    o.utotal()
    st = o.get_state()
    g.UTotal()
    g.GetLinAcc()
    o.set_state(st["ro"], st["rod"], g.get_state()["rodd"])
    eg = g.VelVer(10)
    for k in range(10):
        ek, _ = o.velver_step()
        assert Hp.rel(eg[k]["ekin"], ek) < 1e-9
    sg, so = g.get_state(), o.get_state()
    d = sg["ro"] - so["ro"]
    box = np.asarray(s["boxlen"])
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-9
    assert Hp.rel(eg[-1]["urec"], o.utotal()["urec"]) < 1e-9


def test_oracle_mc_running_energy_equals_fresh_utotal():
    """Monte Carlo with the correction (DUTwoBodyEwaldRec2dlc and the 2d-periodic surface
    difference): the energies carried by the accepted moves equal a fresh UTotal of the
    final configuration."""
    from molsim_b200 import systems as S

    s = Hp.slab_small()
    t, o = _oracle(s)
    u = o.utotal()
    o.mc_seed(11)
    acc, _ = o.mc_pass(2, [2.0] * s["npt"], 1.0 / S.kT(s["temp"]), u)
    assert acc > 0
    o.set_vlist()
    fresh = o.utotal()
    sc = abs(fresh["utwob"][0]) + abs(fresh["urec"]) + 1.0
    for k in ("utot", "urec"):
        assert abs(u[k] - fresh[k]) <= 1e-9 * sc, (k, u[k], fresh[k])


@pytest.mark.gpu
@pytest.mark.parametrize("isamp", [0, 1])
def test_gpu_mc_chain_matches_oracle(isamp):
    """The GPU chain with the correction makes the oracle's moves: the same acceptances,
    bit-identical positions, energies within 1e-9 of the energy scale."""
    from molsim_b200 import systems as S

    s = Hp.slab_small()
    t, o = _oracle(s)
    beta = 1.0 / S.kT(s["temp"])
    dtran = [2.0] * s["npt"] if isamp == 0 else [-3.0] * s["npt"]
    u = o.utotal()
    o.mc_seed(7)
    acc, hs = o.mc_pass(2, dtran, beta, u, isamp=isamp)
    g = Engine(s, t, precision="fp64")
    g.mc_seed(7)
    ag, hg, eg = g.MCPass(2, dtran, beta, isamp)
    assert (int(ag[0]), int(hg[0])) == (acc, hs)
    assert np.array_equal(g.get_state()["ro"], o.get_state()["ro"])
    sc = abs(u["utwob"][0]) + abs(u["urec"]) + 1.0
    for k in ("utot", "urec"):
        assert abs(eg[k] - u[k]) <= 1e-9 * sc, (k, eg[k], u[k])
