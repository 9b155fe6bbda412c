"""Standard Ewald reciprocal space (txewaldrec 'std': UEwaldRecStd with
EwaldSetArray, Src/energy.F90:964-1104, 1401-1426; kfac and ncut from EwaldSetup,
Src/energy.F90:6752-6782, 7066-7081) against the FP64 oracle.

Bars: forces within 1e-5 relative RMS (the FP64 path lands near 1e-12); u%tot
and the virial within 1e-7 relative in both paths; u%rec within 1e-9 in both,
since the standard-Ewald chain is FP64 in both precision modes.
"""
import numpy as np
import pytest

import helpers as Hp
import pyoracle as O
from molsim_b200 import Engine, MolsimGpuError, alpha_to_ncut
from molsim_b200.engine import estimate_bytes

FORCE_TOL = 1e-5
ENERGY_TOL = 1e-7


# ---------------------------------------------------------------- CPU

def test_alpha_to_ncut_matches_oracle():
    for tol, L, alpha in ((1e-5, 100.0, 0.0876), (1e-7, 40.0, 0.2), (1e-3, 250.0, 0.11)):
        assert alpha_to_ncut(tol, 1.0, 17.72, L, alpha) == O.alpha_to_ncut(tol, 1.0, 17.72, L, alpha)


def test_ncut_outside_range_is_rejected():
    s = Hp.std_ewald(Hp.electrolyte_small())
    t = Hp.oracle_table(s)
    assert estimate_bytes(s, t, "fp64") > 0
    for bad in (0, 101):
        tb = dict(t)
        tb["ncut"] = bad
        with pytest.raises(MolsimGpuError) as ei:
            estimate_bytes(s, tb, "fp64")
        assert ei.value.code == 6


# ---------------------------------------------------------------- GPU

def _pair(s, precision):
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    return t, o, Engine(s, t, precision=precision)


MIXED_ENERGY_TOL = 1e-7     # the mixed mode's pair terms are FP64 sums of unbiased FP32 terms
UREC_TOL = 1e-9             # u%rec comes from the FP64 chain alone in both modes


def _check(ro, rg, ftol, etol=ENERGY_TOL):
    assert Hp.rel_rms(rg["force"], ro["force"]) < ftol
    assert Hp.rel_rms(rg["forceo"], ro["forceo"]) < ftol
    assert Hp.rel(rg["urec"], ro["urec"]) < UREC_TOL, (rg["urec"], ro["urec"])
    for k in ("utot", "virial"):
        assert Hp.rel(rg[k], ro[k]) < etol, (k, rg[k], ro[k])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("region", ["sphere", "cube"])
@pytest.mark.parametrize("lsurf", [False, True])
def test_utotal_against_oracle(precision, region, lsurf):
    s = Hp.std_ewald(Hp.electrolyte_small(lsurf=lsurf), ncut=5 if region == "cube" else None, region=region)
    t, o, g = _pair(s, precision)
    ro, rg = o.utotal(), g.UTotal()
    if precision == "fp64":
        _check(ro, rg, 1e-10)
    else:
        _check(ro, rg, FORCE_TOL, MIXED_ENERGY_TOL)


@pytest.mark.gpu
def test_config0_electrolyte_std():
    """The 1000-ion electrolyte (L = 100 A, rc = 30 A) with ncut from AlphaToNcut at 1e-5."""
    s = Hp.std_ewald(Hp.config0())
    t, o, g = _pair(s, "fp64")
    assert t["ncut"] >= 8
    ro, rg = o.utotal(), g.UTotal()
    _check(ro, rg, 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mixed_methods_in_one_handle_equal_alone(precision):
    """An SPME system and a standard-Ewald system advanced in one handle give what
    each gives alone (mixed: bit for bit; FP64: the SPME grid's FP64 atomics repeat
    only to rounding)."""
    a = dict(Hp.electrolyte_small())
    b = Hp.std_ewald(Hp.electrolyte_small(n_pairs=50, L=36.0, seed=4))
    ta, tb = Hp.oracle_table(a), Hp.oracle_table(b)
    both = Engine([a, b], [ta, tb], precision=precision)
    both.UTotal(0)
    both.GetLinAcc()
    both.VelVer(5, energies=False)
    for k, (s, t) in enumerate(((a, ta), (b, tb))):
        one = Engine(s, t, precision=precision)
        one.UTotal()
        one.GetLinAcc()
        one.VelVer(5, energies=False)
        x, y = both.get_state(k)["ro"], one.get_state(0)["ro"]
        ex, ey = both.energy(k), one.energy(0)
        if precision == "mixed":
            assert np.array_equal(x, y)
            assert ex == ey
        else:
            assert np.abs(x - y).max() <= 1e-10 * np.abs(y).max()
            for key in ("utot", "urec", "virial"):
                assert abs(ex[key] - ey[key]) <= 1e-10 * abs(ey[key])


@pytest.mark.gpu
def test_velver_short_trajectory_std():
    """Ten velocity-Verlet steps with the standard Ewald sum against the oracle."""
    s = Hp.std_ewald(Hp.electrolyte_small(lsurf=True))
    s["tstep"] = 0.01
    t, o, g = _pair(s, "fp64")
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
    box = s["boxlen"][0]
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-9
    assert Hp.rel_rms(sg["rod"], so["rod"]) < 1e-9


@pytest.mark.gpu
def test_repeat_is_bitwise_mixed():
    s = Hp.std_ewald(Hp.pe_small())
    t = Hp.oracle_table(s)
    g = Engine(s, t, precision="mixed")
    r1 = g.UTotal()
    r2 = g.UTotal()
    assert np.array_equal(r1["force"], r2["force"])
    assert r1["urec"] == r2["urec"] and r1["virial"] == r2["virial"]


@pytest.mark.gpu
def test_bd_with_injected_noise_std():
    """Brownian dynamics (BDStep, Src/bd.F90:120-155) with the caller's noise on the
    standard Ewald sum: five steps against the oracle."""
    s = Hp.std_ewald(Hp.colloid_small())
    t, o, g = _pair(s, "fp64")
    o.utotal()
    g.UTotal()
    rng = np.random.default_rng(9)
    xi = rng.standard_normal((5, s["np"], 3))
    fac1, fac2 = s["bd_fac"]
    eg = g.BDStep(5, xi=xi)
    for k in range(5):
        o.bd_step(xi[k], fac1, fac2)
    d = g.get_state()["ro"] - o.get_state()["ro"]
    box = s["boxlen"][0]
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-9
    rg, ro = g.UTotal(), o.utotal()
    _check(ro, rg, 1e-10)
    assert Hp.rel(eg[-1]["utot"], ro["utot"]) < ENERGY_TOL
