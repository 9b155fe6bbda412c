"""Pins of the FP64 oracle (oracle/oracle.c) against known answers.

The reference ships no golden outputs (its Testin/ diffs against a locally
generated out_stable/), so the oracle is pinned by
  * the reference's own in-code checks restated as tests: CheckUBuffer's
    table tolerance (Src/potential.F90:1224-1258), TestCellList's neighbour
    completeness (Src/celllist.F90:447-476), SPME against an independent Ewald
    sum (TestEwaldSPM / UEwaldRecStd, Src/potential.F90:3211-3378,
    Src/energy.F90:964-1104), RcutToAlpha against EwaldErrorUReal;
  * analytic answers: erf, B-spline identities, the (1,6,12) potential's
    derivatives, two isolated ions, a harmonic bond, the rock-salt Madelung
    constant, and energy conservation of velocity Verlet.
"""
import math

import numpy as np
import pytest

import helpers as Hp
import pyoracle as O
from molsim_b200 import systems as S

EPSFP = S.EPSI0_FOUR_PI / 78.4


def test_erf2_matches_libm():
    xs = np.concatenate([np.linspace(-7, 7, 4001), [1e-12, -1e-12, 2.0, -2.0, 6.2499]])
    err = max(abs(O.erf2(x) - math.erf(x)) for x in xs)
    assert err < 1e-15


def test_ewald_ufac_definitions():
    alpha = 0.0876
    for r in (1.0, 4.0, 12.5, 29.0):
        c = O.ewald_ufac(r, alpha)
        assert abs(c[0] - math.erfc(alpha * r)) < 1e-15
        # c1 = -r^2 d/dr[erfc(a r)/r], c2 = (r^3/2) d2/dr2[erfc(a r)/r]
        # (central differences; the reference's 2/sqrt(pi) is truncated to 1.12837916709)
        h = 1e-4
        f = lambda x: math.erfc(alpha * x) / x
        d1 = (f(r + h) - f(r - h)) / (2 * h)
        d2 = (f(r + h) - 2 * f(r) + f(r - h)) / h ** 2
        assert abs(c[1] - (-r * r * d1)) < 1e-7
        assert abs(c[2] - (r ** 3 / 2 * d2)) < 1e-5


@pytest.mark.parametrize("order", [3, 4, 5, 6])
def test_cardinal_bspline_identities(order):
    rng = np.random.default_rng(order)
    for pos in np.concatenate([rng.uniform(-50, 50, 20), [0.0, 7.0]]):
        k, v, d = O.bspline(order, pos)
        assert k == math.floor(pos)
        assert abs(v.sum() - 1.0) < 1e-14
        assert abs(d.sum()) < 1e-14
        # derivative against a finite difference of the values (same integer part)
        x = pos - math.floor(pos)
        if 1e-3 < x < 1 - 1e-3:
            h = 1e-6
            _, vp, _ = O.bspline(order, pos + h)
            _, vm, _ = O.bspline(order, pos - h)
            assert np.abs((vp - vm) / (2 * h) - d).max() < 1e-7
    # M4 at the half point: 1/48, 23/48, 23/48, 1/48
    if order == 4:
        _, v, _ = O.bspline(4, 0.5)
        assert np.allclose(v, [1 / 48, 23 / 48, 23 / 48, 1 / 48], atol=1e-15)


def _pot(s, alpha, lewald=1):
    return dict(npt=s["npt"], zat=s["zat"], sigat=s["sigat"], epsat=s["epsat"], rcut=s["rcut"], ualpha=alpha,
                epsi_four_pi=s["epsi_four_pi"], lewald=lewald, lljcut=1,
                **{k: s[k] for k in ("ljrcut", "ljushift", "r2uminin", "utoltab", "ftoltab", "umaxtab",
                                     "fmaxtab", "rumaxfac")})


def test_pot_1_6_12_derivatives_and_cut():
    s = Hp.config0()
    pot = _pot(s, 0.0876)
    sig = 4.0
    rc = pot["ljrcut"] * sig
    for r in (3.7, 4.2, 6.0, 15.0, 29.0):
        u0, u1, u2 = O.pot(pot, 1, 2, r)
        h = 1e-5
        up = O.pot(pot, 1, 2, r + h)[0]
        um = O.pot(pot, 1, 2, r - h)[0]
        if abs(r - rc) > 1e-3:
            assert abs((up - um) / (2 * h) - u1) < 1e-6 * max(1.0, abs(u1))
            assert abs((up - 2 * u0 + um) / h ** 2 - u2) < 1e-3 * max(1.0, abs(u2))
    # LJ cut-and-shift at 2^(1/6) sigma: no LJ part beyond, continuous across the cut
    eps = s["epsat"][0]
    lo = O.pot(pot, 1, 1, rc * (1 - 1e-9))[0]
    hi = O.pot(pot, 1, 1, rc * (1 + 1e-9))[0]
    assert abs(lo - hi) < 1e-6 * eps + 1e-9
    # beyond the cut only erfc-screened Coulomb remains
    r = 10.0
    u0 = O.pot(pot, 1, 1, r)[0]
    assert abs(u0 - EPSFP * math.erfc(0.0876 * r) / r) < 1e-12


@pytest.mark.parametrize("which", ["config0", "config1", "colloid_small"])
def test_table_meets_checkubuffer_tolerance(which):
    """Every interval reproduces u and -du/dr within utoltab/ftoltab (CheckUBuffer's bar),
    here on 50 points per interval rather than the reference's 11."""
    s = getattr(Hp, which)()
    t = Hp.oracle_table(s)
    pot = _pot(s, t["ualpha"], int(s["lewald"]))
    ub = t["ubuf"]
    npt = s["npt"]
    p = 0
    for it in range(1, npt + 1):
        for jt in range(it, npt + 1):
            k0 = t["iubuflow"][p] - 1
            rows = ub[k0:k0 + 12 * t["nugrid"][p]].reshape(-1, 12)
            zs = np.concatenate([[(1.1 * s["rcut"]) ** 2], rows[:, 0]])
            for q, c in enumerate(rows):
                zlo, zhi = zs[q + 1], zs[q]
                for r in np.sqrt(np.linspace(zlo, zhi, 50)):
                    d = r * r - c[0]
                    us = c[1] + d * (c[2] + d * (c[3] + d * (c[4] + d * (c[5] + d * c[6]))))
                    fs = c[7] + d * (c[8] + d * (c[9] + d * (c[10] + d * c[11])))
                    u0, u1, _ = O.pot(pot, it, jt, r)
                    assert abs(us - u0) < 1.5e-5
                    assert abs(r * fs * r + u1 * r) < 1.5e-5 * r
            assert abs(rows[-1, 0] - t["r2umin"][p]) == 0.0
            p += 1


def test_rcut_to_alpha_inverts_error_estimate():
    for L, rc in ((100.0, 30.0), (250.0, 25.0), (1200.0, 30.0)):
        a = O.rcut_to_alpha(1e-5, 1.0, EPSFP, L, rc)
        est = O.lib().or_ewald_error_ureal(1.0, L, a, rc, EPSFP)
        assert abs(est / 1e-5 - 1) < 1e-4


@pytest.mark.parametrize("s", [8, 12, 16, 24, 32])
def test_fft_conventions_match_numpy(s):
    q = np.random.default_rng(s).normal(size=(s, s, s))
    F = O.fft3_r2c(q)
    assert np.abs(F - np.fft.rfftn(q)).max() < 1e-12 * s ** 3
    back = O.fft3_c2r(F)
    assert np.abs(back - q * s ** 3).max() < 1e-10 * s ** 3


def _two_ion_system(r, lewald=False, L=400.0):
    s = S.electrolyte(seed=0, n_pairs=1, L=L, rcut=min(150.0, L / 2 - 2), nmesh=16)
    s["lewald"] = lewald
    s["ro"] = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0]])
    s["rod"] = np.zeros((2, 3))
    return s


def test_two_isolated_ions_known_answer():
    """+1 and -1 at r in a large box, plain (unscreened, cut at rcut) Coulomb + shifted LJ."""
    for r in (4.2, 9.0, 40.0):
        s = _two_ion_system(r)
        t = Hp.oracle_table(s)
        o = Hp.oracle_system(s, t)
        o.set_state(s["ro"], s["rod"])
        o.set_vlist()
        res = o.utotal()
        sig, eps = 4.0, s["epsat"][0]
        lj = 0.0
        dlj = 0.0
        if r < s["ljrcut"] * sig:
            x6 = (sig / r) ** 6
            lj = 4 * eps * (x6 * x6 - x6) + eps
            dlj = -24 * eps * (2 * x6 * x6 - x6) / r
        u = -EPSFP / r + lj
        f = -(EPSFP / r ** 2 + dlj)          # force on particle 2 along +x (attraction: negative)
        assert abs(res["utot"] - u) < 1.5e-5
        assert abs(res["force"][1, 0] - f) < 1.5e-5
        assert abs(res["force"][0, 0] + f) < 1.5e-5


def test_harmonic_bond_known_answer():
    s = _two_ion_system(7.0)
    s["epsat"] = np.zeros(2)
    s["zat"] = np.array([1e-9, -1e-9])
    s["az"] = s["zat"][s["iptpn"] - 1].copy()
    s["nbond"] = 1
    s["bond_ij"] = np.array([[1, 2]], np.int32)
    s["bond_p"] = np.array([2], np.int32)
    k = 0.4 * S.kT(298.0)
    s["bond_k"] = np.array([k / 2])
    s["bond_eq"] = np.array([5.0])
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    res = o.utotal()
    assert abs(res["ubond"] - k / 2 * 4.0) < 1e-12
    assert abs(res["force"][1, 0] - (-k * 2.0)) < 1e-10     # pulled back towards r0
    # virial of the bond: -fac*r2 with fac = -p k' (r - r0) / r  (Src/energy.F90:5362-5376)
    assert abs(res["virial"] - (2 * k / 7.0) * 49.0) < 1e-9


def test_madelung_constant_rock_salt():
    """Rock salt with SPME: the Coulomb energy per ion is -M e^2/(4 pi eps a) with
    M = 1.747564594633 (known answer for the reciprocal + real + self sum)."""
    n, a = 8, 4.5
    L = n * a
    grid = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)], float)
    sign = np.where(grid.sum(1) % 2 == 0, 1, 2).astype(np.int32)
    ro = grid * a - L / 2 + 1e-3
    s = S.electrolyte(seed=0, n_pairs=len(ro) // 2, L=L, rcut=L / 2 - 1.0, nmesh=32, order=6)
    s["iptpn"] = sign
    s["az"] = s["zat"][sign - 1].copy()
    s["epsat"] = np.zeros(2)
    s["uewaldtol"] = 1e-7
    s["ro"] = ro
    s["rod"] = np.zeros_like(ro)
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t, maxnneigh=len(ro))
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    res = o.utotal()
    m = 1.747564594633
    expect = -m * EPSFP / a * len(ro) / 2
    # bar: the pair table's own tolerance (utoltab = 1e-5 kJ/mol per pair, about 170
    # pairs per ion inside rcut) limits the agreement to a few 1e-5 relative
    assert abs(res["utot"] / expect - 1) < 1e-4


def _direct_ewald(ro, q, L, alpha, kmax=14):
    """Independent standard Ewald sum (reciprocal part): energy and forces (minus the
    energy gradient), both in units of e^2/A before the EpsiFourPi scale."""
    V = L ** 3
    e = 0.0
    f = np.zeros_like(ro)
    ks = np.arange(-kmax, kmax + 1)
    K = np.array(np.meshgrid(ks, ks, ks, indexing="ij")).reshape(3, -1).T
    K = K[np.any(K != 0, axis=1)] * 2 * np.pi / L
    k2 = (K ** 2).sum(1)
    phase = ro @ K.T
    Sk = (q[:, None] * np.exp(1j * phase)).sum(0)
    w = 4 * np.pi / V * np.exp(-k2 / (4 * alpha ** 2)) / k2
    e = 0.5 * np.sum(w * np.abs(Sk) ** 2)
    f = -(q[:, None] * ((np.imag(np.exp(-1j * phase) * Sk[None, :]) * w[None, :]) @ K))
    return e, f


def test_spme_against_direct_ewald():
    s = dict(Hp.electrolyte_small())
    s["nmesh"] = 32
    s["order"] = 6
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    res = o.utotal()
    # reciprocal energy from the oracle: u%rec / epsfp + self term
    q = np.asarray(s["az"], float)
    alpha = t["ualpha"]
    urec_grid = res["urec"] / s["epsi_four_pi"] + alpha / math.sqrt(math.pi) * np.sum(q * q)
    e, _ = _direct_ewald(np.asarray(s["ro"]), q, s["boxlen"][0], alpha)
    assert abs(urec_grid - e) < 1e-5 * abs(e) + 1e-6


def test_vlist_pair_set_matches_brute_force_and_cells():
    s = dict(Hp.pe_small())
    t = Hp.oracle_table(s)
    o1 = Hp.oracle_system(s, t)
    o1.set_state(s["ro"], s["rod"])
    o1.set_vlist()
    o2 = Hp.oracle_system(s, t, cell=True)
    o2.set_state(s["ro"], s["rod"])
    o2.set_vlist()
    n1, j1 = o1.get_vlist()
    n2, j2 = o2.get_vlist()
    assert np.array_equal(n1, n2)
    for ip in range(s["np"]):
        assert np.array_equal(j1[ip, :n1[ip]], j2[ip, :n2[ip]])
    # every unordered pair within (rcut+drnlist) appears exactly once (TestCellList-style completeness)
    ro = np.asarray(s["ro"])
    L = s["boxlen"][0]
    d = ro[:, None, :] - ro[None, :, :]
    d = np.where(np.abs(d) > L / 2, d - np.copysign(L, d), d)
    r2 = (d * d).sum(-1)
    want = {(a, b) for a in range(len(ro)) for b in range(a + 1, len(ro))
            if r2[a, b] < (s["rcut"] + s["drnlist"]) ** 2}
    got = set()
    for ip in range(s["np"]):
        for jp in j1[ip, :n1[ip]]:
            key = (min(ip, jp - 1), max(ip, jp - 1))
            assert key not in got
            got.add(key)
    assert got == want
    # ownership follows the parity rule of SetVListMD (Src/nlist.F90:741-744), 1-based
    for ip in range(s["np"]):
        for jp in j1[ip, :n1[ip]]:
            a, b = ip + 1, int(jp)
            assert (a < b and (a + b) % 2 == 1) or (a > b and (a + b) % 2 == 0)


def test_skin_test_running_second_maximum():
    """NList's r2max2 only collects values that were not a new running maximum."""
    s = dict(Hp.electrolyte_small())
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    n = s["np"]
    # increasing displacements: every value is a new maximum, so r2max2 stays 0
    d = np.zeros((n, 3))
    d[:, 0] = np.linspace(0.01, 0.4, n)
    o.set_drosum(np.zeros((n, 3)))
    rb, m1, m2 = o.skin_test(d)
    assert m2 == 0.0 and abs(m1 - 0.16) < 1e-12 and not rb
    # decreasing: the first is the maximum, the second-largest is the true runner-up
    o.set_drosum(np.zeros((n, 3)))
    rb, m1, m2 = o.skin_test(d[::-1].copy())
    assert abs(m1 - 0.16) < 1e-12 and abs(m2 - d[-2, 0] ** 2) < 1e-12


def test_gau_random_stream():
    x = O.gau_random_stream(12345, 20000)
    assert abs(x.mean()) < 0.03 and abs(x.std() - 1) < 0.03
    assert np.array_equal(O.gau_random_stream(12345, 8), x[:8])


def test_velocity_verlet_conserves_energy():
    s = dict(Hp.electrolyte_small())
    s["tstep"] = 0.002
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    r = o.utotal()
    m = s["masspt"][s["iptpn"] - 1][:, None]
    o.set_state(s["ro"], s["rod"], r["forceo"] / m)
    e0 = None
    drift = []
    for k in range(300):
        ek, _ = o.velver_step()
        u = o.utotal()["utot"]
        e = ek + u
        e0 = e if e0 is None else e0
        drift.append(e - e0)
    assert max(abs(x) for x in drift) < 2e-3 * abs(ek)


# ---------------------------------------------------------------- standard Ewald

def test_alpha_to_ncut_fixed_point():
    """AlphaToNcut (Src/energy.F90:7066-7081): the 40-step fixed point, restated
    here as a plain loop, and ncut grows as the tolerance tightens."""
    q2, epsfp, L, alpha = 1.0, 17.72, 100.0, 0.0876
    for tol in (1e-3, 1e-5, 1e-7):
        y = (tol / (q2 * epsfp)) * (math.pi ** 2 / (alpha ** 2 * L))
        xo = 1.0
        for _ in range(40):
            xn = (alpha * L / math.pi) * math.sqrt(-math.log(y * xo / (1 + 1 / (alpha * L * math.sqrt(xo)))))
            if abs(xo - xn) / xn < 1e-6:
                break
            xo = xn
        assert O.alpha_to_ncut(tol, q2, epsfp, L, alpha) == int(xn + 1)
    assert O.alpha_to_ncut(1e-3, q2, epsfp, L, alpha) < O.alpha_to_ncut(1e-7, q2, epsfp, L, alpha)


def _std_result(s, ncut, region):
    d = Hp.std_ewald(s, ncut=ncut, region=region)
    t = Hp.oracle_table(d)
    o = Hp.oracle_system(d, t)
    o.set_state(d["ro"], d["rod"])
    o.set_vlist()
    return o.utotal(), t


def test_std_ewald_cube_equals_direct_sum():
    """ncutregion 'cube' sums every k = 2 pi n / L with |n_i| <= ncut, as the direct
    sum above does: the reciprocal energy agrees to rounding, and the difference of
    two cut-offs (which cancels the pair forces) gives the direct sum's force
    difference to rounding."""
    s = dict(Hp.electrolyte_small())
    q = np.asarray(s["az"], float)
    ro = np.asarray(s["ro"], float)
    L = s["boxlen"][0]
    epsfp = s["epsi_four_pi"]
    r6, t = _std_result(s, 6, "cube")
    r3, _ = _std_result(s, 3, "cube")
    alpha = t["ualpha"]
    self_term = alpha / math.sqrt(math.pi) * np.sum(q * q)
    e6, f6 = _direct_ewald(ro, q, L, alpha, kmax=6)
    e3, f3 = _direct_ewald(ro, q, L, alpha, kmax=3)
    assert abs(r6["urec"] / epsfp + self_term - e6) <= 1e-11 * abs(e6)
    assert abs(r3["urec"] / epsfp + self_term - e3) <= 1e-11 * abs(e3)
    df = r6["force"] - r3["force"]
    want = epsfp * (f6 - f3)
    assert Hp.rel_rms(df, want) <= 1e-9


def test_std_ewald_sphere_agrees_with_converged_spme():
    """With ncut from AlphaToNcut at uewaldtol (sphere), standard Ewald and an SPME
    of order 6 on a fine grid compute the same Ewald sum: totals agree to the
    tolerances both methods are set up for."""
    s = dict(Hp.electrolyte_small())
    s["nmesh"] = 48
    s["order"] = 6
    rs, t = _std_result(s, None, "sphere")
    assert t["ncut"] >= 3
    ts = Hp.oracle_table(s)
    o = Hp.oracle_system(s, ts)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    rp = o.utotal()
    assert Hp.rel_rms(rs["force"], rp["force"]) <= 1e-4
    assert Hp.rel(rs["urec"], rp["urec"]) <= 1e-5
    assert Hp.rel(rs["virial"], rp["virial"]) <= 1e-5


# ---------------------------------------------------------------- Monte Carlo

def _random_py(iseed, n):
    """Random (Src/mollib.F90:2689-2708) restated with Python integers: 32-bit
    xorshift and Park-Miller by Schrage's method; am is nearest(1.0,-1.0)/im in
    single precision."""
    am = float(np.float32(np.nextafter(np.float32(1.0), np.float32(0.0))) / np.float32(2147483647))
    a = abs(iseed)
    iy = (888889999 ^ a) | 1
    ix = 777755555 ^ a
    out = []
    for _ in range(n):
        ix &= 0xFFFFFFFF
        ix ^= (ix << 13) & 0xFFFFFFFF
        ix ^= ix >> 17
        ix ^= (ix << 5) & 0xFFFFFFFF
        k = iy // 127773
        iy = 16807 * (iy - k * 127773) - 2836 * k
        if iy < 0:
            iy += 2147483647
        six = ix - (1 << 32) if ix >= (1 << 31) else ix
        out.append(am * ((2147483647 & (six ^ iy)) | 1))
    return np.array(out)


def test_random_stream_matches_restatement():
    for seed in (1, 17, 123457, -5):
        a = O.random_stream(seed, 2000)
        b = _random_py(seed, 2000)
        assert np.array_equal(a, b)
        assert a.min() > 0.0 and a.max() < 1.0
        assert abs(a.mean() - 0.5) < 0.03


def _mc_system(s, seed=11):
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    u = o.utotal()
    o.mc_seed(seed)
    return o, u


@pytest.mark.parametrize("which", ["std", "std_surf", "std_bonds", "noewald"])
def test_mc_running_energy_equals_fresh_utotal(which):
    """After MC sweeps the energies carried by the accepted moves' differences
    (MCUpdate) equal a fresh UTotal of the final configuration: the restatement's
    DUTotal is consistent with its UTotal (the check MOLSIM's TestSimulation makes)."""
    if which == "std":
        s = Hp.std_ewald(Hp.electrolyte_small())
    elif which == "std_surf":
        s = Hp.std_ewald(Hp.electrolyte_small(lsurf=True))
    elif which == "std_bonds":
        s = Hp.std_ewald(Hp.pe_small())
    else:
        s = dict(Hp.electrolyte_small())
        s["lewald"] = False
    o, u = _mc_system(s)
    beta = 1.0 / S.kT(s["temp"])
    acc, hs = o.mc_pass(3, [2.0] * s["npt"], beta, u, isamp=1)
    n = 3 * s["np"]
    assert 0.1 * n < acc < 0.95 * n
    o.set_vlist()                       # the moves went past the list's skin
    fresh = o.utotal()
    scale = abs(fresh["utwob"][0]) + abs(fresh["urec"]) + abs(fresh["ubond"]) + 1.0
    for k in ("utot", "urec", "ubond"):
        assert abs(u[k] - fresh[k]) <= 1e-9 * scale, (k, u[k], fresh[k])
    assert np.abs(np.asarray(u["utwob"]) - np.asarray(fresh["utwob"])).max() <= 1e-9 * scale


def test_mc_spme_sweep_moves_and_keeps_the_mesh_energy():
    """The oracle's SPME chain (the mesh re-transformed per trial) accepts moves and its
    carried u%rec equals a fresh UTotal's."""
    s = dict(Hp.electrolyte_small())
    o, u = _mc_system(s)
    acc, _ = o.mc_pass(1, [1.0] * s["npt"], 1.0, u)
    assert acc > 0
    o.set_vlist()
    assert abs(u["urec"] - o.utotal()["urec"]) <= 1e-9 * (abs(u["urec"]) + 1.0)


# ---------------------------------------------------------------- chain moves (oracle)

def _pe_oracle(ewald):
    s = dict(Hp.pe_small())
    if ewald == "std":
        s = Hp.std_ewald(s)
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    return s, o, o.utotal()


_CHAINS = [(0, 50), (50, 50), (100, 50), (150, 50)]


def test_mc_moves_with_single_particle_moves_only_is_mcpass():
    """With pspart = 1 for every type the move-selecting pass is MCPass: the same chain."""
    s, o1, u1 = _pe_oracle("std")
    _, o2, u2 = _pe_oracle("std")
    beta = 1.0 / S.kT(s["temp"])
    o1.mc_seed(3)
    o2.mc_seed(3)
    a1 = o1.mc_pass(2, [2.0, 2.0], beta, u1)
    a2 = o2.mc_pass_moves(2, [2.0, 2.0], beta, u2, [1.0, 1.0], [1.0, 1.0], [5.0, 5.0], _CHAINS)
    assert a1 == a2
    assert np.array_equal(o1.get_state()["ro"], o2.get_state()["ro"])
    assert abs(u1["utot"] - u2["utot"]) <= 1e-12 * abs(u1["utot"])


@pytest.mark.parametrize("ewald", ["std", "spme"])
def test_mc_chain_moves_keep_chains_rigid_and_energies_carried(ewald):
    """Beads make only chain moves (pspart 0, pchain 1), counterions only single-particle moves:
    the bonds keep their lengths (whole chains translate) and the carried energies equal a fresh
    UTotal."""
    s, o, u = _pe_oracle(ewald)
    beta = 1.0 / S.kT(s["temp"])
    bij = np.asarray(s["bond_ij"]) - 1

    def lengths(ro):
        d = ro[bij[:, 0]] - ro[bij[:, 1]]
        d -= s["boxlen"][0] * np.round(d / s["boxlen"][0])
        return np.sqrt((d * d).sum(1))

    l0 = lengths(o.get_state()["ro"])
    o.mc_seed(5)
    acc, _ = o.mc_pass_moves(2, [2.0, 2.0], beta, u, [0.0, 1.0], [1.0, 1.0], [3.0, 3.0], _CHAINS)
    assert acc > 0
    assert np.abs(lengths(o.get_state()["ro"]) - l0).max() < 1e-11
    o.set_vlist()
    fresh = o.utotal()
    sc = abs(fresh["utwob"][0]) + abs(fresh["urec"]) + abs(fresh["ubond"]) + 1.0
    for k in ("utot", "urec", "ubond"):
        assert abs(u[k] - fresh[k]) <= 1e-9 * sc, (k, u[k], fresh[k])


def test_mc_chain_move_of_a_particle_in_no_chain_is_refused():
    s, o, u = _pe_oracle("std")
    with pytest.raises(RuntimeError):
        o.mc_pass_moves(1, [2.0, 2.0], 1.0, u, [0.0, 0.0], [1.0, 1.0], [3.0, 3.0], _CHAINS)
