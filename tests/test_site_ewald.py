"""UEwald over the sites of polyatomic particles (Src/energy.F90:905-958): the standard
reciprocal sum over sites (UEwaldRecStd, :964-1104), UEwaldSelf's atomic and molecular
terms (:1301-1345) and UEwaldSurf (:1349-1371), on the GPU (msg_uewald_sites) against
the oracle.

The oracle's restatement is pinned two ways: in the monoatomic limit (one site per
particle, no intramolecular pairs) its u%rec and forces are those of the monoatomic
UTotal with standard Ewald; on rigid three-site molecules the Ewald total (the
erfc-screened site pairs of UTwoBodyP plus the site sum) does not depend on alpha.
GPU bars: u%rec within 1e-10 of the self-energy scale EpsiFourPi alpha/sqrt(pi) sum q^2
(u%rec is a small difference of terms that size), its virial within 1e-10 relative,
forces within 1e-10 relative RMS (64-bit fixed-point energy sums, structure factors
summed in a fixed order)."""
import numpy as np
import pytest

import helpers as Hp
import pyoracle as O
from molsim_b200 import systems as S


def _monoatomic_as_polyatomic(s, o):
    nn, jp = o.get_vlist()
    n = s["np"]
    return dict(np=n, na=n, npt=s["npt"], nat=s["npt"], boxlen=s["boxlen"], rcut=s["rcut"], ro=s["ro"], r=s["ro"],
                iptpn=s["iptpn"], ianpn=np.arange(1, n + 1, dtype=np.int32), napt=np.ones(s["npt"], np.int32),
                iatan=s["iptpn"], nneighpn=nn, jpnlist=jp, epsi_four_pi=s["epsi_four_pi"])


def _site_charges(s):
    return np.asarray(s["zat"], np.float64)[np.asarray(s["iatan"]) - 1]


def _screened_site_table(s, alpha, tol):
    """The atom-type table of a rigid_molecules system with erfc(alpha r)/r screening."""
    d = S.site_table_params(s)
    pot = dict(npt=d["npt"], zat=d["zat"], sigat=d["sigat"], epsat=d["epsat"], rcut=d["rcut"], ualpha=alpha,
               epsi_four_pi=d["epsi_four_pi"], lewald=1, lljcut=int(d["lljcut"]), utoltab=tol, ftoltab=tol,
               **{k: d[k] for k in ("ljrcut", "ljushift", "r2uminin", "umaxtab", "fmaxtab", "rumaxfac")})
    return O.pot_tab(pot)


def _self_scale(s, az, alpha):
    return s["epsi_four_pi"] * alpha / np.sqrt(np.pi) * float(np.sum(np.asarray(az) ** 2))


def _molecules():
    return S.rigid_molecules(seed=3, nmol=120, nsolute=0, L=24.0, rcut=11.0)


@pytest.mark.parametrize("lsurf", [False, True])
def test_monoatomic_limit_equals_utotal_std(lsurf):
    s = Hp.std_ewald(Hp.electrolyte_small(lsurf=lsurf), ncut=8)
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    ref = o.utotal()
    p = _monoatomic_as_polyatomic(s, o)
    pair = O.utwobody_p(p, t)
    e = O.uewald_sites(p, s["az"], t["ualpha"], t["ncut"], lsurf=lsurf)
    assert e["urec"] == pytest.approx(ref["urec"], rel=1e-14, abs=1e-12)
    assert Hp.rel_rms(pair["force"] + e["force"], ref["force"]) < 1e-13


def test_ewald_total_is_independent_of_alpha():
    """Site pairs screened with erfc(alpha r)/r (table tolerance 1e-7) plus the site Ewald sum:
    the total energy of 120 rigid three-site molecules agrees across alpha within 1e-3 kJ/mol
    (about 5e-6 relative; without the molecular self term it would move by hundreds of kJ/mol),
    the forces within 1e-3 of their largest, and the net force vanishes."""
    s = _molecules()
    az = _site_charges(s)
    assert abs(az.sum()) < 1e-12
    tot, forces = [], []
    for alpha, ncut in ((0.35, 16), (0.45, 20)):
        pair = O.utwobody_p(s, _screened_site_table(s, alpha, 1e-7))
        e = O.uewald_sites(s, az, alpha, ncut)
        f = pair["force"] + e["force"]
        assert np.abs(f.sum(0)).max() <= 1e-10 * np.abs(f).max()
        tot.append(pair["utwob"][0] + e["urec"])
        forces.append(f)
    assert abs(tot[0] - tot[1]) < 1e-3, tot
    assert np.abs(forces[0] - forces[1]).max() < 1e-3 * np.abs(forces[0]).max()


def test_bad_arguments_are_refused_on_the_host():
    from molsim_b200.engine import MolsimGpuError
    from molsim_b200.polyatomic import uewald_sites

    s = dict(_molecules())
    az = _site_charges(s)
    with pytest.raises(MolsimGpuError) as ei:
        uewald_sites(s, az, 0.35, 0)
    assert ei.value.code == 6
    with pytest.raises(MolsimGpuError) as ei:
        uewald_sites(s, az, 0.35, 101)
    assert ei.value.code == 6
    ian = np.array(s["ianpn"], np.int32)
    ian[-1] = s["na"]                        # the last particle's sites run past na
    bad = dict(s)
    bad["ianpn"] = ian
    with pytest.raises(MolsimGpuError) as ei:
        uewald_sites(bad, az, 0.35, 8)
    assert ei.value.code == 6
    with pytest.raises(ValueError):
        uewald_sites(s, az[:-1], 0.35, 8)


@pytest.mark.gpu
@pytest.mark.parametrize("region,lsurf", [("sphere", False), ("cube", True)])
def test_gpu_matches_oracle(region, lsurf):
    from molsim_b200.polyatomic import uewald_sites

    s = _molecules()
    az = _site_charges(s)
    ref = O.uewald_sites(s, az, 0.35, 12, region=region, lsurf=lsurf)
    got = uewald_sites(s, az, 0.35, 12, region=region, lsurf=lsurf)
    assert abs(got["urec"] - ref["urec"]) <= 1e-10 * _self_scale(s, az, 0.35)
    assert got["virrec"] == pytest.approx(ref["virrec"], rel=1e-10)
    assert Hp.rel_rms(got["force"], ref["force"]) < 1e-10
    again = uewald_sites(s, az, 0.35, 12, region=region, lsurf=lsurf)
    assert again["urec"] == got["urec"] and np.array_equal(again["force"], got["force"])


@pytest.mark.gpu
def test_gpu_monoatomic_limit_matches_the_handle():
    """One site per particle: the GPU site sum plus the GPU site pairs give the FP64
    handle's UTotal with standard Ewald."""
    from molsim_b200 import Engine
    from molsim_b200.polyatomic import uewald_sites, utwobody_p

    s = Hp.std_ewald(Hp.electrolyte_small(lsurf=True), ncut=8)
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    p = _monoatomic_as_polyatomic(s, o)
    pair = utwobody_p(p, t)
    e = uewald_sites(p, s["az"], t["ualpha"], t["ncut"], lsurf=True)
    g = Engine(s, t, precision="fp64").UTotal()
    assert abs(e["urec"] - g["urec"]) <= 1e-10 * _self_scale(s, s["az"], t["ualpha"])
    assert Hp.rel_rms(pair["force"] + e["force"], g["force"]) < 1e-10


@pytest.mark.gpu
def test_gpu_large_system_net_force_and_alpha():
    """4000 molecules (12000 sites, several site chunks of the structure-factor sum): the
    net force is zero and the GPU's Ewald total agrees across alpha as the oracle's does."""
    from molsim_b200.polyatomic import uewald_sites, utwobody_p

    s = S.rigid_molecules(seed=5, nmol=4000, nsolute=0, L=75.0, rcut=11.0)
    az = _site_charges(s)
    tot = []
    for alpha, ncut in ((0.35, 40), (0.45, 52)):
        pair = utwobody_p(s, _screened_site_table(s, alpha, 1e-7))
        e = uewald_sites(s, az, alpha, ncut)
        f = pair["force"] + e["force"]
        assert np.abs(f.sum(0)).max() <= 1e-9 * np.abs(f).max()
        tot.append(pair["utwob"][0] + e["urec"])
    assert abs(tot[0] - tot[1]) <= 5e-6 * abs(tot[0]), tot


# ------------------------------------------------- rigid-body dynamics with site Ewald

def _rigid_charged():
    return S.rigid_bodies(seed=1, nmol=200, nsolute=60, L=30.0, rcut=9.0, drnlist=2.5, tstep=0.001)


def _rigid_ewald(s, alpha=0.35, ncut=14, lsurf=False):
    return dict(az=_site_charges(s), ualpha=alpha, ncut=ncut, lsurf=lsurf)


def _total_energy(s, u):
    """Pair + reciprocal + centre-of-mass and rotational kinetic energy (kJ/mol)."""
    ipt = np.asarray(s["iptpn"]) - 1
    m = s["masspt"][ipt]
    ket = 0.5 * (m[:, None] * s["rod"] ** 2).sum() * 0.01
    q, qd = s["qua"], s["quad"]
    w = np.stack([2 * (-q[:, 3] * qd[:, 2] + q[:, 0] * qd[:, 1] + q[:, 2] * qd[:, 3] - q[:, 1] * qd[:, 0]),
                  2 * (-q[:, 0] * qd[:, 2] - q[:, 3] * qd[:, 1] + q[:, 1] * qd[:, 3] + q[:, 2] * qd[:, 0]),
                  2 * (+q[:, 1] * qd[:, 2] - q[:, 2] * qd[:, 1] + q[:, 0] * qd[:, 3] - q[:, 3] * qd[:, 0])], 1)
    ker = 0.5 * (s["momp"][ipt] * w ** 2)[ipt == 0].sum() * 0.01
    return u["utwob"][0] + u["urec"] + ket + ker, ket


def test_rigid_body_ewald_oracle_conserves_energy():
    """The oracle's rigid-body step with the site Ewald sum (erfc-screened site table) conserves
    energy as well as the same system with a plainly truncated site table does: over 200 steps
    of 1 fs the total energy, u%rec included, fluctuates by under twice the plain run's
    fluctuation (both about 2 % of the kinetic energy's: the 1 fs step and the particle list
    held fixed set that level), and u%rec changes as the molecules turn."""
    import helpers

    def run(ewald):
        s = _rigid_charged()
        t = _screened_site_table(s, 0.35, 1e-7) if ewald else helpers.site_table(s)
        ew = _rigid_ewald(s) if ewald else None
        E, ur = [], []
        for k in range(41):
            u = O.velver_p(s, t, 1 if k == 0 else 5, ewald=ew)
            u.setdefault("urec", 0.0)
            E.append(_total_energy(s, u))
            ur.append(u["urec"])
        return np.array(E), np.array(ur)

    Ee, ur = run(True)
    Ep, _ = run(False)
    assert Ee[:, 0].std() < 2.0 * Ep[:, 0].std(), (Ee[:, 0].std(), Ep[:, 0].std())
    assert Ee[:, 0].std() < 0.05 * Ee[:, 1].std()
    assert np.ptp(ur) > 10.0 * Ee[:, 0].std()


def test_forces_are_the_energy_gradient():
    """Central differences of u%rec (h = 1e-5 A) on sites of three molecules, surface term on:
    the Ewald forces, the molecular self term's included, are -grad u%rec within 1e-6 of the
    largest force."""
    s = dict(_molecules())
    az = _site_charges(s)
    ref = O.uewald_sites(s, az, 0.35, 12, lsurf=True)
    fmax = np.abs(ref["force"]).max()
    h = 1e-5
    r0 = np.array(s["r"], np.float64)
    for ia in (0, 1, 5, 100, 359):
        for c in range(3):
            up, dn = r0.copy(), r0.copy()
            up[ia, c] += h
            dn[ia, c] -= h
            eu = O.uewald_sites(dict(s, r=up), az, 0.35, 12, lsurf=True)["urec"]
            ed = O.uewald_sites(dict(s, r=dn), az, 0.35, 12, lsurf=True)["urec"]
            assert abs(-(eu - ed) / (2 * h) - ref["force"][ia, c]) < 1e-6 * fmax, (ia, c)


@pytest.mark.gpu
@pytest.mark.parametrize("lsurf", [False, True])
def test_gpu_rigid_body_ewald_steps_match_oracle(lsurf):
    """Ten rigid-body steps with the site Ewald sum on the GPU (msg_velver_p_ewald) against
    the oracle from the same state: centres, velocities, quaternions and their velocities
    within 1e-8, u%rec within 1e-10 of the self-energy scale, pair energies and virial within
    1e-8 relative."""
    import copy

    from molsim_b200.polyatomic import velver_p

    s = _rigid_charged()
    t = _screened_site_table(s, 0.35, 1e-7)
    ew = _rigid_ewald(s, lsurf=lsurf)
    so, sg = copy.deepcopy(s), copy.deepcopy(s)
    uo = O.velver_p(so, t, 10, ewald=ew)
    ug = velver_p(sg, t, 10, ewald=ew)
    box = s["boxlen"][0]
    d = np.asarray(sg["ro"]) - np.asarray(so["ro"])
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-8
    for key in ("rod", "qua", "quad"):
        assert np.abs(np.asarray(sg[key]) - np.asarray(so[key])).max() <= 1e-8 * max(1.0, np.abs(so[key]).max()), key
    assert abs(ug["urec"] - uo["urec"]) <= 1e-10 * _self_scale(s, ew["az"], 0.35)
    assert np.abs(ug["utwob"] - uo["utwob"]).max() <= 1e-8 * np.abs(uo["utwob"]).max()
    assert abs(ug["virial"] - uo["virial"]) <= 1e-8 * abs(uo["virial"])


# ------------------------------------------------------------------ SPME over the sites

@pytest.mark.parametrize("lsurf", [False, True])
def test_spm_monoatomic_limit_equals_utotal_spme(lsurf):
    """SPME over sites, one site per particle: u%rec and forces of the monoatomic UTotal with SPME."""
    s = Hp.electrolyte_small(lsurf=lsurf)
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    ref = o.utotal()
    p = _monoatomic_as_polyatomic(s, o)
    pair = O.utwobody_p(p, t)
    e = O.uewald_sites(p, s["az"], t["ualpha"], order=s["order"], nmesh=s["nmesh"], lsurf=lsurf)
    assert e["urec"] == pytest.approx(ref["urec"], rel=1e-14, abs=1e-12)
    assert Hp.rel_rms(pair["force"] + e["force"], ref["force"]) < 1e-13


def test_spm_converges_to_the_standard_sum():
    """On rigid molecules, SPME over the sites approaches the standard Ewald sum as the mesh
    refines: order 8 on a 64^3 mesh agrees within 1e-6 of the self-energy scale in u%rec and
    1e-6 of the largest force."""
    s = _molecules()
    az = _site_charges(s)
    std = O.uewald_sites(s, az, 0.35, 16)
    spm = O.uewald_sites(s, az, 0.35, order=8, nmesh=64)
    assert abs(spm["urec"] - std["urec"]) < 1e-6 * _self_scale(s, az, 0.35)
    assert np.abs(spm["force"] - std["force"]).max() < 1e-6 * np.abs(std["force"]).max()


def test_spm_bad_arguments_are_refused_on_the_host():
    from molsim_b200.engine import MolsimGpuError
    from molsim_b200.polyatomic import uewald_sites

    s = _molecules()
    az = _site_charges(s)
    for order, nmesh in ((3, 32), (9, 32), (5, 33), (5, 6)):
        with pytest.raises(MolsimGpuError) as ei:
            uewald_sites(s, az, 0.35, order=order, nmesh=nmesh)
        assert ei.value.code == 6


@pytest.mark.gpu
@pytest.mark.parametrize("order,nmesh,lsurf", [(5, 32, False), (6, 40, True), (8, 64, False)])
def test_gpu_spm_matches_oracle(order, nmesh, lsurf):
    from molsim_b200.polyatomic import uewald_sites

    s = _molecules()
    az = _site_charges(s)
    ref = O.uewald_sites(s, az, 0.35, order=order, nmesh=nmesh, lsurf=lsurf)
    got = uewald_sites(s, az, 0.35, order=order, nmesh=nmesh, lsurf=lsurf)
    # the mesh sums of u%rec and its virial (weights of both signs over the spectrum, a cuFFT
    # transform against the oracle's) are held to the self-energy scale
    assert abs(got["urec"] - ref["urec"]) <= 1e-10 * _self_scale(s, az, 0.35)
    assert abs(got["virrec"] - ref["virrec"]) <= 1e-10 * _self_scale(s, az, 0.35)
    assert Hp.rel_rms(got["force"], ref["force"]) < 1e-10
    again = uewald_sites(s, az, 0.35, order=order, nmesh=nmesh, lsurf=lsurf)
    assert again["urec"] == got["urec"] and np.array_equal(again["force"], got["force"])


@pytest.mark.gpu
def test_gpu_rigid_body_spm_steps_match_oracle():
    """Ten rigid-body steps with SPME over the sites (order 5, 32^3) on the GPU against the oracle."""
    import copy

    from molsim_b200.polyatomic import velver_p

    s = _rigid_charged()
    t = _screened_site_table(s, 0.35, 1e-7)
    ew = dict(az=_site_charges(s), ualpha=0.35, order=5, nmesh=32, lsurf=True)
    so, sg = copy.deepcopy(s), copy.deepcopy(s)
    uo = O.velver_p(so, t, 10, ewald=ew)
    ug = velver_p(sg, t, 10, ewald=ew)
    box = s["boxlen"][0]
    d = np.asarray(sg["ro"]) - np.asarray(so["ro"])
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-8
    for key in ("rod", "qua", "quad"):
        assert np.abs(np.asarray(sg[key]) - np.asarray(so[key])).max() <= 1e-8 * max(1.0, np.abs(so[key]).max()), key
    assert abs(ug["urec"] - uo["urec"]) <= 1e-10 * _self_scale(s, ew["az"], 0.35)
    assert abs(ug["virial"] - uo["virial"]) <= 1e-8 * abs(uo["virial"])


def test_rigid_body_ewald_arguments_are_refused_on_the_host():
    """msg_velver_p_ewald checks its site Ewald parameters before touching the device: an
    unknown method, ncut outside 1..100, an SPME order outside 4..8 or an odd mesh."""
    from molsim_b200.engine import MolsimGpuError
    from molsim_b200.polyatomic import velver_p

    s = _rigid_charged()
    t = Hp.site_table(s)
    az = _site_charges(s)
    for ew in (dict(az=az, ualpha=0.35, ncut=0), dict(az=az, ualpha=0.35, ncut=101),
               dict(az=az, ualpha=0.35, order=3, nmesh=32), dict(az=az, ualpha=0.35, order=5, nmesh=33),
               dict(az=az, ualpha=-1.0, ncut=8)):
        with pytest.raises(MolsimGpuError) as ei:
            velver_p(dict(s), t, 1, ewald=ew)
        assert ei.value.code == 6, ew
    with pytest.raises(ValueError):
        velver_p(dict(s), t, 1, ewald=dict(az=az[:-1], ualpha=0.35, ncut=8))
