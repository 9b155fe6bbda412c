"""Polyatomic particles: UTwoBodyP (Src/energy.F90:786-896), the site-site pair energy,
forces and virial over the particle list, on the GPU (msg_utwobody_p) against the oracle.

The oracle's restatement is pinned by the monoatomic limit (one site per particle: the
same pairs, table and sums as UTwoBodyA) and by Newton's third law on rigid molecules.
GPU bars: forces within 1e-10 relative RMS, energies and virial within 1e-10 relative
(64-bit fixed-point sums at 2^-40 of the unit)."""
import numpy as np
import pytest

import helpers as Hp
import pyoracle as O
from molsim_b200 import systems as S


def _monoatomic_as_polyatomic(s, o):
    """A monoatomic system written as polyatomic particles of one site each."""
    nn, jp = o.get_vlist()
    n = s["np"]
    return dict(np=n, na=n, npt=s["npt"], nat=s["npt"], boxlen=s["boxlen"], rcut=s["rcut"], ro=s["ro"], r=s["ro"],
                iptpn=s["iptpn"], ianpn=np.arange(1, n + 1, dtype=np.int32),
                napt=np.ones(s["npt"], np.int32), iatan=s["iptpn"], nneighpn=nn, jpnlist=jp)


def test_monoatomic_limit_equals_utwobody_a():
    s = dict(Hp.electrolyte_small())
    s["lewald"] = False
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    ref = o.utotal()
    p = O.utwobody_p(_monoatomic_as_polyatomic(s, o), t)
    assert Hp.rel_rms(p["force"], ref["force"]) < 1e-13
    assert np.abs(p["utwob"] - ref["utwob"]).max() <= 1e-12 * np.abs(ref["utwob"]).max()
    assert abs(p["virial"] - ref["virial"]) <= 1e-12 * abs(ref["virial"])


def test_rigid_molecules_newton_third_law():
    s = Hp.rigid_small()
    p = O.utwobody_p(s, Hp.site_table(s))
    f = p["force"]
    assert np.abs(f.sum(0)).max() <= 1e-10 * np.abs(f).max()
    assert p["utwob"][0] == pytest.approx(p["utwob"][1:].sum(), rel=1e-14)
    assert np.abs(f).max() > 0.0 and p["utwob"][0] != 0.0


def test_entry_point_rejects_bad_indices_on_the_host():
    s = dict(Hp.rigid_small())
    t = Hp.site_table(s)
    jp = np.array(s["jpnlist"], np.int32)
    i = int(np.argmax(s["nneighpn"]))
    jp[i, 0] = s["np"] + 1                   # a partner past the last particle
    bad = dict(s)
    bad["jpnlist"] = jp
    from molsim_b200.polyatomic import utwobody_p
    from molsim_b200.engine import MolsimGpuError
    with pytest.raises(MolsimGpuError) as ei:
        utwobody_p(bad, t)
    assert ei.value.code == 6


@pytest.mark.gpu
def test_gpu_matches_oracle():
    from molsim_b200.polyatomic import utwobody_p

    s = Hp.rigid_small()
    t = Hp.site_table(s)
    ref = O.utwobody_p(s, t)
    got = utwobody_p(s, t)
    assert Hp.rel_rms(got["force"], ref["force"]) < 1e-10
    assert np.abs(got["utwob"] - ref["utwob"]).max() <= 1e-10 * np.abs(ref["utwob"]).max()
    assert abs(got["virial"] - ref["virial"]) <= 1e-10 * abs(ref["virial"])
    # deterministic: the fixed-point sums repeat bit for bit
    again = utwobody_p(s, t)
    assert np.array_equal(again["force"], got["force"]) and np.array_equal(again["utwob"], got["utwob"])


@pytest.mark.gpu
def test_gpu_monoatomic_limit_matches_the_handle():
    """One site per particle: msg_utwobody_p gives the FP64 handle's pair energy."""
    from molsim_b200 import Engine
    from molsim_b200.polyatomic import utwobody_p

    s = dict(Hp.electrolyte_small())
    s["lewald"] = False
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    got = utwobody_p(_monoatomic_as_polyatomic(s, o), t)
    g = Engine(s, t, precision="fp64").UTotal()
    assert Hp.rel_rms(got["force"], g["force"]) < 1e-10
    # the handle rounds each particle's pair energy to 2^-32 before it sums: 1e-9 here
    assert abs(got["utwob"][0] - g["utwob"][0]) <= 1e-9 * abs(g["utwob"][0])


@pytest.mark.gpu
def test_site_below_the_table_is_an_error():
    from molsim_b200.engine import MolsimGpuError
    from molsim_b200.polyatomic import utwobody_p

    s = dict(Hp.rigid_small())
    t = Hp.site_table(s)
    r = np.array(s["r"])
    ro = np.array(s["ro"])
    # put the first solute 0.1 A from the first molecule's centre site
    k = int(np.where(np.asarray(s["iptpn"]) == 2)[0][0])
    ro[k] = r[0] + np.array([0.1, 0.0, 0.0])
    r[int(s["ianpn"][k]) - 1] = ro[k]
    bad = dict(s)
    bad["ro"], bad["r"] = ro, r
    bad["nneighpn"], bad["jpnlist"] = S.particle_list(ro, s["boxlen"][0], s["rcut"] + s["drnlist"])
    with pytest.raises(MolsimGpuError) as ei:
        utwobody_p(bad, t)
    assert ei.value.code == 1


# ---------------------------------------------------------------- rigid-body dynamics

def _rigid():
    return S.rigid_bodies(seed=1, nmol=200, nsolute=60, L=30.0, rcut=9.0, drnlist=2.5, tstep=0.001)


def _energies(s, u):
    """Total energy (kJ/mol): pair energy + centre-of-mass and rotational kinetic energy,
    the angular velocity from QuaVelToAngVel in the principal frame."""
    ipt = np.asarray(s["iptpn"]) - 1
    m = s["masspt"][ipt]
    ket = 0.5 * (m[:, None] * s["rod"] ** 2).sum() * 0.01     # g/mol (A/ps)^2 -> kJ/mol
    q, qd = s["qua"], s["quad"]
    w = np.stack([2 * (-q[:, 3] * qd[:, 2] + q[:, 0] * qd[:, 1] + q[:, 2] * qd[:, 3] - q[:, 1] * qd[:, 0]),
                  2 * (-q[:, 0] * qd[:, 2] - q[:, 3] * qd[:, 1] + q[:, 1] * qd[:, 3] + q[:, 2] * qd[:, 0]),
                  2 * (+q[:, 1] * qd[:, 2] - q[:, 2] * qd[:, 1] + q[:, 0] * qd[:, 3] - q[:, 3] * qd[:, 0])], 1)
    ker = 0.5 * (s["momp"][ipt] * w ** 2)[ipt == 0].sum() * 0.01
    return u["utwob"][0] + ket + ker, ket, ker


def test_rigid_body_oracle_conserves_energy_and_shape():
    """The oracle's VelVer for rigid bodies (quaternions, torques, GetAngAcc with nvvite
    iterations): over 200 steps of 1 fs the total energy moves by under 2 % of the kinetic
    energy's fluctuation while rotation picks up tens of kJ/mol, and the molecules stay rigid."""
    s = _rigid()
    t = Hp.site_table(s)
    E = [_energies(s, O.velver_p(s, t, 1))]
    for _ in range(40):
        E.append(_energies(s, O.velver_p(s, t, 5)))
    E = np.array(E)
    assert E[-1, 2] > 10.0                                  # the molecules rotate
    assert abs(E[-1, 0] - E[0, 0]) < 0.02 * E[:, 1].std()
    r = np.asarray(s["r"])
    for k in range(0, 600, 3):
        assert abs(np.linalg.norm(r[k] - r[k + 1]) - 1.0) < 1e-12
        assert abs(np.linalg.norm(r[k] - r[k + 2]) - 1.0) < 1e-12


@pytest.mark.gpu
def test_rigid_body_steps_match_oracle():
    """Ten rigid-body steps on the GPU against the oracle from the same state: centres,
    velocities, quaternions and their velocities within 1e-8 (the site forces are summed
    in fixed point, so the trajectories part at rounding level), energies and virial
    within 1e-8 relative."""
    import copy

    from molsim_b200.polyatomic import velver_p

    s = _rigid()
    t = Hp.site_table(s)
    so, sg = copy.deepcopy(s), copy.deepcopy(s)
    uo = O.velver_p(so, t, 10)
    ug = velver_p(sg, t, 10)
    box = s["boxlen"][0]
    d = np.asarray(sg["ro"]) - np.asarray(so["ro"])
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-8
    for key in ("rod", "qua", "quad"):
        assert np.abs(np.asarray(sg[key]) - np.asarray(so[key])).max() <= 1e-8 * max(1.0, np.abs(so[key]).max()), key
    assert np.abs(ug["utwob"] - uo["utwob"]).max() <= 1e-8 * np.abs(uo["utwob"]).max()
    assert abs(ug["virial"] - uo["virial"]) <= 1e-8 * abs(uo["virial"])
    assert np.abs(np.asarray(sg["quad"])).max() > 0.0          # the bodies turn
