"""MCAllPass (Src/mc.F90:4024-4178): every particle displaced at once, one UTotal of the
trial, Metropolis on du%tot, on the GPU (msg_mcall_pass) against the oracle.

The device draws each particle's five Random numbers (Src/mollib.F90:2689-2708) from its
place in the chain's stream by jumping the generator ahead (msg_random_jump); the jump is
checked here against the sequential stream.  GPU bars: the same acceptances as the
oracle, positions within 1e-12 (both wrap the same sums), energies within 1e-9 of the
energy scale."""
import ctypes as C

import numpy as np
import pytest

import helpers as Hp
import pyoracle as O
from molsim_b200 import Engine, _lib
from molsim_b200 import systems as S


def _jump(state, k):
    out = (C.c_int32 * 2)()
    assert _lib.lib().msg_random_jump(int(state[0]), int(state[1]), int(k), out) == 0
    return int(out[0]), int(out[1])


def test_random_jump_equals_the_sequential_stream():
    """msg_random_jump(k) followed by one draw gives the (k+1)-th draw of the stream."""
    st = (C.c_int32 * 2)()
    O.lib().or_random_init(12345, st)
    s0 = (int(st[0]), int(st[1]))
    seq = O.random_stream(12345, 5000)
    for k in (0, 1, 2, 5, 17, 999, 4096, 4999):
        j = _jump(s0, k)
        t = (C.c_int32 * 2)(j[0], j[1])
        r = O.lib().or_random_next(t)
        assert r == seq[k], k
    assert _lib.lib().msg_random_jump(1, 0, 3, (C.c_int32 * 2)()) == 6


def test_oracle_carried_energy_equals_fresh_utotal():
    s = dict(Hp.electrolyte_small(lsurf=True))
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    u = o.utotal()
    o.mc_seed(9)
    acc = o.mcall_pass(6, [0.3] * s["npt"], 1.0 / S.kT(s["temp"]), u)
    assert 0 < acc < 6
    o.set_vlist()
    fresh = o.utotal()
    assert abs(u["utot"] - fresh["utot"]) <= 1e-12 * abs(fresh["utot"])


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["std", "spme", "polyelectrolyte"])
def test_gpu_chain_matches_oracle(which):
    s = {"std": lambda: Hp.std_ewald(Hp.electrolyte_small(lsurf=True)),
         "spme": lambda: dict(Hp.electrolyte_small()),
         "polyelectrolyte": lambda: dict(Hp.pe_small())}[which]()
    t = Hp.oracle_table(s)
    beta = 1.0 / S.kT(s["temp"])
    dt = [0.3] * s["npt"]
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    u = o.utotal()
    o.mc_seed(4)
    acc = o.mcall_pass(8, dt, beta, u)
    g = Engine(s, t, precision="fp64")
    g.mc_seed(4)
    ag, eg = g.MCAllPass(8, dt, beta)
    assert int(ag[0]) == acc
    d = g.get_state()["ro"] - o.get_state()["ro"]
    box = np.asarray(s["boxlen"])
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-12
    sc = abs(u["utwob"][0]) + abs(u["urec"]) + abs(u["ubond"]) + 1.0
    for k in ("utot", "urec", "ubond"):
        assert abs(eg[k] - u[k]) <= 1e-9 * sc, (k, eg[k], u[k])


@pytest.mark.gpu
def test_gpu_systems_in_one_handle_run_their_own_chains():
    a = dict(Hp.electrolyte_small())
    b = Hp.std_ewald(Hp.electrolyte_small(n_pairs=50, L=36.0, seed=4))
    ta, tb = Hp.oracle_table(a), Hp.oracle_table(b)
    both = Engine([a, b], [ta, tb], precision="fp64")
    for k in range(2):
        both.mc_seed(40 + k, isys=k)
    acc, _ = both.MCAllPass(5, [[0.3] * a["npt"], [0.3] * b["npt"]])
    for k, (s, t) in enumerate(((a, ta), (b, tb))):
        one = Engine(s, t, precision="fp64")
        one.mc_seed(40 + k)
        a1, _ = one.MCAllPass(5, [0.3] * s["npt"])
        assert int(a1[0]) == int(acc[k])
        assert np.array_equal(one.get_state()["ro"], both.get_state(k)["ro"])


@pytest.mark.gpu
def test_gpu_mixed_handle_makes_the_same_decisions():
    """The mixed-precision handle (FP32 pair terms over the fixed-point position mirror, which
    the trial and the restore keep current) accepts the trials the FP64 handle accepts and
    ends at the same positions; with the list kept across trials by the skin test."""
    s = dict(Hp.electrolyte_small(lsurf=True))
    t = Hp.oracle_table(s)
    out = []
    for prec in ("fp64", "mixed"):
        g = Engine(s, t, precision=prec)
        g.mc_seed(21)
        acc, e = g.MCAllPass(10, [0.3] * s["npt"])
        out.append((int(acc[0]), g.get_state()["ro"], e["utot"], g.UTotal()["utot"]))
    assert out[0][0] == out[1][0] and 0 < out[0][0] < 10
    assert np.array_equal(out[0][1], out[1][1])
    for a in out:
        assert abs(a[2] - a[3]) <= 1e-9 * abs(a[3])      # carried = fresh UTotal
    assert abs(out[0][2] - out[1][2]) <= 1e-6 * abs(out[0][2])


def test_entry_point_refuses_bad_arguments_on_the_host():
    """No handle, or no per-system parameters: MSG_ERR_ARG before any device work."""
    lib = _lib.lib()
    par = (_lib.MsgMcAllParams * 1)()
    assert lib.msg_mcall_pass(None, 1, par, None, 0, None) == 6
    assert lib.msg_mcall_pass(None, 1, None, None, 0, None) == 6


def test_random_jump_composes():
    """Jumping k1 then k2 draws equals jumping k1 + k2, jumping 0 changes nothing, and a jump
    across 2^31 draws stays consistent (the Park-Miller part has period 2^31 - 2)."""
    rng = np.random.default_rng(5)
    st = (C.c_int32 * 2)()
    O.lib().or_random_init(-77, st)
    s0 = (int(st[0]), int(st[1]))
    assert _jump(s0, 0) == s0
    for _ in range(50):
        k1, k2 = (int(x) for x in rng.integers(0, 2 ** 31, 2))
        assert _jump(_jump(s0, k1), k2) == _jump(_jump(s0, k2), k1)
        if k1 + k2 < 2 ** 32:
            assert _jump(_jump(s0, k1), k2) == _jump(s0, k1 + k2)
    # the Park-Miller part returns after its period 2^31 - 2
    assert _jump(s0, 2 ** 31 - 2)[1] == s0[1]
