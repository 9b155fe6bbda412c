"""GPU parity of the FP64 drop-in path against the FP64 oracle, through the C-ABI.

Bars (from the task's correctness contract):
  * neighbour-pair set bit-exact (MOLSIM layout: nneighpn and sorted jpnlist rows);
  * forces within 1e-5 relative RMS (the FP64 path lands near 1e-12);
  * total energy, its terms and the virial within 1e-7 relative.
"""
import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine
from molsim_b200 import systems as S

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
ENERGY_TOL = 1e-7


def _pair(s, **kw):
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t, cell=s["np"] > 20000)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    g = Engine(s, t, **kw)
    return t, o, g


def _check_nlist(o, g, n):
    nn_o, jp_o = o.get_vlist()
    nn_g, jp_g, npair = g.SetVList(0, export=True, maxnneigh=o.maxnneigh)
    assert npair == int(nn_o.sum())
    assert np.array_equal(nn_o, nn_g)
    for ip in range(n):
        k = nn_o[ip]
        assert np.array_equal(jp_o[ip, :k], jp_g[ip, :k]), ip


def _check_utotal(o, g, ftol=FORCE_TOL, etol=ENERGY_TOL):
    ro = o.utotal()
    rg = g.UTotal()
    assert Hp.rel_rms(rg["force"], ro["force"]) < ftol
    assert Hp.rel_rms(rg["forceo"], ro["forceo"]) < ftol
    for k in ("utot", "urec", "virial"):
        assert Hp.rel(rg[k], ro[k]) < etol, (k, rg[k], ro[k])
    for p, v in enumerate(ro["utwob"]):
        assert abs(rg["utwob"][p] - v) <= etol * max(abs(ro["utot"]), abs(v)), (p, rg["utwob"][p], v)
    # u%bond on the total-energy scale (a fresh chain sits at r0: u%bond ~ 0)
    assert abs(rg["ubond"] - ro["ubond"]) <= etol * max(abs(ro["ubond"]), abs(ro["utot"]))
    return ro, rg


@pytest.mark.parametrize("lsurf", [False, True])
def test_small_electrolyte_nlist_and_utotal(lsurf):
    s = dict(Hp.electrolyte_small(lsurf=lsurf))
    t, o, g = _pair(s)
    _check_nlist(o, g, s["np"])
    ro, rg = _check_utotal(o, g)
    assert Hp.rel_rms(rg["force"], ro["force"]) < 1e-10


def test_config0_electrolyte():
    s = Hp.config0()
    t, o, g = _pair(s)
    _check_nlist(o, g, s["np"])
    _check_utotal(o, g)


def test_config1_polyelectrolyte():
    s = Hp.config1()
    t, o, g = _pair(s)
    _check_nlist(o, g, s["np"])
    ro, rg = _check_utotal(o, g)
    assert ro["ubond"] > 0.0


def test_velver_short_trajectory():
    """Ten velocity-Verlet steps (with NList skin tests) against the oracle."""
    s = dict(Hp.pe_small())
    s["tstep"] = 0.01
    t, o, g = _pair(s)
    o.utotal()
    st = o.get_state()
    rodd = np.zeros_like(st["ro"])
    # GetLinAcc on both sides from the same forces
    g.UTotal()
    g.GetLinAcc()
    rodd = g.get_state()["rodd"]
    o.set_state(st["ro"], st["rod"], rodd)
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


def test_bd_with_injected_noise():
    """Brownian dynamics with the caller's noise (the drop-in mode): five steps."""
    s = dict(Hp.colloid_small())
    t, o, g = _pair(s)
    o.utotal()
    g.UTotal()
    rng = np.random.default_rng(7)
    xi = rng.standard_normal((5, s["np"], 3))
    fac1, fac2 = s["bd_fac"]
    eg = g.BDStep(5, xi=xi)
    for k in range(5):
        o.bd_step(xi[k], fac1, fac2)
    sg, so = g.get_state(), o.get_state()
    d = sg["ro"] - so["ro"]
    box = s["boxlen"][0]
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-9
    rg, ro = g.UTotal(), o.utotal()
    assert Hp.rel_rms(rg["force"], ro["force"]) < FORCE_TOL
    assert Hp.rel(eg[-1]["utot"], ro["utot"]) < ENERGY_TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_alone(precision):
    """Systems advanced together in one handle give the results they give alone, bit for
    bit in both precisions: the charge grid, the half-list partner forces and the energies
    are summed as 64-bit integers, and every other sum runs in a fixed order."""
    sys_list = [dict(Hp.electrolyte_small()), dict(Hp.pe_small())]
    sys_list[1]["order"] = 4
    tabs = [Hp.oracle_table(s) for s in sys_list]
    gb = Engine(sys_list, tabs, precision=precision)
    for k, (s, t) in enumerate(zip(sys_list, tabs)):
        ga = Engine(s, t, precision=precision)
        ra, rb = ga.UTotal(), gb.UTotal(k)
        assert np.array_equal(rb["force"], ra["force"])
        assert rb["utot"] == ra["utot"] and rb["virial"] == ra["virial"] and rb["urec"] == ra["urec"]


def test_graph_replay_matches_direct_launches(monkeypatch):
    """The CUDA-graph step (rebuild in a conditional node) equals the directly launched step."""
    s = dict(Hp.pe_small())
    s["tstep"] = 0.02
    s["drnlist"] = 0.6
    t = Hp.oracle_table(s)
    ga = Engine(s, t)
    monkeypatch.setenv("MSG_NO_GRAPHS", "1")
    gb = Engine(s, t)
    monkeypatch.delenv("MSG_NO_GRAPHS")
    for g in (ga, gb):
        g.UTotal()
        g.GetLinAcc()
    ea, eb = ga.VelVer(40), gb.VelVer(40)
    assert ga.nrebuild() == gb.nrebuild() > 1
    for x, y in zip(ea, eb):
        assert Hp.rel(x["utot"], y["utot"]) < 1e-10
    sa, sb = ga.get_state(), gb.get_state()
    assert np.abs(sa["ro"] - sb["ro"]).max() < 1e-9


def test_rebuild_schedule_matches_oracle():
    """The skin test (with MOLSIM's running second maximum) triggers the same rebuilds."""
    s = dict(Hp.pe_small())
    s["tstep"] = 0.02
    s["drnlist"] = 0.6
    t, o, g = _pair(s)
    g.UTotal()
    g.GetLinAcc()
    st = g.get_state()
    o.set_state(st["ro"], st["rod"], st["rodd"])
    o.utotal()
    nb0 = g.nrebuild()
    for k in range(25):
        _, rb = o.velver_step()
        g.VelVer(1, energies=False)
        nb = g.nrebuild()
        assert (nb - nb0) == int(rb), k
        nb0 = nb


# ---------------------------------------------------------------------------
# Mixed precision: FP32 pair and grid forces, 64-bit fixed-point sums, FP64
# positions/integrator/energies.  Bars, the same as the FP64 path's: forces
# 1e-5 relative RMS against the FP64 oracle; u%tot, u%rec, the virial and
# every u%twob term 1e-7 relative (the pair energies and virial are FP64 sums of
# terms formed from the exact r2 and the table's FP64 leading coefficients; the
# reciprocal energy and virial come from an FP64 forward transform).
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("which", ["electrolyte_small", "config0", "config1", "pe_small"])
def test_mixed_precision_utotal(which):
    s = dict(getattr(Hp, which)())
    t, o, g = _pair(s, precision="mixed")
    _check_utotal(o, g)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_results_are_deterministic(precision):
    """Fixed-point force and grid sums: two runs give bitwise identical forces, energies
    and, after twenty MD steps with list rebuilds, positions."""
    s = dict(Hp.pe_small())
    s["tstep"] = 0.02
    t = Hp.oracle_table(s)
    out = []
    for _ in range(2):
        g = Engine(s, t, precision=precision)
        r = g.UTotal()
        g.GetLinAcc()
        e = g.VelVer(20)
        out.append((r, e, g.get_state(), g.nrebuild()))
    (a, ea, sa, na), (b, eb, sb, nb) = out
    assert na == nb and na > 1
    assert np.array_equal(a["force"], b["force"])
    assert a["utot"] == b["utot"] and a["urec"] == b["urec"] and a["virial"] == b["virial"]
    assert [x["utot"] for x in ea] == [x["utot"] for x in eb]
    for k in ("ro", "rod", "rodd"):
        assert np.array_equal(sa[k], sb[k]), k


def test_mixed_velver_tracks_fp64():
    s = dict(Hp.pe_small())
    t = Hp.oracle_table(s)
    gm, gd = Engine(s, t, precision="mixed"), Engine(s, t)
    for g in (gm, gd):
        g.UTotal()
        g.GetLinAcc()
    em, ed = gm.VelVer(20), gd.VelVer(20)
    for x, y in zip(em, ed):
        assert Hp.rel(x["utot"], y["utot"]) < 1e-5


@pytest.mark.parametrize("which", ["electrolyte_small", "config0", "config1"])
def test_half_list_export_and_forces(which):
    """The mixed path stores each pair once (half list, the parity rule on the internal
    order).  Its MOLSIM export is still SetVListMD's pair set row for row, and its forces
    and energies equal the full-list kernels' within FP32 rounding."""
    s = dict(getattr(Hp, which)())
    t, o, g = _pair(s, precision="mixed")
    _check_nlist(o, g, s["np"])
    rh = g.UTotal()
    for kind, tol in ((3, 1e-7), (1, 1e-6)):
        # the same kernel over a full list (FP64 sums: 1e-7), the lean FP32 kernel (1e-6)
        g.tune_pair_kernel(kind)
        _check_nlist(o, g, s["np"])
        rf = g.UTotal()
        assert Hp.rel_rms(rh["force"], rf["force"]) < 1e-6, kind
        for k in ("utot", "urec", "virial"):
            assert Hp.rel(rh[k], rf[k]) < tol, (kind, k)
    g.tune_pair_kernel(2)
    rh2 = g.UTotal()
    assert np.array_equal(rh["force"], rh2["force"]) and rh["utot"] == rh2["utot"]


def _check_nlist_fast(o, g, n):
    """As _check_nlist, vectorised for large systems."""
    nn_o, jp_o = o.get_vlist()
    nn_g, jp_g, npair = g.SetVList(0, export=True, maxnneigh=o.maxnneigh)
    assert npair == int(nn_o.sum())
    assert np.array_equal(nn_o, nn_g)
    mask = np.arange(jp_o.shape[1])[None, :] < nn_o[:, None]
    assert np.array_equal(np.where(mask, jp_o, 0), np.where(mask, jp_g, 0))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_past_one_scan_round_equals_alone(precision):
    """Two copies of the 200,000-particle BD config in one handle: 400,000 keys make the
    list rebuild's radix sort scan each digit's tile counts in more than one round of 256
    tiles (a copy alone needs one).  Each copy's list and forces equal the copy alone, bit
    for bit."""
    s = Hp.config2()
    t = Hp.oracle_table(s)
    sb = [dict(s), dict(s)]
    sb[1]["ro"] = np.array(s["ro"])[::-1].copy()      # the second copy in another MOLSIM order
    sb[1]["iptpn"] = np.array(s["iptpn"])[::-1].copy()
    sb[1]["az"] = np.array(s["az"])[::-1].copy()
    if "rod" in s:
        sb[1]["rod"] = np.array(s["rod"])[::-1].copy()
    gb = Engine(sb, [t, t], precision=precision, maxnneigh=256)
    for k in range(2):
        ga = Engine(sb[k], t, precision=precision, maxnneigh=256)
        ra, rb = ga.UTotal(), gb.UTotal(k)
        assert np.array_equal(rb["force"], ra["force"]), k
        assert rb["utot"] == ra["utot"] and rb["virial"] == ra["virial"], k
        nn_a, jp_a, _ = ga.SetVList(0, export=True, maxnneigh=256)
        nn_b, jp_b, _ = gb.SetVList(k, export=True, maxnneigh=256)
        assert np.array_equal(nn_a, nn_b) and np.array_equal(jp_a, jp_b), k
        del ga


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config2_colloid_bd_full_size(precision):
    """The 200,000-particle Brownian-dynamics config at full size against the oracle with
    its cell-list build: pair set bit-exact, UTotal, and two BD steps with injected noise."""
    s = Hp.config2()
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t, cell=True, maxnneigh=256)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    g = Engine(s, t, precision=precision, maxnneigh=256)
    _check_nlist_fast(o, g, s["np"])
    ro = o.utotal()
    rg = g.UTotal()
    assert Hp.rel_rms(rg["force"], ro["force"]) < FORCE_TOL
    for k in ("utot", "urec", "virial"):
        assert Hp.rel(rg[k], ro[k]) < ENERGY_TOL, (k, rg[k], ro[k])
    for p, v in enumerate(ro["utwob"]):
        assert abs(rg["utwob"][p] - v) <= ENERGY_TOL * max(abs(ro["utot"]), abs(v)), (p, rg["utwob"][p], v)
    rng = np.random.default_rng(11)
    xi = rng.standard_normal((2, s["np"], 3))
    fac1, fac2 = s["bd_fac"]
    g.BDStep(2, xi=xi, energies=False)
    for k in range(2):
        o.bd_step(xi[k], fac1, fac2)
    d = g.get_state()["ro"] - o.get_state()["ro"]
    box = s["boxlen"][0]
    d -= box * np.round(d / box)
    assert np.abs(d).max() < (1e-9 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("host", ["pageable", "pinned", "registered"])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_velver_host_equals_put_step_get(precision, host):
    """msg_velver_host (state in, steps, state out in one call) gives what
    msg_put_state + msg_velver + msg_get_state give, bit for bit in both precisions.
    Page-locked host arrays (allocated pinned, or plain arrays registered with
    cudaHostRegister) take the one-graph zero-copy path (one step per call),
    pageable ones the call-by-call path."""
    import torch

    s = dict(Hp.pe_small())
    t = Hp.oracle_table(s)
    a = Engine(s, t, precision=precision)
    b = Engine(s, t, precision=precision)
    for g in (a, b):
        g.UTotal()
        g.GetLinAcc()
    sa = a.get_state()
    sb = b.get_state()
    pinned = host != "pageable"
    registered = []
    if host == "pinned":
        for k in ("ro", "rod", "rodd"):
            buf = torch.empty(sb[k].shape, dtype=torch.float64, pin_memory=True).numpy()
            buf[:] = sb[k]
            sb[k] = buf
    elif host == "registered":
        rt = torch.cuda.cudart()
        for k in ("ro", "rod", "rodd"):
            sb[k] = np.ascontiguousarray(sb[k])
            # cudaHostRegisterMapped = 2
            assert int(rt.cudaHostRegister(sb[k].ctypes.data, sb[k].nbytes, 2)) == 0
            registered.append(sb[k])
    nstep = 1 if pinned else 2
    for _ in range(4):
        a.put_state(0, sa["ro"], sa["rod"], sa["rodd"], keep_list=True)
        la = a.launch_count()
        ea = a.VelVer(nstep)
        la = a.launch_count() - la
        sa = a.get_state()
        lb = b.launch_count()
        eb = b.VelVerHost(sb, nsteps=nstep)
        lb = b.launch_count() - lb
        # pageable: conversion in, the step graph, conversion out; page-locked: the same
        # step graph carrying conversion in, positions out early, the rest out and the read-back
        assert lb == la + (4 if pinned else 2), (la, lb)
    for arr in registered:
        assert int(torch.cuda.cudart().cudaHostUnregister(arr.ctypes.data)) == 0
    for k in ("ro", "rod", "rodd"):
        assert np.array_equal(sa[k], sb[k]), k
    for x, y in zip(ea, eb):
        for k in ("utot", "virial", "ekin"):
            assert x[k] == y[k], k


def test_set_state_all_equals_set_state_per_system():
    """msg_set_state_all (every system's state, one rebuild, one wait) leaves a batch
    handle exactly as msg_set_state per system does: same lists, forces and energies."""
    from molsim_b200 import _lib

    sy = [dict(Hp.electrolyte_small()), dict(Hp.electrolyte_small(seed=5)),
          dict(Hp.electrolyte_small(n_pairs=50, L=36.0, seed=4))]
    tb = [Hp.oracle_table(s) for s in sy]
    a = Engine(sy, tb, precision="mixed")            # built through msg_set_state_all
    b = Engine(sy, tb, precision="mixed")
    for k, s in enumerate(sy):
        b.set_state(k, s["ro"], s.get("rod"), s.get("rodd"))
    for g in (a, b):
        g.UTotal(0)
    for k, s in enumerate(sy):
        na, ja, pa = a.SetVList(k, export=True, maxnneigh=s["np"])
        nb, jb, pb = b.SetVList(k, export=True, maxnneigh=s["np"])
        assert pa == pb and np.array_equal(na, nb) and np.array_equal(ja, jb)
        assert np.array_equal(a.forces(k)[0], b.forces(k)[0])
        assert a.energy(k) == b.energy(k)
    assert _lib.lib().msg_set_state_all(a.h, None, None, None) == 6
