"""The allocation-free pair entry point (msg_utwobody_noalloc).

msg_utwobody_noalloc exists for callers that cannot call cudaMalloc -- hosts
whose device memory all comes from their own pool or a framework allocator --
so it takes only caller-owned buffers and keeps its scratch in a fixed static
device array.  Here the caller's buffers come from torch.  It is checked
against the handle path (msg_utotal of a handle without SPME and bonds, so its
force, u%twob and virial are the pair terms alone) and against the FP64 oracle
on the oracle's own MOLSIM-layout lists: the MD half list, and a Monte Carlo
full list (lmc = 1).  Two calls in a row must agree, which also checks that the
shared scratch is cleared between calls.  The error statuses are host-visible
values: a pair below the table's r2umin reports MSG_ERR_TABLE_MIN with its
(ip, jp), and a row longer than maxnneigh reports MSG_ERR_ARG.
"""
import ctypes as C

import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine, _lib

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
ENERGY_TOL = 1e-7
MSG_ERR_TABLE_MIN = 1
MSG_ERR_ARG = 6


def _pair_only(s):
    s = dict(s)
    s["lewald"] = False
    s["lsurf"] = False
    return s


def _call(s, t, nn, jp, maxnneigh, lmc=0, ro=None, calls=2):
    """Run the entry point `calls` times on device copies of the caller's arrays; returns
    (status, stop_ipjp, force, utwob, virial) of each call."""
    import torch

    n = int(s["np"])
    natat = len(t["r2umin"])
    dev = torch.device("cuda")
    rod = torch.tensor(np.ascontiguousarray(s["ro"] if ro is None else ro), dtype=torch.float64, device=dev)
    ipt = torch.tensor(np.asarray(s["iptpn"], np.int32), device=dev)
    nnd = torch.tensor(np.ascontiguousarray(nn, np.int32), device=dev)
    jpd = torch.tensor(np.ascontiguousarray(jp, np.int32), device=dev)
    ubuf = torch.tensor(t["ubuf"], dtype=torch.float64, device=dev)
    force = torch.full((n, 3), 7.0, dtype=torch.float64, device=dev)    # must be overwritten
    utwob = torch.zeros(natat + 1, dtype=torch.float64, device=dev)
    vir = torch.zeros(1, dtype=torch.float64, device=dev)
    box = (C.c_double * 3)(*s["boxlen"])
    iub = np.ascontiguousarray(t["iubuflow"], np.int32)
    r2umin = np.ascontiguousarray(t["r2umin"], np.float64)
    r2atat = np.zeros(natat)
    f64 = C.POINTER(C.c_double)
    i32 = C.POINTER(C.c_int32)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    out = []
    for _ in range(calls):
        stop = np.full(2, -1, np.int32)
        rc = L.msg_utwobody_noalloc(n, int(s["npt"]), box, s["rcut"], C.c_void_p(rod.data_ptr()),
                                    C.c_void_p(ipt.data_ptr()), C.c_void_p(nnd.data_ptr()),
                                    C.c_void_p(jpd.data_ptr()), int(maxnneigh), int(lmc),
                                    C.c_void_p(ubuf.data_ptr()), len(t["ubuf"]), iub.ctypes.data_as(i32),
                                    r2umin.ctypes.data_as(f64), r2atat.ctypes.data_as(f64),
                                    C.c_void_p(force.data_ptr()), C.c_void_p(utwob.data_ptr()),
                                    C.c_void_p(vir.data_ptr()), stop.ctypes.data_as(i32), stream)
        out.append((rc, stop.copy(), force.cpu().numpy().copy(), utwob.cpu().numpy().copy(),
                    float(vir.cpu().numpy()[0])))
        force.fill_(7.0)
    return out


def _check(res, ref, natat):
    for call, (rc, stop, f, u, v) in enumerate(res):
        assert rc == 0 and list(stop) == [0, 0], (call, rc, stop)
        assert Hp.rel_rms(f, ref["force"]) < FORCE_TOL, call
        assert Hp.rel(u[0], ref["utwob"][0]) < ENERGY_TOL, call
        for p in range(natat):
            assert abs(u[1 + p] - ref["utwob"][1 + p]) <= ENERGY_TOL * abs(ref["utwob"][0]), (call, p)
        assert Hp.rel(v, ref["virial"]) < ENERGY_TOL, call


def test_noalloc_pair_matches_handle_path():
    s = _pair_only(Hp.electrolyte_small())
    t = Hp.oracle_table(s)
    g = Engine(s, t)
    ref = g.UTotal()
    n = int(s["np"])
    nn, jp, _ = g.SetVList(0, export=True, maxnneigh=n)
    _check(_call(s, t, nn, jp, n), ref, len(t["r2umin"]))


def _oracle(s):
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    nn, jp = o.get_vlist()
    return t, o, nn, jp, o.utotal()


@pytest.mark.parametrize("which", ["config0", "colloid_small"])
def test_noalloc_pair_matches_oracle(which):
    """On the oracle's own half list: the 1000-ion electrolyte (2 types) and the colloid
    system with three particle types (npt = 3, six type pairs)."""
    s = _pair_only(getattr(Hp, which)())
    t, o, nn, jp, ref = _oracle(s)
    assert int(s["npt"]) == (2 if which == "config0" else 3)
    _check(_call(s, t, nn, jp, jp.shape[1]), ref, len(t["r2umin"]))


def test_noalloc_full_list_with_lmc():
    """A Monte Carlo full list (every pair in both rows, as SetVListMC stores it) with
    lmc = 1 gives the half list's answer; without lmc it would count every pair twice."""
    s = _pair_only(Hp.electrolyte_small())
    t, o, nn, jp, ref = _oracle(s)
    n = int(s["np"])
    rows = [[] for _ in range(n)]
    for ip in range(n):
        for k in range(nn[ip]):
            j = int(jp[ip, k])
            rows[ip].append(j)
            rows[j - 1].append(ip + 1)
    mx = max(len(r) for r in rows)
    nnf = np.array([len(r) for r in rows], np.int32)
    jpf = np.zeros((n, mx), np.int32)
    for ip, r in enumerate(rows):
        jpf[ip, :len(r)] = sorted(r)
    assert int(nnf.sum()) == 2 * int(nn.sum())
    _check(_call(s, t, nnf, jpf, mx, lmc=1), ref, len(t["r2umin"]))
    rc, _, _, u, _ = _call(s, t, nnf, jpf, mx, lmc=0, calls=1)[0]
    assert rc == 0 and Hp.rel(u[0], 2.0 * ref["utwob"][0]) < ENERGY_TOL


def test_noalloc_reports_the_pair_below_the_table():
    """Two ions moved 0.05 A apart lie below r2umin: the call returns MSG_ERR_TABLE_MIN
    with that pair's 1-based (ip, jp), as StopUTwoBodyA reports it; the next clean call
    is back to status 0 (the shared error word is cleared)."""
    s = _pair_only(Hp.electrolyte_small())
    t = Hp.oracle_table(s)
    ro = np.array(s["ro"], np.float64)
    ro[7] = ro[3] + np.array([0.05, 0.0, 0.0])
    d = dict(s)
    d["ro"] = ro
    o = Hp.oracle_system(d, t)
    o.set_state(ro, s["rod"])
    o.set_vlist()
    nn, jp = o.get_vlist()
    assert 0.05 ** 2 < t["r2umin"].min()
    rc, stop, _, _, _ = _call(d, t, nn, jp, jp.shape[1], calls=1)[0]
    assert rc == MSG_ERR_TABLE_MIN
    assert sorted(stop.tolist()) == [4, 8]
    t2, o2, nn2, jp2, ref = _oracle(s)
    _check(_call(s, t2, nn2, jp2, jp2.shape[1], calls=1), ref, len(t2["r2umin"]))


def test_noalloc_rejects_a_row_longer_than_maxnneigh():
    s = _pair_only(Hp.electrolyte_small())
    t, o, nn, jp, ref = _oracle(s)
    bad = nn.copy()
    ip = int(np.argmax(nn))
    bad[ip] = jp.shape[1] + 1
    rc, stop, _, _, _ = _call(s, t, bad, jp, jp.shape[1], calls=1)[0]
    assert rc == MSG_ERR_ARG and stop.tolist() == [ip + 1, 0]


def test_noalloc_rejects_sizes_beyond_its_scratch():
    """np above the static scratch's limit is refused before any launch."""
    L = _lib.lib()
    box = (C.c_double * 3)(10.0, 10.0, 10.0)
    one = np.ones(1, np.int32)
    z = np.zeros(1)
    f64 = C.POINTER(C.c_double)
    rc = L.msg_utwobody_noalloc(262144 + 1, 1, box, 4.0, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                C.c_void_p(1), 1, 0, C.c_void_p(1), 12, one.ctypes.data_as(C.POINTER(C.c_int32)),
                                z.ctypes.data_as(f64), None, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None,
                                None)
    assert rc == MSG_ERR_ARG
