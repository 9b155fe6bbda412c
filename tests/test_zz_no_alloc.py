"""The allocation-free pair entry point (msg_utwobody_noalloc) against the
handle-based path.

msg_utwobody_noalloc exists for callers that cannot call cudaMalloc -- hosts
whose device memory all comes from their own pool or a framework allocator --
so it takes only caller-owned buffers and keeps its scratch in a fixed static
device array.  Here the caller's buffers come from torch; the reference answer
is msg_utotal of a handle for the same system without SPME and bonds (so its
force, u%twob and virial are the pair terms alone), and its MOLSIM-layout
Verlet list from msg_build_nlist.  Two calls in a row must both agree, which
also checks that the shared scratch is cleared between calls.
"""
import ctypes as C

import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine, _lib

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
ENERGY_TOL = 1e-7


def test_noalloc_pair_matches_handle_path():
    import torch

    s = dict(Hp.electrolyte_small())
    s["lewald"] = False
    s["lsurf"] = False
    t = Hp.oracle_table(s)
    g = Engine(s, t)
    ref = g.UTotal()
    n = int(s["np"])
    nn, jp, _ = g.SetVList(0, export=True, maxnneigh=n)
    natat = len(t["r2umin"])

    dev = torch.device("cuda")
    ro = torch.tensor(np.ascontiguousarray(s["ro"]), dtype=torch.float64, device=dev)
    ipt = torch.tensor(np.asarray(s["iptpn"], np.int32), device=dev)
    nnd = torch.tensor(nn, device=dev)
    jpd = torch.tensor(jp, device=dev)
    ubuf = torch.tensor(t["ubuf"], dtype=torch.float64, device=dev)
    force = torch.full((n, 3), 7.0, dtype=torch.float64, device=dev)    # must be overwritten
    utwob = torch.zeros(natat + 1, dtype=torch.float64, device=dev)
    vir = torch.zeros(1, dtype=torch.float64, device=dev)
    box = (C.c_double * 3)(*s["boxlen"])
    iub = np.ascontiguousarray(t["iubuflow"], np.int32)
    r2umin = np.ascontiguousarray(t["r2umin"], np.float64)
    r2atat = np.zeros(natat)
    f64 = C.POINTER(C.c_double)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    L = _lib.lib()
    for call in range(2):
        rc = L.msg_utwobody_noalloc(n, int(s["npt"]), box, s["rcut"], C.c_void_p(ro.data_ptr()),
                                    C.c_void_p(ipt.data_ptr()), C.c_void_p(nnd.data_ptr()),
                                    C.c_void_p(jpd.data_ptr()), n, C.c_void_p(ubuf.data_ptr()), len(t["ubuf"]),
                                    iub.ctypes.data_as(C.POINTER(C.c_int32)), r2umin.ctypes.data_as(f64),
                                    r2atat.ctypes.data_as(f64), C.c_void_p(force.data_ptr()),
                                    C.c_void_p(utwob.data_ptr()), C.c_void_p(vir.data_ptr()), stream)
        assert rc == 0, (call, rc)
        f = force.cpu().numpy()
        u = utwob.cpu().numpy()
        v = float(vir.cpu().numpy()[0])
        assert Hp.rel_rms(f, ref["force"]) < FORCE_TOL, call
        assert Hp.rel(u[0], ref["utwob"][0]) < ENERGY_TOL, call
        for p in range(natat):
            assert abs(u[1 + p] - ref["utwob"][1 + p]) <= ENERGY_TOL * abs(ref["utwob"][0]), (call, p)
        assert Hp.rel(v, ref["virial"]) < ENERGY_TOL, call
        force.fill_(7.0)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    """np above the static scratch's limit is refused before any launch."""
    L = _lib.lib()
    box = (C.c_double * 3)(10.0, 10.0, 10.0)
    one = np.ones(1, np.int32)
    z = np.zeros(1)
    f64 = C.POINTER(C.c_double)
    rc = L.msg_utwobody_noalloc(262144 + 1, 1, box, 4.0, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                C.c_void_p(1), 1, C.c_void_p(1), 12, one.ctypes.data_as(C.POINTER(C.c_int32)),
                                z.ctypes.data_as(f64), None, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), None)
    assert rc == 6   # MSG_ERR_ARG
