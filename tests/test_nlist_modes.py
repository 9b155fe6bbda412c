"""NList's other modes (Src/nlist.F90:597-621, 686-811, 1168-1260): the linked-list
Verlet build (lvlistllist: SetLList(rcut+drnlist) + SetVListMDLList, whose pair set can
leave out skin pairs and whose rows run cell by cell) and the fixed update interval
(inlist > 0: a rebuild whenever mod(istep2, inlist) == 0), against the oracle's
restatements of those routines."""
import numpy as np
import pytest

import helpers as Hp
from molsim_b200 import Engine, MolsimGpuError
from molsim_b200.engine import estimate_bytes


def _llist(s):
    d = dict(s)
    d["lvlistllist"] = True
    return d


def test_llist_refuses_more_than_1000_cells():
    """SetLList caps its cell arrays at 1000 (Src/nlist.F90:1195) without guarding larger
    grids; the library refuses such a system at set-up (checked without a GPU)."""
    s = _llist(Hp.config2())
    with pytest.raises(MolsimGpuError) as e:
        estimate_bytes(s, Hp.oracle_table(s))
    assert e.value.code == 6
    assert estimate_bytes(_llist(Hp.config0()), Hp.oracle_table(Hp.config0())) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("which", ["electrolyte_small", "config0", "pe_small"])
def test_llist_pair_set_and_rows_match_oracle(which, precision):
    """The exported list equals SetVListMDLList's entry for entry (row order included), it
    differs from SetVListMD's in the rows each pair lands in, and UTotal over it matches."""
    s = _llist(getattr(Hp, which)())
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    nn_o, jp_o = o.get_vlist()
    g = Engine(s, t, precision=precision)
    nn_g, jp_g, npair = g.SetVList(0, export=True, maxnneigh=o.maxnneigh)
    assert npair == int(nn_o.sum())
    assert np.array_equal(nn_o, nn_g)
    mask = np.arange(jp_o.shape[1])[None, :] < nn_o[:, None]
    assert np.array_equal(np.where(mask, jp_o, 0), np.where(mask, jp_g, 0))
    # rows run cell by cell, so some are not ascending
    assert any(np.any(np.diff(jp_o[i, :nn_o[i]]) < 0) for i in range(s["np"]))
    ro, rg = o.utotal(), g.UTotal()
    assert Hp.rel_rms(rg["force"], ro["force"]) < (1e-10 if precision == "fp64" else 1e-5)
    assert Hp.rel(rg["utot"], ro["utot"]) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("llist", [False, True])
def test_inlist_rebuilds_every_n_steps(llist, precision):
    """inlist = 3: the list is rebuilt after steps 3, 6, 9, ... of the macrostep, drosum
    is left alone, and msg_nlist_before_macrostep restarts the count; the trajectory
    follows the oracle's."""
    s = dict(Hp.pe_small())
    s["tstep"] = 0.02
    s["inlist"] = 3
    if llist:
        s = _llist(s)
    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    g = Engine(s, t, precision=precision)
    g.UTotal()
    g.GetLinAcc()
    st = g.get_state()
    o.set_state(st["ro"], st["rod"], st["rodd"])
    o.utotal()
    g.nlist_before_macrostep()
    o.nlist_before_macrostep()
    nb0 = g.nrebuild()
    for k in range(8):
        _, rb = o.velver_step()
        g.VelVer(1, energies=False)
        nb = g.nrebuild()
        assert (nb - nb0) == int(rb) == int((k + 1) % 3 == 0), k
        nb0 = nb
    g.nlist_before_macrostep()
    o.nlist_before_macrostep()
    for k in range(4):
        _, rb = o.velver_step()
        g.VelVer(1, energies=False)
        nb = g.nrebuild()
        assert (nb - nb0) == int(rb) == int(k == 2), k
        nb0 = nb
    sg, so = g.get_state(), o.get_state()
    d = sg["ro"] - so["ro"]
    box = s["boxlen"][0]
    d -= box * np.round(d / box)
    assert np.abs(d).max() < (1e-9 if precision == "fp64" else 1e-6)
