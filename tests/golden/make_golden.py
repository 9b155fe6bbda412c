"""Generate the golden fixtures of this directory from the FP64 oracle.

    python tests/golden/make_golden.py

Each fixture is a self-contained .npz: the system (every msg_params input,
positions and velocities), MOLSIM's pair table for it, and the oracle's
outputs: the Verlet list in MOLSIM's layout (SetVListMD, parity rule),
UTotal's force/forceo/energies/virial, and the state after three VelVer
steps.  They pin the oracle and the CUDA path against drift.  They are NOT
outputs of the compiled reference (none exists here: see the oracle header).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

SCALARS = ("np", "npt", "rcut", "drnlist", "lewald", "order", "nmesh", "lsurf", "epsi_four_pi", "tstep", "nbond")
ARRAYS = ("boxlen", "iptpn", "az", "masspt", "zat", "sigat", "epsat", "ro", "rod", "bond_ij", "bond_k", "bond_eq",
          "bond_p")


def cases():
    from molsim_b200 import systems as S

    e = S.electrolyte(seed=21, n_pairs=40, L=40.0, rcut=15.0, nmesh=16, order=4)
    p = S.polyelectrolyte(seed=22, nchain=3, nbead=20, L=50.0, rcut=16.0, nmesh=24, order=5)
    p["lsurf"] = True
    return {"electrolyte_80": e, "polyelectrolyte_120": p}


def make(name, s):
    import helpers as Hp

    t = Hp.oracle_table(s)
    o = Hp.oracle_system(s, t)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    nn, jp = o.get_vlist()
    u = o.utotal()
    # VelVer from rest of forces: rodd = forceo / mass (GetLinAcc)
    st = o.get_state()
    o.set_state(st["ro"], st["rod"], u["forceo"] / np.asarray(s["masspt"])[np.asarray(s["iptpn"]) - 1][:, None])
    ek = [o.velver_step()[0] for _ in range(3)]
    st3 = o.get_state()
    out = {k: np.asarray(s[k]) for k in SCALARS + ARRAYS}
    out.update({"tab_" + k: np.asarray(v) for k, v in t.items()})
    out.update(nneighpn=nn, jpnlist=jp, force=u["force"], forceo=u["forceo"], utot=u["utot"],
               utwob=u["utwob"], urec=u["urec"], ubond=u["ubond"], virial=u["virial"],
               ro3=st3["ro"], rod3=st3["rod"], ekin3=np.asarray(ek))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


def load(path):
    """(system dict, table dict, expected dict) of a fixture."""
    from molsim_b200 import systems as S

    z = np.load(path)
    s = {k: (z[k].item() if z[k].ndim == 0 else z[k]) for k in SCALARS + ARRAYS}
    s["boxlen"] = [float(x) for x in s["boxlen"]]
    for k in ("np", "npt", "lewald", "order", "nmesh", "lsurf", "nbond"):
        s[k] = int(s[k])
    # the table inputs that are not arrays (pot_tab is rebuilt only by the oracle-pin test)
    s.update(S.POT_DEFAULTS)
    s["uewaldtol"] = 1e-5
    s["lljcut"] = True
    t = {k[4:]: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files if k.startswith("tab_")}
    want = {k: (z[k].item() if z[k].ndim == 0 else z[k]) for k in z.files
            if k not in SCALARS + ARRAYS and not k.startswith("tab_")}
    return s, t, want


if __name__ == "__main__":
    for name, s in cases().items():
        make(name, s)
        print("wrote", name)
