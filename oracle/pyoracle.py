"""ctypes binding of the FP64 oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by the tests, the smoke check and the CPU
baseline leg of the benchmark, never by the product package.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)


class TabParams(C.Structure):
    _fields_ = [("npt", C.c_int32), ("zat", f64p), ("sigat", f64p), ("epsat", f64p),
                ("rcut", C.c_double), ("ualpha", C.c_double), ("epsi_four_pi", C.c_double),
                ("lewald", C.c_int32), ("lljcut", C.c_int32), ("ljrcut", C.c_double),
                ("ljushift", C.c_double), ("r2uminin", C.c_double), ("utoltab", C.c_double),
                ("ftoltab", C.c_double), ("umaxtab", C.c_double), ("fmaxtab", C.c_double),
                ("rumaxfac", C.c_double)]


class Params(C.Structure):
    _fields_ = [("np", C.c_int32), ("npt", C.c_int32), ("boxlen", C.c_double * 3),
                ("rcut", C.c_double), ("drnlist", C.c_double), ("iptpn", i32p), ("az", f64p),
                ("masspt", f64p), ("ubuf", f64p), ("nbuf", C.c_int32), ("iubuflow", i32p),
                ("r2umin", f64p), ("r2atat", f64p), ("lewald", C.c_int32), ("order", C.c_int32),
                ("nmesh", C.c_int32), ("lsurf", C.c_int32), ("ualpha", C.c_double),
                ("epsi_four_pi", C.c_double), ("nbond", C.c_int32), ("bond_ij", i32p),
                ("bond_k", f64p), ("bond_eq", f64p), ("bond_p", i32p), ("tstep", C.c_double),
                ("maxnneigh", C.c_int32), ("lcellbuild", C.c_int32), ("ncut", C.c_int32),
                ("ncutregion", C.c_int32), ("lewald2dlc", C.c_int32), ("inlist", C.c_int32),
                ("lvlistllist", C.c_int32)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE])
        L = C.CDLL(path)
        L.or_erf2.restype = C.c_double
        L.or_erf2.argtypes = [C.c_double]
        L.or_epsi0_four_pi.restype = C.c_double
        L.or_gas_constant.restype = C.c_double
        L.or_ewald_ufac.argtypes = [C.c_double, C.c_double, f64p]
        L.or_cardinal_bspline.argtypes = [C.c_int, C.c_double, i32p, f64p, f64p]
        L.or_rcut_to_alpha.restype = C.c_double
        L.or_rcut_to_alpha.argtypes = [C.c_double] * 5 + [i32p]
        L.or_random_next.restype = C.c_double
        L.or_random_next.argtypes = [i32p]
        L.or_random_init.argtypes = [C.c_int32, i32p]
        L.or_mc_seed.argtypes = [C.c_void_p, C.c_int32]
        L.or_mc_pass.restype = C.c_int
        L.or_mc_pass.argtypes = [C.c_void_p, C.c_int, C.c_int, f64p, C.c_double, f64p,
                                 C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.or_utwobody_p.restype = C.c_int
        L.or_utwobody_p.argtypes = [C.c_int32] * 4 + [f64p, C.c_double, f64p, f64p] + [i32p] * 6 + \
            [C.c_int32, f64p, C.c_int32, i32p, f64p, f64p, f64p, f64p]
        L.or_alpha_to_ncut.restype = C.c_int32
        L.or_alpha_to_ncut.argtypes = [C.c_double] * 5 + [i32p]
        L.or_ewald_error_ureal.restype = C.c_double
        L.or_ewald_error_ureal.argtypes = [C.c_double] * 5
        L.or_pot_1_6_12.argtypes = [C.POINTER(TabParams), C.c_int, C.c_int, C.c_double, f64p, f64p, f64p]
        L.or_pot_tab.restype = C.c_int
        L.or_pot_tab.argtypes = [C.POINTER(TabParams), f64p, C.c_int32, i32p, i32p, f64p, f64p, f64p, i32p]
        L.or_ewald_setup_spm.argtypes = [C.c_int, C.c_int, C.c_double, f64p, f64p, f64p, f64p]
        L.or_fft3_r2c.argtypes = [C.c_int, f64p, f64p]
        L.or_fft3_c2r.argtypes = [C.c_int, f64p, f64p]
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.POINTER(Params)]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_set_state.argtypes = [C.c_void_p, f64p, f64p, f64p]
        L.or_get_state.argtypes = [C.c_void_p, f64p, f64p, f64p, f64p]
        L.or_set_drosum.argtypes = [C.c_void_p, f64p]
        L.or_set_vlist.restype = C.c_int
        L.or_set_vlist.argtypes = [C.c_void_p]
        L.or_nlist_before_macrostep.argtypes = [C.c_void_p]
        L.or_get_vlist.argtypes = [C.c_void_p, i32p, i32p]
        L.or_npair.restype = C.c_int64
        L.or_npair.argtypes = [C.c_void_p]
        L.or_utotal.restype = C.c_int
        L.or_utotal.argtypes = [C.c_void_p, f64p, f64p, f64p, f64p]
        L.or_velver_step.restype = C.c_int
        L.or_velver_step.argtypes = [C.c_void_p, f64p, i32p]
        L.or_bd_step.restype = C.c_int
        L.or_bd_step.argtypes = [C.c_void_p, f64p, f64p, f64p, i32p]
        L.or_gau_random.restype = C.c_double
        L.or_gau_random.argtypes = [i32p, i32p, f64p]
        L.or_skin_test.restype = C.c_int
        L.or_skin_test.argtypes = [C.c_void_p, f64p, f64p, f64p]
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def erf2(x):
    return lib().or_erf2(float(x))


def ewald_ufac(r, alpha):
    c = np.zeros(3)
    lib().or_ewald_ufac(r, alpha, _p(c, C.c_double))
    return c


def bspline(order, pos):
    v = np.zeros(order)
    d = np.zeros(order)
    k = C.c_int32()
    lib().or_cardinal_bspline(order, pos, C.byref(k), _p(v, C.c_double), _p(d, C.c_double))
    return k.value, v, d


def rcut_to_alpha(uewaldtol, q2sum, epsfp, boxlenshort, rcut):
    st = C.c_int32()
    a = lib().or_rcut_to_alpha(uewaldtol, q2sum, epsfp, boxlenshort, rcut, C.byref(st))
    if st.value:
        raise RuntimeError("RcutToAlpha did not converge")
    return a


def alpha_to_ncut(uewaldtol, q2sum, epsfp, boxlenshort, ualpha):
    st = C.c_int32()
    n = lib().or_alpha_to_ncut(uewaldtol, q2sum, epsfp, boxlenshort, ualpha, C.byref(st))
    if st.value:
        raise RuntimeError("AlphaToNcut did not converge")
    return int(n)


def ewald_mode(sysd):
    """lewald as the oracle takes it: 0 none, 1 SPME, 2 standard Ewald (txewaldrec 'std')."""
    if not sysd["lewald"]:
        return 0
    return 2 if sysd.get("ewaldrec", "spm") == "std" else 1


def tab_params(pot):
    """pot: dict with npt, zat, sigat, epsat, rcut, ualpha, epsi_four_pi, lewald, lljcut,
    ljrcut, ljushift, r2uminin, utoltab, ftoltab, umaxtab, fmaxtab, rumaxfac."""
    keep = {k: np.ascontiguousarray(pot[k], dtype=np.float64) for k in ("zat", "sigat", "epsat")}
    tp = TabParams(pot["npt"], _p(keep["zat"], C.c_double), _p(keep["sigat"], C.c_double),
                   _p(keep["epsat"], C.c_double), pot["rcut"], pot["ualpha"], pot["epsi_four_pi"],
                   int(pot["lewald"]), int(pot["lljcut"]), pot["ljrcut"], pot["ljushift"],
                   pot["r2uminin"], pot["utoltab"], pot["ftoltab"], pot["umaxtab"], pot["fmaxtab"],
                   pot["rumaxfac"])
    return tp, keep


def pot(potd, iat, jat, r):
    tp, keep = tab_params(potd)
    u = [C.c_double(), C.c_double(), C.c_double()]
    lib().or_pot_1_6_12(C.byref(tp), iat, jat, r, *[C.byref(x) for x in u])
    return tuple(x.value for x in u)


def pot_tab(potd, nbuf=200000):
    tp, keep = tab_params(potd)
    natat = potd["npt"] * (potd["npt"] + 1) // 2
    ubuf = np.zeros(nbuf)
    iub = np.zeros(natat, np.int32)
    nug = np.zeros(natat, np.int32)
    r2umin = np.zeros(natat)
    rumin = np.zeros(natat)
    rumax = np.zeros(natat)
    nused = C.c_int32()
    rc = lib().or_pot_tab(C.byref(tp), _p(ubuf, C.c_double), nbuf, _p(iub, C.c_int32),
                          _p(nug, C.c_int32), _p(r2umin, C.c_double), _p(rumin, C.c_double),
                          _p(rumax, C.c_double), C.byref(nused))
    if rc:
        raise RuntimeError("or_pot_tab failed: %d" % rc)
    return dict(ubuf=ubuf[:nused.value].copy(), iubuflow=iub, nugrid=nug, r2umin=r2umin,
                rumin=rumin, rumax=rumax)


def ewald_setup_spm(s, order, alpha, box):
    h = s // 2 + 1
    mf = np.zeros(h ** 3)
    ef = np.zeros(h ** 3)
    vf = np.zeros(h ** 3)
    b = np.ascontiguousarray(box, dtype=np.float64)
    lib().or_ewald_setup_spm(s, order, alpha, _p(b, C.c_double), _p(mf, C.c_double),
                             _p(ef, C.c_double), _p(vf, C.c_double))
    sh = (h, h, h)
    return mf.reshape(sh), ef.reshape(sh), vf.reshape(sh)


def fft3_r2c(q):
    s = q.shape[0]
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.zeros((s, s, s // 2 + 1), np.complex128)
    lib().or_fft3_r2c(s, _p(q, C.c_double), out.ctypes.data_as(f64p))
    return out


def fft3_c2r(f):
    s = f.shape[0]
    f = np.ascontiguousarray(f, dtype=np.complex128)
    out = np.zeros((s, s, s))
    lib().or_fft3_c2r(s, f.ctypes.data_as(f64p), _p(out, C.c_double))
    return out


class System:
    """The oracle's MolModule state for one system (see or_params in oracle.h)."""

    def __init__(self, sysd, table, maxnneigh=None, lcellbuild=False):
        L = lib()
        self.np = int(sysd["np"])
        self.npt = int(sysd["npt"])
        self.natat = self.npt * (self.npt + 1) // 2
        k = {}
        k["iptpn"] = np.ascontiguousarray(sysd["iptpn"], np.int32)
        k["az"] = np.ascontiguousarray(sysd["az"], np.float64)
        k["masspt"] = np.ascontiguousarray(sysd["masspt"], np.float64)
        k["ubuf"] = np.ascontiguousarray(table["ubuf"], np.float64)
        k["iubuflow"] = np.ascontiguousarray(table["iubuflow"], np.int32)
        k["r2umin"] = np.ascontiguousarray(table["r2umin"], np.float64)
        k["r2atat"] = np.ascontiguousarray(sysd.get("r2atat", np.zeros(self.natat)), np.float64)
        nb = int(sysd.get("nbond", 0))
        k["bond_ij"] = np.ascontiguousarray(sysd.get("bond_ij", np.zeros((0, 2))), np.int32).reshape(-1)
        k["bond_k"] = np.ascontiguousarray(sysd.get("bond_k", np.zeros(0)), np.float64)
        k["bond_eq"] = np.ascontiguousarray(sysd.get("bond_eq", np.zeros(0)), np.float64)
        k["bond_p"] = np.ascontiguousarray(sysd.get("bond_p", np.zeros(0)), np.int32)
        self._keep = k
        if maxnneigh is None:
            maxnneigh = self.np
        self.maxnneigh = int(maxnneigh)
        box = (C.c_double * 3)(*sysd["boxlen"])
        P = Params(self.np, self.npt, box, sysd["rcut"], sysd["drnlist"],
                   _p(k["iptpn"], C.c_int32), _p(k["az"], C.c_double), _p(k["masspt"], C.c_double),
                   _p(k["ubuf"], C.c_double), len(k["ubuf"]), _p(k["iubuflow"], C.c_int32),
                   _p(k["r2umin"], C.c_double), _p(k["r2atat"], C.c_double),
                   ewald_mode(sysd), int(sysd["order"]), int(sysd["nmesh"]), int(sysd["lsurf"]),
                   sysd["ualpha"], sysd["epsi_four_pi"], nb, _p(k["bond_ij"], C.c_int32),
                   _p(k["bond_k"], C.c_double), _p(k["bond_eq"], C.c_double),
                   _p(k["bond_p"], C.c_int32), sysd["tstep"], self.maxnneigh, int(lcellbuild),
                   int(sysd.get("ncut", 0)), 1 if sysd.get("ncutregion", "sphere") == "cube" else 0,
                   int(bool(sysd.get("lewald2dlc", False))), int(sysd.get("inlist", 0)),
                   int(bool(sysd.get("lvlistllist", False))))
        self.h = L.or_create(C.byref(P))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    def set_state(self, ro, rod=None, rodd=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (ro, rod, rodd)]
        ptrs = [None if a is None else _p(a, C.c_double) for a in arrs]
        lib().or_set_state(self.h, *ptrs)

    def get_state(self):
        out = [np.zeros((self.np, 3)) for _ in range(4)]
        lib().or_get_state(self.h, *[_p(a, C.c_double) for a in out])
        return dict(ro=out[0], rod=out[1], rodd=out[2], drosum=out[3])

    def set_vlist(self):
        rc = lib().or_set_vlist(self.h)
        if rc:
            raise RuntimeError("SetVListMD failed: %d" % rc)

    def nlist_before_macrostep(self):
        """NList(iBeforeMacrostep): drosum = 0, istep2 restarts."""
        lib().or_nlist_before_macrostep(self.h)

    def get_vlist(self):
        nn = np.zeros(self.np, np.int32)
        jp = np.zeros((self.np, self.maxnneigh), np.int32)
        lib().or_get_vlist(self.h, _p(nn, C.c_int32), _p(jp, C.c_int32))
        return nn, jp

    def npair(self):
        return lib().or_npair(self.h)

    def utotal(self):
        f = np.zeros((self.np, 3))
        fo = np.zeros((self.np, 3))
        u = np.zeros(4 + self.natat)
        vir = C.c_double()
        rc = lib().or_utotal(self.h, _p(f, C.c_double), _p(fo, C.c_double), _p(u, C.c_double),
                             C.byref(vir))
        if rc:
            raise RuntimeError("UTotal failed: %d" % rc)
        return dict(force=f, forceo=fo, utot=u[0], utwob=u[1:2 + self.natat].copy(),
                    urec=u[2 + self.natat], ubond=u[3 + self.natat], virial=vir.value)

    def velver_step(self):
        ek = C.c_double()
        rb = C.c_int32()
        rc = lib().or_velver_step(self.h, C.byref(ek), C.byref(rb))
        if rc:
            raise RuntimeError("VelVer failed: %d" % rc)
        return ek.value, bool(rb.value)

    def bd_step(self, xi, fac1, fac2):
        xi = np.ascontiguousarray(xi, np.float64)
        f1 = np.ascontiguousarray(fac1, np.float64)
        f2 = np.ascontiguousarray(fac2, np.float64)
        rb = C.c_int32()
        rc = lib().or_bd_step(self.h, _p(xi, C.c_double), _p(f1, C.c_double), _p(f2, C.c_double),
                              C.byref(rb))
        if rc:
            raise RuntimeError("BDStep failed: %d" % rc)
        return bool(rb.value)

    def mc_seed(self, iseed):
        lib().or_mc_seed(self.h, int(iseed))

    def mc_pass(self, npass, dtran, beta, u, isamp=0):
        """npass MC sweeps; u (the utotal() energies) is advanced in place.
        Returns (accepted, hard-core rejects)."""
        d = np.ascontiguousarray(dtran, np.float64)
        uu = np.concatenate([[u["utot"]], u["utwob"], [u["urec"], u["ubond"]]]).astype(np.float64)
        acc = C.c_int64(0)
        hs = C.c_int64(0)
        rc = lib().or_mc_pass(self.h, int(npass), int(isamp), _p(d, C.c_double), float(beta),
                              _p(uu, C.c_double), C.byref(acc), C.byref(hs))
        if rc:
            raise RuntimeError("MC pass failed: %d" % rc)
        u["utot"] = uu[0]
        u["utwob"] = uu[1:2 + self.natat].copy()
        u["urec"] = uu[2 + self.natat]
        u["ubond"] = uu[3 + self.natat]
        return acc.value, hs.value

    def mc_pass_moves(self, npass, dtran, beta, u, pspart, pchain, dtranchain, chains, isamp=0):
        """npass MCPass sweeps with single-particle and chain moves (cumulative pspart, pchain
        [npt]; dtranchain [npt]; chains: (first 0-based, length) pairs); u advanced in place.
        Returns (accepted, hard-core rejects)."""
        L = lib()
        L.or_mc_pass_moves.restype = C.c_int
        L.or_mc_pass_moves.argtypes = [C.c_void_p, C.c_int, C.c_int, f64p, f64p, f64p, f64p, C.c_int, i32p, i32p,
                                       C.c_double, f64p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        arr = [np.ascontiguousarray(x, np.float64) for x in (dtran, pspart, pchain, dtranchain)]
        cf = np.ascontiguousarray([c[0] for c in chains], np.int32)
        cl = np.ascontiguousarray([c[1] for c in chains], np.int32)
        uu = np.concatenate([[u["utot"]], u["utwob"], [u["urec"], u["ubond"]]]).astype(np.float64)
        acc = C.c_int64(0)
        hs = C.c_int64(0)
        rc = L.or_mc_pass_moves(self.h, int(npass), int(isamp), *[_p(x, C.c_double) for x in arr], len(chains),
                                _p(cf, C.c_int32), _p(cl, C.c_int32), float(beta), _p(uu, C.c_double),
                                C.byref(acc), C.byref(hs))
        if rc:
            raise RuntimeError("MC pass with moves failed: %d" % rc)
        u["utot"] = uu[0]
        u["utwob"] = uu[1:2 + self.natat].copy()
        u["urec"] = uu[2 + self.natat]
        u["ubond"] = uu[3 + self.natat]
        return acc.value, hs.value

    def mcall_pass(self, npass, dtranall, beta, u):
        """npass MCAll trials (all particles at once); u advanced in place.  Returns accepted."""
        L = lib()
        L.or_mcall_pass.restype = C.c_int
        L.or_mcall_pass.argtypes = [C.c_void_p, C.c_int, f64p, C.c_double, f64p, C.POINTER(C.c_int64)]
        d = np.ascontiguousarray(dtranall, np.float64)
        uu = np.concatenate([[u["utot"]], u["utwob"], [u["urec"], u["ubond"]]]).astype(np.float64)
        acc = C.c_int64(0)
        rc = L.or_mcall_pass(self.h, int(npass), _p(d, C.c_double), float(beta), _p(uu, C.c_double), C.byref(acc))
        if rc:
            raise RuntimeError("MCAll pass failed: %d" % rc)
        u["utot"] = uu[0]
        u["utwob"] = uu[1:2 + self.natat].copy()
        u["urec"] = uu[2 + self.natat]
        u["ubond"] = uu[3 + self.natat]
        return acc.value

    def set_drosum(self, drosum):
        d = np.ascontiguousarray(drosum, np.float64)
        lib().or_set_drosum(self.h, _p(d, C.c_double))

    def skin_test(self, drostep):
        d = np.ascontiguousarray(drostep, np.float64)
        m1 = C.c_double()
        m2 = C.c_double()
        r = lib().or_skin_test(self.h, _p(d, C.c_double), C.byref(m1), C.byref(m2))
        return bool(r), m1.value, m2.value


def utwobody_p(s, table):
    """UTwoBodyP (oracle) for a polyatomic system dict (molsim_b200.systems.rigid_molecules
    layout) and its atom-type table.  Returns dict(force, utwob, virial)."""
    k = {}
    for key, dt in (("ro", np.float64), ("r", np.float64), ("iptpn", np.int32), ("ianpn", np.int32),
                    ("napt", np.int32), ("iatan", np.int32), ("nneighpn", np.int32), ("jpnlist", np.int32)):
        k[key] = np.ascontiguousarray(s[key], dt)
    ub = np.ascontiguousarray(table["ubuf"], np.float64)
    iub = np.ascontiguousarray(table["iubuflow"], np.int32)
    r2 = np.ascontiguousarray(table["r2umin"], np.float64)
    na, npt = int(s["na"]), int(s["npt"])
    force = np.zeros((na, 3))
    utwob = np.zeros(npt * (npt + 1) // 2 + 1)
    vir = C.c_double()
    box = (C.c_double * 3)(*s["boxlen"])
    rc = lib().or_utwobody_p(int(s["np"]), na, npt, int(s["nat"]), box, float(s["rcut"]),
                             _p(k["ro"], C.c_double), _p(k["r"], C.c_double), _p(k["iptpn"], C.c_int32),
                             _p(k["ianpn"], C.c_int32), _p(k["napt"], C.c_int32), _p(k["iatan"], C.c_int32),
                             _p(k["nneighpn"], C.c_int32), _p(k["jpnlist"], C.c_int32), int(k["jpnlist"].shape[1]),
                             _p(ub, C.c_double), len(ub), _p(iub, C.c_int32), _p(r2, C.c_double),
                             _p(force, C.c_double), _p(utwob, C.c_double), C.byref(vir))
    if rc:
        raise RuntimeError("UTwoBodyP failed: %d" % rc)
    return dict(force=force, utwob=utwob, virial=vir.value)


def velver_p(s, table, nsteps, ewald=None):
    """nsteps of rigid-body VelVer (oracle) on a systems.rigid_bodies dict, advanced in place
    (ro, rod, rodd, qua, quad, quadd, r).  ewald (optional): dict(az, ualpha, lsurf and either
    ncut, region (standard Ewald) or order, nmesh (SPME)) adds the site Ewald sum to every step.  Returns dict(utwob, virial[, urec]) of the
    last step."""
    L = lib()
    if not getattr(L, "_velver_p_typed", False):
        common = [C.c_int32] * 5 + [f64p, C.c_double, C.c_double, C.c_int32, C.c_double] + \
            [f64p] * 7 + [i32p] * 4 + [f64p, C.c_int32, f64p, f64p, i32p, i32p, C.c_int32, f64p, C.c_int32,
                                         i32p, f64p]
        L.or_velver_p.restype = C.c_int
        L.or_velver_p.argtypes = common + [f64p, f64p]
        L.or_velver_p_ewald.restype = C.c_int
        L.or_velver_p_ewald.argtypes = common + [f64p, C.c_double] + [C.c_int32] * 6 + [C.c_double, f64p, f64p,
                                                                                         f64p]
        L._velver_p_typed = True
    k = {}
    for key in ("ro", "rod", "rodd", "qua", "quad", "quadd", "r", "ra", "masspt", "momp"):
        k[key] = np.ascontiguousarray(s[key], np.float64)
    for key in ("iptpn", "ianpn", "napt", "iatan", "nneighpn", "jpnlist"):
        k[key] = np.ascontiguousarray(s[key], np.int32)
    ub = np.ascontiguousarray(table["ubuf"], np.float64)
    iub = np.ascontiguousarray(table["iubuflow"], np.int32)
    r2 = np.ascontiguousarray(table["r2umin"], np.float64)
    npt = int(s["npt"])
    utwob = np.zeros(npt * (npt + 1) // 2 + 1)
    vir = C.c_double()
    box = (C.c_double * 3)(*s["boxlen"])
    args = [int(nsteps), int(s["np"]), int(s["na"]), npt, int(s["nat"]), box, float(s["rcut"]),
            float(s["tstep"]), int(s["nvvite"]), float(s["tvvite"]),
            *[_p(k[x], C.c_double) for x in ("ro", "rod", "rodd", "qua", "quad", "quadd", "r")],
            *[_p(k[x], C.c_int32) for x in ("iptpn", "ianpn", "napt", "iatan")],
            _p(k["ra"], C.c_double), int(s["maxsite"]), _p(k["masspt"], C.c_double),
            _p(k["momp"], C.c_double), _p(k["nneighpn"], C.c_int32), _p(k["jpnlist"], C.c_int32),
            int(k["jpnlist"].shape[1]), _p(ub, C.c_double), len(ub), _p(iub, C.c_int32), _p(r2, C.c_double)]
    urec = C.c_double()
    if ewald is None:
        rc = L.or_velver_p(*args, _p(utwob, C.c_double), C.byref(vir))
    else:
        az = np.ascontiguousarray(ewald["az"], np.float64)
        spm = "nmesh" in ewald
        rc = L.or_velver_p_ewald(*args, _p(az, C.c_double), float(ewald["ualpha"]), 1 if spm else 2,
                                 int(ewald.get("ncut", 0)), 1 if ewald.get("region", "sphere") == "cube" else 0,
                                 int(ewald.get("order", 0)), int(ewald.get("nmesh", 0)),
                                 int(bool(ewald.get("lsurf"))), float(s["epsi_four_pi"]), _p(utwob, C.c_double),
                                 C.byref(urec), C.byref(vir))
    if rc:
        raise RuntimeError("VelVer (polyatomic) failed: %d" % rc)
    for key in ("ro", "rod", "rodd", "qua", "quad", "quadd", "r"):
        s[key] = k[key]
    out = dict(utwob=utwob, virial=vir.value)
    if ewald is not None:
        out["urec"] = urec.value
    return out


def uewald_sites(s, az, ualpha, ncut=None, region="sphere", lsurf=False, order=None, nmesh=None):
    """UEwald over the sites of a polyatomic system dict (oracle): dict(force, urec, virrec).
    Standard Ewald with ncut (region 'sphere' or 'cube'), or SPME with order and nmesh."""
    L = lib()
    if not getattr(L, "_uewald_sites_typed", False):
        for fn in (L.or_uewald_sites, L.or_uewald_sites_spm):
            fn.restype = C.c_int
            fn.argtypes = [C.c_int32, f64p, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                           f64p, f64p, C.c_int32, i32p, i32p, i32p, f64p, f64p, f64p]
        L._uewald_sites_typed = True
    r = np.ascontiguousarray(s["r"], np.float64)
    q = np.ascontiguousarray(az, np.float64)
    ipt = np.ascontiguousarray(s["iptpn"], np.int32)
    ian = np.ascontiguousarray(s["ianpn"], np.int32)
    napt = np.ascontiguousarray(s["napt"], np.int32)
    force = np.zeros((int(s["na"]), 3))
    urec = C.c_double()
    vir = C.c_double()
    box = (C.c_double * 3)(*s["boxlen"])
    fn, a1, a2 = (L.or_uewald_sites_spm, int(order), int(nmesh)) if nmesh else \
        (L.or_uewald_sites, int(ncut), 1 if region == "cube" else 0)
    rc = fn(int(s["na"]), box, float(ualpha), a1, a2, int(lsurf), float(s["epsi_four_pi"]), _p(r, C.c_double),
            _p(q, C.c_double), int(s["np"]), _p(ipt, C.c_int32), _p(ian, C.c_int32), _p(napt, C.c_int32),
            _p(force, C.c_double), C.byref(urec), C.byref(vir))
    if rc:
        raise RuntimeError("UEwald over sites failed: %d" % rc)
    return dict(force=force, urec=urec.value, virrec=vir.value)


def random_stream(iseed, n):
    """n successive Random(iseed) values from the first call (Src/mollib.F90:2689-2708)."""
    st = (C.c_int32 * 2)()
    lib().or_random_init(int(iseed), st)
    return np.array([lib().or_random_next(st) for _ in range(n)])


def gau_random_stream(iseed, n):
    """n successive GauRandom(iseed) values from a fresh SAVEd state."""
    s = C.c_int32(iseed)
    flag = C.c_int32(1)
    save = C.c_double(0.0)
    return np.array([lib().or_gau_random(C.byref(s), C.byref(flag), C.byref(save)) for _ in range(n)])
