"""Host-side mirror of MOLSIM's force/energy entry points over the C-ABI.

The class `Engine` holds one library handle (one or many systems) and exposes
the reference's routine names: `SetVList` (Src/nlist.F90:686), `UTotal`
(Src/energy.F90:280), `GetLinAcc` (Src/md.F90:601), `VelVer` (Src/md.F90:252,
with GetKinEnergy and NList after every step) and `BDStep` (Src/bd.F90:120,
followed by UTotal and NList).  Errors raise `MolsimGpuError` carrying the
status code of the Stop() site the reference would have hit.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import MsgEnergy, MsgParams, MsgTabParams, f64p, i32p


class MolsimGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (status %d): %s" % (_lib.STATUS.get(code, "error"), code, msg))
        self.code = code


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def rcut_to_alpha(uewaldtol, q2sum, epsi_four_pi, boxlenshort, rcut):
    """RcutToAlpha (Src/energy.F90:7090-7105)."""
    st = C.c_int32()
    a = _lib.lib().msg_rcut_to_alpha(uewaldtol, q2sum, epsi_four_pi, boxlenshort, rcut, C.byref(st))
    if st.value:
        raise MolsimGpuError(st.value, "RcutToAlpha did not converge")
    return a


def alpha_to_ncut(uewaldtol, q2sum, epsi_four_pi, boxlenshort, ualpha):
    """AlphaToNcut (Src/energy.F90:7066-7081): the standard Ewald k-space cut."""
    st = C.c_int32()
    n = _lib.lib().msg_alpha_to_ncut(uewaldtol, q2sum, epsi_four_pi, boxlenshort, ualpha, C.byref(st))
    if st.value:
        raise MolsimGpuError(st.value, "AlphaToNcut did not converge")
    return int(n)


def ewald_mode(sysd):
    """msg_params.lewald: 0 no Ewald sum, 1 SPME (txewaldrec 'spm', the default),
    2 standard Ewald (txewaldrec 'std')."""
    if not sysd["lewald"]:
        return 0
    rec = sysd.get("ewaldrec", "spm")
    if rec not in ("spm", "std"):
        raise ValueError("ewaldrec must be 'spm' or 'std'")
    return 2 if rec == "std" else 1


def pot_tab(sysd, ualpha, nbuf=100000):
    """MOLSIM's pair table (PotTwoBodyTab1/2/3, Src/potential.F90:868-1135) for the (1,6,12)
    potential of the system's types."""
    npt = int(sysd["npt"])
    natat = npt * (npt + 1) // 2
    keep = [np.ascontiguousarray(sysd[k], np.float64) for k in ("zat", "sigat", "epsat")]
    tp = MsgTabParams(npt, _p(keep[0], C.c_double), _p(keep[1], C.c_double), _p(keep[2], C.c_double),
                      sysd["rcut"], ualpha, sysd["epsi_four_pi"], int(sysd["lewald"]), int(sysd["lljcut"]),
                      sysd["ljrcut"], sysd["ljushift"], sysd["r2uminin"], sysd["utoltab"], sysd["ftoltab"],
                      sysd["umaxtab"], sysd["fmaxtab"], sysd["rumaxfac"])
    ubuf = np.zeros(nbuf)
    iub = np.zeros(natat, np.int32)
    nug = np.zeros(natat, np.int32)
    r2umin = np.zeros(natat)
    nused = C.c_int32()
    rc = _lib.lib().msg_pot_tab(C.byref(tp), _p(ubuf, C.c_double), nbuf, _p(iub, C.c_int32), _p(nug, C.c_int32),
                                _p(r2umin, C.c_double), C.byref(nused))
    if rc:
        raise MolsimGpuError(rc, "msg_pot_tab")
    return dict(ubuf=ubuf[:nused.value].copy(), iubuflow=iub, nugrid=nug, r2umin=r2umin)


def prepare(sysd):
    """Derive alpha (IOPotTwoBody -> EwaldSetup, iewaldopt=3) and the pair table."""
    q2sum = float(np.mean(np.asarray(sysd["az"], np.float64) ** 2))
    alpha = rcut_to_alpha(sysd["uewaldtol"], q2sum, sysd["epsi_four_pi"], min(sysd["boxlen"]), sysd["rcut"]) \
        if sysd["lewald"] else 0.0
    tab = pot_tab(sysd, alpha)
    natat = sysd["npt"] * (sysd["npt"] + 1) // 2
    tab["r2atat"] = np.zeros(natat)
    tab["ualpha"] = alpha
    if ewald_mode(sysd) == 2:
        # EwaldSetup iewaldopt=3: ncut from alpha unless the system fixes it
        tab["ncut"] = int(sysd.get("ncut") or alpha_to_ncut(sysd["uewaldtol"], q2sum, sysd["epsi_four_pi"],
                                                            min(sysd["boxlen"]), alpha))
    return tab


def params_array(systems, tables, maxnneigh=0):
    """msg_params for the systems (and the arrays they point into, which must outlive the call)."""
    keep = []
    arr = (MsgParams * len(systems))()
    for k, (s, t) in enumerate(zip(systems, tables)):
        arr[k] = Engine._params_for(s, t, maxnneigh, keep)
    return arr, keep


def estimate_bytes(systems, tables, precision="mixed"):
    """Device bytes a handle for these systems would hold (msg_estimate_bytes)."""
    if isinstance(systems, dict):
        systems, tables = [systems], [tables]
    arr, _keep = params_array(systems, tables)
    out = C.c_int64()
    prec = _lib.MSG_PREC_MIXED if precision == "mixed" else _lib.MSG_PREC_FP64
    rc = _lib.lib().msg_estimate_bytes(arr, len(systems), prec, C.byref(out))
    if rc:
        raise MolsimGpuError(rc, "msg_estimate_bytes")
    return int(out.value)


class Engine:
    """One library handle for `systems` (a list of system dicts, see systems.py) with their
    tables (`tables[k]` from `prepare` or from a caller such as the oracle)."""

    def __init__(self, systems, tables=None, precision="fp64", maxnneigh=0):
        if isinstance(systems, dict):
            systems = [systems]
        if tables is None:
            tables = [prepare(s) for s in systems]
        elif isinstance(tables, dict):
            tables = [tables]
        self.systems = systems
        self.tables = tables
        self.nsys = len(systems)
        self.natat = [s["npt"] * (s["npt"] + 1) // 2 for s in systems]
        self._keep = []
        arr = (MsgParams * self.nsys)()
        for k, (s, t) in enumerate(zip(systems, tables)):
            arr[k] = self._params(s, t, maxnneigh)
        prec = _lib.MSG_PREC_MIXED if precision == "mixed" else _lib.MSG_PREC_FP64
        h = C.c_void_p()
        L = _lib.lib()
        rc = L.msg_create_batch(arr, self.nsys, prec, C.byref(h)) if self.nsys > 1 else \
            L.msg_create(arr, prec, C.byref(h))
        if rc:
            raise MolsimGpuError(rc, "msg_create failed")
        self.h = h
        self.reset_states()

    def reset_states(self):
        """Every system back to the state its dict holds (ro, rod, rodd; the last two may be
        absent): one call, one list rebuild, one device wait."""
        systems = self.systems
        if self.nsys == 1:
            self.set_state(0, systems[0]["ro"], systems[0].get("rod"), systems[0].get("rodd"))
            return
        cat = []
        for key in ("ro", "rod", "rodd"):
            parts = [s.get(key) for s in systems]
            cat.append(None if any(x is None for x in parts) else
                       np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64).reshape(-1, 3)
                                                            for x in parts]), np.float64))
        ptrs = [None if a is None else _p(a, C.c_double) for a in cat]
        self._check(_lib.lib().msg_set_state_all(self.h, *ptrs))

    def _params(self, s, t, maxnneigh):
        return Engine._params_for(s, t, maxnneigh, self._keep)

    @staticmethod
    def _params_for(s, t, maxnneigh, keep):
        k = {}
        k["iptpn"] = np.ascontiguousarray(s["iptpn"], np.int32)
        k["az"] = np.ascontiguousarray(s["az"], np.float64)
        k["masspt"] = np.ascontiguousarray(s["masspt"], np.float64)
        k["ubuf"] = np.ascontiguousarray(t["ubuf"], np.float64)
        k["iubuflow"] = np.ascontiguousarray(t["iubuflow"], np.int32)
        k["r2umin"] = np.ascontiguousarray(t["r2umin"], np.float64)
        k["r2atat"] = np.ascontiguousarray(t.get("r2atat", np.zeros(len(t["r2umin"]))), np.float64)
        k["bond_ij"] = np.ascontiguousarray(s.get("bond_ij", np.zeros((0, 2))), np.int32).reshape(-1)
        k["bond_k"] = np.ascontiguousarray(s.get("bond_k", np.zeros(0)), np.float64)
        k["bond_eq"] = np.ascontiguousarray(s.get("bond_eq", np.zeros(0)), np.float64)
        k["bond_p"] = np.ascontiguousarray(s.get("bond_p", np.zeros(0)), np.int32)
        fac = s.get("bd_fac")
        if fac is not None:
            k["fac1"] = np.ascontiguousarray(fac[0], np.float64)
            k["fac2"] = np.ascontiguousarray(fac[1], np.float64)
        keep.append(k)
        null = C.POINTER(C.c_double)()
        return MsgParams(int(s["np"]), int(s["npt"]), (C.c_double * 3)(*s["boxlen"]), s["rcut"], s["drnlist"],
                         _p(k["iptpn"], C.c_int32), _p(k["az"], C.c_double), _p(k["masspt"], C.c_double),
                         _p(k["ubuf"], C.c_double), len(k["ubuf"]), _p(k["iubuflow"], C.c_int32),
                         _p(k["r2umin"], C.c_double), _p(k["r2atat"], C.c_double), ewald_mode(s),
                         int(s["order"]), int(s["nmesh"]), int(s["lsurf"]), t["ualpha"] if "ualpha" in t else s["ualpha"],
                         s["epsi_four_pi"], len(k["bond_p"]), _p(k["bond_ij"], C.c_int32),
                         _p(k["bond_k"], C.c_double), _p(k["bond_eq"], C.c_double), _p(k["bond_p"], C.c_int32),
                         s["tstep"], _p(k["fac1"], C.c_double) if "fac1" in k else null,
                         _p(k["fac2"], C.c_double) if "fac2" in k else null, int(maxnneigh),
                         int(t.get("ncut", s.get("ncut", 0)) or 0),
                         1 if s.get("ncutregion", "sphere") == "cube" else 0,
                         int(bool(s.get("lewald2dlc", False))), int(s.get("inlist", 0)),
                         int(bool(s.get("lvlistllist", False))))

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().msg_destroy(h)
            except TypeError:           # interpreter shutdown: the module globals are gone
                pass
            self.h = None

    def _check(self, rc):
        if rc:
            raise MolsimGpuError(rc, _lib.lib().msg_last_error(self.h).decode())

    # --- state -------------------------------------------------------------
    def set_state(self, isys, ro, rod=None, rodd=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (ro, rod, rodd)]
        ptrs = [None if a is None else _p(a, C.c_double) for a in arrs]
        self._check(_lib.lib().msg_set_state(self.h, isys, *ptrs))

    def get_state(self, isys=0):
        n = int(self.systems[isys]["np"])
        out = [np.zeros((n, 3)) for _ in range(3)]
        self._check(_lib.lib().msg_get_state(self.h, isys, *[_p(a, C.c_double) for a in out]))
        return dict(ro=out[0], rod=out[1], rodd=out[2])

    # --- MOLSIM entry points --------------------------------------------------
    def SetVList(self, isys=0, export=True, maxnneigh=None):
        """Rebuild now; return (nneighpn, jpnlist, npair) in MOLSIM's layout (1-based)."""
        n = int(self.systems[isys]["np"])
        npair = C.c_int64()
        if not export:
            self._check(_lib.lib().msg_build_nlist(self.h, isys, None, None, 0, C.byref(npair)))
            return None, None, npair.value
        maxn = int(maxnneigh or n)
        nn = np.zeros(n, np.int32)
        jp = np.zeros((n, maxn), np.int32)
        self._check(_lib.lib().msg_build_nlist(self.h, isys, _p(nn, C.c_int32), _p(jp, C.c_int32), maxn,
                                               C.byref(npair)))
        return nn, jp, npair.value

    def UTotal(self, isys=0):
        n = int(self.systems[isys]["np"])
        f = np.zeros((n, 3))
        fo = np.zeros((n, 3))
        e = MsgEnergy()
        self._check(_lib.lib().msg_utotal(self.h, isys, _p(f, C.c_double), _p(fo, C.c_double), C.byref(e)))
        d = e.as_dict(self.natat[isys])
        d["force"] = f
        d["forceo"] = fo
        return d

    def forces(self, isys=0):
        """(force, forceo) of system isys from the last force evaluation, no recomputation."""
        n = int(self.systems[isys]["np"])
        f = np.zeros((n, 3))
        fo = np.zeros((n, 3))
        self._check(_lib.lib().msg_get_forces(self.h, isys, _p(f, C.c_double), _p(fo, C.c_double)))
        return f, fo

    def tune(self, key, value):
        """msg_tune: one scheduling knob (MSG_TUNE_*) of this handle."""
        self._check(_lib.lib().msg_tune(self.h, int(key), int(value)))

    def tune_pair_lanes(self, shift):
        """Lanes per particle in the pair kernel scaled by 2**shift (results move by rounding only)."""
        self._check(_lib.lib().msg_tune(self.h, _lib.MSG_TUNE_PAIR_LANES, int(shift)))

    def tune_pair_kernel(self, kind):
        """Pair kernel of a mixed-precision handle: 2 the half-list kernel (default: each pair
        stored and evaluated once, partner forces as fixed-point atomics), 1 the full-list lean
        kernel, 0 the generic full-list kernel.  Switching list layouts rebuilds the lists."""
        self._check(_lib.lib().msg_tune(self.h, _lib.MSG_TUNE_PAIR_KERNEL, int(kind)))

    def GetLinAcc(self):
        self._check(_lib.lib().msg_get_linacc(self.h))

    def VelVer(self, nsteps=1, isys=0, energies=True):
        """nsteps of MDDriver(iSimulationStep) + NList for every system; energies of system isys."""
        if not energies:
            self._check(_lib.lib().msg_velver(self.h, nsteps, isys, None))
            return None
        e = (MsgEnergy * max(1, nsteps))()
        self._check(_lib.lib().msg_velver(self.h, nsteps, isys, e))
        return [e[k].as_dict(self.natat[isys]) for k in range(nsteps)]

    def mc_seed(self, iseed, isys=0):
        """Random's state of system isys from iseed (MOLSIM's iseed)."""
        self._check(_lib.lib().msg_mc_seed(self.h, isys, int(iseed)))

    def MCPass(self, npass=1, dtran=None, beta=None, isamp=0, isys=0):
        """npass MCPass sweeps of single-particle translations (Src/mc.F90:1470-1755) for every
        system.  dtran: per-type displacements ([npt], or one list per system); beta: 1/kT in
        mol/kJ (one value or one per system; default from each system's temperature).
        Returns (accepted[nsys], hard-core rejects[nsys], energies of system isys)."""
        from ._lib import MsgMcParams
        from .systems import kT

        par = (MsgMcParams * self.nsys)()
        keep = []
        for k, s in enumerate(self.systems):
            d = dtran[k] if dtran is not None and np.ndim(dtran) == 2 else dtran
            d = np.ascontiguousarray(d if d is not None else [1.0] * s["npt"], np.float64)
            keep.append(d)
            b = beta[k] if isinstance(beta, (list, tuple, np.ndarray)) else beta
            b = float(b) if b is not None else 1.0 / kT(s["temp"])
            par[k] = MsgMcParams(b, _p(d, C.c_double), int(isamp), 0)
        acc = np.zeros(self.nsys, np.int64)
        hs = np.zeros(self.nsys, np.int64)
        e = MsgEnergy()
        self._check(_lib.lib().msg_mc_pass(self.h, int(npass), par, _p(acc, C.c_int64), _p(hs, C.c_int64), isys,
                                           C.byref(e)))
        return acc, hs, e.as_dict(self.natat[isys])

    def MCAllPass(self, npass=1, dtranall=None, beta=None, isys=0):
        """npass MCAllPass trials (Src/mc.F90:4024-4178) for every system: all particles displaced
        at once, UTotal, Metropolis.  dtranall: per-type displacements ([npt], or one list per
        system); beta as in MCPass.  Returns (accepted[nsys], energies of system isys)."""
        from ._lib import MsgMcAllParams
        from .systems import kT

        par = (MsgMcAllParams * self.nsys)()
        keep = []
        for k, s in enumerate(self.systems):
            d = dtranall[k] if dtranall is not None and np.ndim(dtranall) == 2 else dtranall
            d = np.ascontiguousarray(d if d is not None else [0.1] * s["npt"], np.float64)
            keep.append(d)
            b = beta[k] if isinstance(beta, (list, tuple, np.ndarray)) else beta
            b = float(b) if b is not None else 1.0 / kT(s["temp"])
            par[k] = MsgMcAllParams(b, _p(d, C.c_double))
        acc = np.zeros(self.nsys, np.int64)
        e = MsgEnergy()
        self._check(_lib.lib().msg_mcall_pass(self.h, int(npass), par, _p(acc, C.c_int64), isys, C.byref(e)))
        return acc, e.as_dict(self.natat[isys])

    def BDStep(self, nsteps=1, seed=0, isys=0, xi=None, return_noise=False, energies=True):
        """nsteps of BDDriver(iSimulationStep) + NList.  xi: caller noise [nsteps][np][3]."""
        n = int(self.systems[isys]["np"])
        xin = None if xi is None else np.ascontiguousarray(xi, np.float64).reshape(nsteps, n, 3)
        xout = np.zeros((nsteps, n, 3)) if return_noise else None
        e = (MsgEnergy * max(1, nsteps))() if energies else None
        self._check(_lib.lib().msg_bd_step(self.h, nsteps, seed, isys,
                                           None if xin is None else _p(xin, C.c_double),
                                           None if xout is None else _p(xout, C.c_double), e))
        en = [e[k].as_dict(self.natat[isys]) for k in range(nsteps)] if energies else None
        return (en, xout) if return_noise else en

    def VelVerHost(self, state, nsteps=1, isys=0, energies=True):
        """nsteps of MDDriver with host-held state: state = dict(ro, rod, rodd) ([np][3]
        float64 arrays, continuing the device's trajectory) is sent, stepped and overwritten
        with the new state, in one call (msg_velver_host)."""
        arrs = [np.ascontiguousarray(state[k], np.float64) for k in ("ro", "rod", "rodd")]
        e = (MsgEnergy * max(1, nsteps))() if energies else None
        self._check(_lib.lib().msg_velver_host(self.h, isys, nsteps, *[_p(a, C.c_double) for a in arrs], e))
        for k, a in zip(("ro", "rod", "rodd"), arrs):
            state[k] = a
        return [e[k].as_dict(self.natat[isys]) for k in range(nsteps)] if energies else None

    def nlist_before_macrostep(self):
        """NList(iBeforeMacrostep) for every system: drosum = 0, istep2 restarts."""
        self._check(_lib.lib().msg_nlist_before_macrostep(self.h))

    def nrebuild(self, isys=0):
        return _lib.lib().msg_nrebuild(self.h, isys)

    def put_state(self, isys, ro, rod=None, rodd=None, keep_list=True):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (ro, rod, rodd)]
        ptrs = [None if a is None else _p(a, C.c_double) for a in arrs]
        self._check(_lib.lib().msg_put_state(self.h, isys, *ptrs, 1 if keep_list else 0))

    # --- serving support -----------------------------------------------------
    def velver_async(self, nsteps):
        """Enqueue nsteps MD steps of every system and return at once."""
        self._check(_lib.lib().msg_velver_async(self.h, nsteps))

    def pending(self):
        """Asynchronous step batches still on the device; raises on a device error."""
        r = _lib.lib().msg_pending(self.h)
        if r < 0:
            raise MolsimGpuError(-r, _lib.lib().msg_last_error(self.h).decode())
        return r

    def energy(self, isys=0):
        e = MsgEnergy()
        self._check(_lib.lib().msg_get_energy(self.h, isys, C.byref(e)))
        return e.as_dict(self.natat[isys])

    def device_bytes(self):
        return int(_lib.lib().msg_device_bytes(self.h))

    # --- instrumentation ---------------------------------------------------
    def stream(self):
        return _lib.lib().msg_stream(self.h)

    def launch_count(self):
        return _lib.lib().msg_launch_count(self.h)

    def set_timing(self, on=True):
        self._check(_lib.lib().msg_set_timing(self.h, 1 if on else 0))

    def kernel_times(self):
        """{timer name: (total device ms, launches)} since the last set_timing."""
        L = _lib.lib()
        out = {}
        for k in range(L.msg_ntimers()):
            name = C.c_char_p()
            ms = C.c_double()
            n = C.c_int64()
            self._check(L.msg_kernel_time(self.h, k, C.byref(name), C.byref(ms), C.byref(n)))
            out[name.value.decode()] = (ms.value, n.value)
        return out
