"""Polyatomic particles: UTwoBodyP (Src/energy.F90:786-896), UEwald over the sites
(Src/energy.F90:905-1104, 1301-1371) and the rigid-body MD step (VelVer with lpolyatom,
Src/md.F90:252-410) on the GPU through the C-ABI (msg_utwobody_p, msg_uewald_sites,
msg_velver_p).  The caller's arrays follow MOLSIM's layout (see
systems.rigid_molecules); the atom-type table comes from engine.pot_tab."""
import ctypes as C

import numpy as np

from . import _lib
from .engine import MolsimGpuError


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def utwobody_p(s, table):
    """Site-site pair energy, forces and virial of polyatomic system s with its atom-type table.
    Returns dict(force [na][3], utwob [nptpt+1] = u%twob(0:nptpt), virial, kernel_ms)."""
    k = {}
    for key, dt in (("ro", np.float64), ("r", np.float64), ("iptpn", np.int32), ("ianpn", np.int32),
                    ("napt", np.int32), ("iatan", np.int32), ("nneighpn", np.int32), ("jpnlist", np.int32)):
        k[key] = np.ascontiguousarray(s[key], dt)
    k["ubuf"] = np.ascontiguousarray(table["ubuf"], np.float64)
    k["iubuflow"] = np.ascontiguousarray(table["iubuflow"], np.int32)
    k["r2umin"] = np.ascontiguousarray(table["r2umin"], np.float64)
    na, npt = int(s["na"]), int(s["npt"])
    force = np.zeros((na, 3))
    utwob = np.zeros(npt * (npt + 1) // 2 + 1)
    vir = C.c_double()
    ms = C.c_float()
    box = (C.c_double * 3)(*s["boxlen"])
    i32 = C.c_int32
    rc = _lib.lib().msg_utwobody_p(int(s["np"]), na, npt, int(s["nat"]), box, float(s["rcut"]),
                                   _p(k["ro"], C.c_double), _p(k["r"], C.c_double), _p(k["iptpn"], i32),
                                   _p(k["ianpn"], i32), _p(k["napt"], i32), _p(k["iatan"], i32),
                                   _p(k["nneighpn"], i32), _p(k["jpnlist"], i32), int(k["jpnlist"].shape[1]),
                                   _p(k["ubuf"], C.c_double), len(k["ubuf"]), _p(k["iubuflow"], i32),
                                   _p(k["r2umin"], C.c_double), _p(force, C.c_double), _p(utwob, C.c_double),
                                   C.byref(vir), C.byref(ms))
    if rc:
        raise MolsimGpuError(rc, "msg_utwobody_p")
    return dict(force=force, utwob=utwob, virial=vir.value, kernel_ms=ms.value)


def site_ewald_params(ewald, epsi_four_pi, az):
    """msg_site_ewald from dict(ualpha, lsurf and either ncut, region (standard Ewald) or
    order, nmesh (SPME)); az must stay alive while the struct is used."""
    spm = "nmesh" in ewald
    return _lib.MsgSiteEwald(1 if spm else 2, int(ewald.get("order", 0)), int(ewald.get("nmesh", 0)),
                             int(ewald.get("ncut", 0)), 1 if ewald.get("region", "sphere") == "cube" else 0,
                             int(bool(ewald.get("lsurf"))), float(ewald["ualpha"]), float(epsi_four_pi),
                             _p(az, C.c_double))


def velver_p(s, table, nsteps=1, ewald=None):
    """nsteps of the rigid-body MD step for a systems.rigid_bodies dict, its state (ro, rod,
    rodd, qua, quad, quadd, r) advanced in place.  ewald (optional): dict(az, ualpha, lsurf and
    either ncut, region (standard Ewald) or order, nmesh (SPME)) adds the site Ewald sum
    (msg_velver_p_ewald) to every step.  Returns dict(utwob, virial, kernel_ms[, urec]) of
    the last step."""
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
    ms = C.c_float()
    box = (C.c_double * 3)(*s["boxlen"])
    i32 = C.c_int32
    args = [int(nsteps), int(s["np"]), int(s["na"]), npt, int(s["nat"]), box, float(s["rcut"]),
            float(s["tstep"]), int(s["nvvite"]), float(s["tvvite"]),
            *[_p(k[x], C.c_double) for x in ("ro", "rod", "rodd", "qua", "quad", "quadd", "r")],
            *[_p(k[x], i32) for x in ("iptpn", "ianpn", "napt", "iatan")],
            _p(k["ra"], C.c_double), int(s["maxsite"]), _p(k["masspt"], C.c_double),
            _p(k["momp"], C.c_double), _p(k["nneighpn"], i32), _p(k["jpnlist"], i32),
            int(k["jpnlist"].shape[1]), _p(ub, C.c_double), len(ub), _p(iub, i32), _p(r2, C.c_double)]
    urec = C.c_double()
    if ewald is None:
        name = "msg_velver_p"
        rc = _lib.lib().msg_velver_p(*args, _p(utwob, C.c_double), C.byref(vir), C.byref(ms))
    else:
        name = "msg_velver_p_ewald"
        az = np.ascontiguousarray(ewald["az"], np.float64)
        if az.shape != (int(s["na"]),):
            raise ValueError("ewald['az'] must hold one charge per site")
        ep = site_ewald_params(ewald, s["epsi_four_pi"], az)
        rc = _lib.lib().msg_velver_p_ewald(*args, C.byref(ep), _p(utwob, C.c_double), C.byref(urec), C.byref(vir),
                                           C.byref(ms))
    if rc:
        raise MolsimGpuError(rc, name)
    for key in ("ro", "rod", "rodd", "qua", "quad", "quadd", "r"):
        s[key] = k[key]
    out = dict(utwob=utwob, virial=vir.value, kernel_ms=ms.value)
    if ewald is not None:
        out["urec"] = urec.value
    return out


def uewald_sites(s, az, ualpha, ncut=None, region="sphere", lsurf=False, order=None, nmesh=None):
    """UEwald over the sites of polyatomic system s with site charges az [na]: the standard
    reciprocal sum with ncut (region 'sphere' or 'cube'; msg_uewald_sites) or SPME with order
    and nmesh (msg_uewald_sites_spm), the atomic and molecular self terms and, when lsurf,
    the surface term.  Returns dict(force [na][3], urec, virrec, kernel_ms), urec and virrec
    scaled by EpsiFourPi as UEwald does."""
    r = np.ascontiguousarray(s["r"], np.float64)
    q = np.ascontiguousarray(az, np.float64)
    ipt = np.ascontiguousarray(s["iptpn"], np.int32)
    ian = np.ascontiguousarray(s["ianpn"], np.int32)
    napt = np.ascontiguousarray(s["napt"], np.int32)
    na = int(s["na"])
    if q.shape != (na,):
        raise ValueError("az must hold one charge per site")
    force = np.zeros((na, 3))
    urec = C.c_double()
    vir = C.c_double()
    ms = C.c_float()
    box = (C.c_double * 3)(*s["boxlen"])
    i32 = C.c_int32
    if nmesh:
        name, fn, a1, a2 = "msg_uewald_sites_spm", _lib.lib().msg_uewald_sites_spm, int(order), int(nmesh)
    else:
        name, fn, a1, a2 = "msg_uewald_sites", _lib.lib().msg_uewald_sites, int(ncut), 1 if region == "cube" else 0
    rc = fn(na, box, float(ualpha), a1, a2, int(bool(lsurf)), float(s["epsi_four_pi"]), _p(r, C.c_double),
            _p(q, C.c_double), int(s["np"]), _p(ipt, i32), _p(ian, i32), _p(napt, i32), len(napt),
            _p(force, C.c_double), C.byref(urec), C.byref(vir), C.byref(ms))
    if rc:
        raise MolsimGpuError(rc, name)
    return dict(force=force, urec=urec.value, virrec=vir.value, kernel_ms=ms.value)
