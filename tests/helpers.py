"""Shared helpers of the tests: systems with their tables, and comparison metrics."""
import functools

import numpy as np

import pyoracle as O
from molsim_b200 import systems as S


def oracle_table(s):
    """Alpha and pair table from the oracle (RcutToAlpha + PotTwoBodyTab1)."""
    q2 = float(np.mean(np.asarray(s["az"]) ** 2))
    alpha = O.rcut_to_alpha(s["uewaldtol"], q2, s["epsi_four_pi"], min(s["boxlen"]), s["rcut"]) \
        if s["lewald"] else 0.0
    pot = dict(npt=s["npt"], zat=s["zat"], sigat=s["sigat"], epsat=s["epsat"], rcut=s["rcut"], ualpha=alpha,
               epsi_four_pi=s["epsi_four_pi"], lewald=int(s["lewald"]), lljcut=int(s["lljcut"]),
               **{k: s[k] for k in ("ljrcut", "ljushift", "r2uminin", "utoltab", "ftoltab", "umaxtab",
                                    "fmaxtab", "rumaxfac")})
    t = O.pot_tab(pot)
    t["ualpha"] = alpha
    t["r2atat"] = np.zeros(len(t["r2umin"]))
    if s["lewald"] and s.get("ewaldrec", "spm") == "std":
        # EwaldSetup iewaldopt=3: ncut from alpha (AlphaToNcut) unless the system fixes it
        t["ncut"] = int(s.get("ncut") or O.alpha_to_ncut(s["uewaldtol"], q2, s["epsi_four_pi"],
                                                         min(s["boxlen"]), alpha))
    return t


def std_ewald(s, ncut=None, region="sphere"):
    """The same system with standard Ewald (txewaldrec 'std') in reciprocal space."""
    d = dict(s)
    d["ewaldrec"] = "std"
    d["ncutregion"] = region
    if ncut:
        d["ncut"] = int(ncut)
    return d


def oracle_system(s, t, cell=False, maxnneigh=None):
    d = dict(s)
    d["ualpha"] = t["ualpha"]
    if "ncut" in t:
        d["ncut"] = t["ncut"]
    return O.System(d, t, maxnneigh=maxnneigh or s["np"], lcellbuild=cell)


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@functools.lru_cache(maxsize=None)
def electrolyte_small(n_pairs=64, L=40.0, seed=1, lsurf=False):
    s = S.electrolyte(seed=seed, n_pairs=n_pairs, L=L, rcut=min(18.0, L / 2 - 2.0), nmesh=16)
    s["lsurf"] = lsurf
    return s


@functools.lru_cache(maxsize=None)
def config0():
    return S.electrolyte(0)


@functools.lru_cache(maxsize=None)
def config1():
    return S.polyelectrolyte(0)


@functools.lru_cache(maxsize=None)
def pe_small():
    return S.polyelectrolyte(seed=3, nchain=4, nbead=50, L=80.0, rcut=20.0, nmesh=32, order=5)


@functools.lru_cache(maxsize=None)
def colloid_small():
    s = S.colloid_bd(seed=2, n_macro=8, n_salt_pairs=400, L=200.0, nmesh=32)
    s["bd_fac"] = S.bd_factors(s)
    return s


@functools.lru_cache(maxsize=None)
def config2():
    """200,000-particle charged-colloid BD system (2000 macroions +20e, 40000 counterions,
    79000 salt pairs, L = 1200 A, SPME 128^3 order 4, rc = 30 A)."""
    s = S.colloid_bd(seed=0)
    s["bd_fac"] = S.bd_factors(s)
    return s


def site_table(s):
    """The atom-type (site-site) table of a polyatomic system from the oracle."""
    d = S.site_table_params(s)
    pot = dict(npt=d["npt"], zat=d["zat"], sigat=d["sigat"], epsat=d["epsat"], rcut=d["rcut"], ualpha=0.0,
               epsi_four_pi=d["epsi_four_pi"], lewald=0, lljcut=int(d["lljcut"]),
               **{k: d[k] for k in ("ljrcut", "ljushift", "r2uminin", "utoltab", "ftoltab", "umaxtab",
                                    "fmaxtab", "rumaxfac")})
    return O.pot_tab(pot)


@functools.lru_cache(maxsize=None)
def rigid_small():
    return S.rigid_molecules(seed=2, nmol=150, nsolute=60, L=30.0, rcut=10.0)


def slab_small(Lz=120.0, seed=3, lsurf=True, ncut=12, region="sphere", elc=True):
    """The small electrolyte as a slab: its ions placed in |z| < 10 A (at least 4 A apart) of
    a 40 x 40 x Lz box, standard Ewald with ncut, the 2D layer correction (lewald2dlc) on."""
    rng = np.random.default_rng(seed)
    s = dict(electrolyte_small(lsurf=lsurf))
    n = s["np"]
    pts = []
    while len(pts) < n:
        x = np.array([rng.uniform(-20, 20), rng.uniform(-20, 20), rng.uniform(-10, 10)])
        if all(np.sum(((x - p + 20) % 40 - 20)[:2] ** 2) + (x - p)[2] ** 2 > 16.0 for p in pts):
            pts.append(x)
    s["boxlen"] = np.array([40.0, 40.0, float(Lz)])
    s["ro"] = np.array(pts)
    s["rod"] = np.zeros((n, 3))
    d = std_ewald(s, ncut=ncut, region=region)
    d["lewald2dlc"] = bool(elc)
    return d
