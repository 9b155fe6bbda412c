"""Seeded synthetic systems for the force/energy path.

Each generator returns a plain dict describing one monoatomic charged system in
MOLSIM's units (A, g/mol, ps, kJ/mol, K; Src/molsim.F90:786-805):

    np, npt, boxlen[3], rcut, drnlist, iptpn[np] (1-based), az[np], masspt[npt],
    zat/sigat/epsat[npt], temp, relpermitt, epsi_four_pi, uewaldtol, order, nmesh,
    lewald, lsurf, tstep, bonds (bond_ij[nb][2] 1-based, bond_k (already divided by
    the power, Src/potential.F90:3561), bond_eq, bond_p), ro[np][3], rod[np][3].

The Ewald alpha and the pair table are derived from these by the library's own
setup routines (`molsim_b200.setup`), exactly as MOLSIM derives them in
IOPotTwoBody/EwaldSetup/PotTwoBodyTab1 from its namelists.
"""
import math

import numpy as np

# Src/mol.F90:60-80 and Src/molsim.F90:786-805
PI = 3.1415926535897932
AVNO = 6.02214179e23
ECH = 1.602176487e-19
GAS_CONSTANT = 8.314472
EPSI0 = 8.854187817e-12
SCLLEN, SCLMAS, SCLTIM, SCLENE, SCLDIF = 1.0e-10, 1.0e-03, 1.0e-12, 1.0e+03, 1.0e-09
SCLVEL = SCLLEN / SCLTIM
SCLFOR = SCLVEL / SCLTIM * SCLMAS
EPSI0_FOUR_PI = ECH ** 2 / (4.0 * PI * EPSI0 * SCLLEN) * AVNO / SCLENE

# nmlPotential defaults, Src/potential.F90:340-367.  utoltab/ftoltab and the
# exponent of ljrcut are single-precision literals in the reference.
F32_1EM5 = float(np.float32(1e-5))
POT_DEFAULTS = dict(r2uminin=0.1, utoltab=F32_1EM5, ftoltab=F32_1EM5, umaxtab=20000.0,
                    fmaxtab=20000.0, ljrcut=2.0 ** float(np.float32(1.0) / np.float32(6.0)),
                    ljushift=1.0, rumaxfac=1.1)


def kT(temp):
    """k_B T in kJ/mol."""
    return GAS_CONSTANT * temp / 1000.0


def _min_image(d, box):
    return d - box * np.round(d / box)


def place_uniform(rng, n, box, mind, existing=None, exist_mind=None, batch=4096):
    """Uniform positions in [-L/2, L/2)^3 with no pair closer than `mind` (and no
    point closer than `exist_mind` to an `existing` point), by seeded rejection."""
    from scipy.spatial import cKDTree

    L = float(box)
    pts = np.zeros((0, 3))
    ex_tree = None
    if existing is not None and len(existing):
        ex_tree = cKDTree(np.mod(existing + L / 2, L), boxsize=L)
    while len(pts) < n:
        cand = rng.uniform(-L / 2, L / 2, size=(batch, 3))
        cw = np.mod(cand + L / 2, L)
        ok = np.ones(len(cand), bool)
        if ex_tree is not None:
            d, _ = ex_tree.query(cw, k=1)
            ok &= d >= exist_mind
        if len(pts):
            t = cKDTree(np.mod(pts + L / 2, L), boxsize=L)
            d, _ = t.query(cw, k=1)
            ok &= d >= mind
        cand, cw = cand[ok], cw[ok]
        if len(cand) > 1:
            t = cKDTree(cw, boxsize=L)
            pairs = t.query_pairs(mind, output_type="ndarray")
            if len(pairs):
                drop = np.zeros(len(cand), bool)
                for a, b in pairs:          # keep the earlier candidate of each close pair
                    if not drop[a]:
                        drop[b] = True
                cand = cand[~drop]
        pts = np.concatenate([pts, cand[: n - len(pts)]])
    return pts


def maxwell_velocities(rng, masses, temp):
    """SetLinVel, Src/md.F90:802-822: v = sqrt(R T/(m sclmas sclvel^2)) * N(0,1)."""
    fac = GAS_CONSTANT * temp / (SCLMAS * SCLVEL ** 2)
    return rng.standard_normal((len(masses), 3)) * np.sqrt(fac / masses)[:, None]


def _base(np_, npt, L, rcut, temp, relp, order, nmesh, tstep, drnlist=2.0, lsurf=False):
    return dict(np=int(np_), npt=int(npt), boxlen=[float(L)] * 3, rcut=float(rcut),
                drnlist=float(drnlist), temp=float(temp), relpermitt=float(relp),
                epsi_four_pi=EPSI0_FOUR_PI / relp, uewaldtol=1e-5, order=int(order),
                nmesh=int(nmesh), lewald=True, lsurf=bool(lsurf), lljcut=True, tstep=float(tstep),
                nbond=0, bond_ij=np.zeros((0, 2), np.int32), bond_k=np.zeros(0),
                bond_eq=np.zeros(0), bond_p=np.zeros(0, np.int32), **POT_DEFAULTS)


def electrolyte(seed=0, n_pairs=500, L=100.0, temp=298.0, relp=78.4, sigma=4.0, mass=23.0,
                rcut=30.0, nmesh=32, order=4, tstep=0.005, eps_kT=0.1):
    """1:1 primitive-model electrolyte (500 + 500 ions, L=100 A, SPME 32^3 order 4, rc=30 A)."""
    rng = np.random.default_rng(seed)
    n = 2 * n_pairs
    s = _base(n, 2, L, rcut, temp, relp, order, nmesh, tstep)
    s["zat"] = np.array([1.0, -1.0])
    s["sigat"] = np.array([sigma, sigma])
    s["epsat"] = np.array([eps_kT * kT(temp)] * 2)
    s["masspt"] = np.array([mass, mass])
    s["iptpn"] = np.array([1] * n_pairs + [2] * n_pairs, np.int32)
    s["az"] = s["zat"][s["iptpn"] - 1].copy()
    s["ro"] = place_uniform(rng, n, L, 0.8 * sigma)
    s["rod"] = maxwell_velocities(rng, s["masspt"][s["iptpn"] - 1], temp)
    s["name"] = "electrolyte_%d" % n
    return s


def polyelectrolyte(seed=0, nchain=40, nbead=200, L=250.0, temp=298.0, relp=78.4, sigma=4.0,
                    mass=23.0, rcut=25.0, nmesh=64, order=5, tstep=0.005, bond_kT=0.4, r0=5.0,
                    eps_kT=0.1):
    """40 chains x 200 beads (-1e) + 8000 counterions (+1e), L=250 A, SPME 64^3 order 5, rc=25 A.
    Chains are random walks with 5 A steps rejecting overlaps below 0.8 sigma."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    nb = nchain * nbead
    n = 2 * nb
    s = _base(n, 2, L, rcut, temp, relp, order, nmesh, tstep)
    s["zat"] = np.array([-1.0, 1.0])
    s["sigat"] = np.array([sigma, sigma])
    s["epsat"] = np.array([eps_kT * kT(temp)] * 2)
    s["masspt"] = np.array([mass, mass])
    s["iptpn"] = np.array([1] * nb + [2] * nb, np.int32)
    s["az"] = s["zat"][s["iptpn"] - 1].copy()
    mind = 0.8 * sigma
    beads = []
    for c in range(nchain):
        for _attempt in range(1000):
            chain = [rng.uniform(-L / 2, L / 2, 3)]
            ok = True
            prev = np.array(beads) if beads else None
            tree = cKDTree(np.mod(prev + L / 2, L), boxsize=L) if prev is not None else None
            if tree is not None and tree.query(np.mod(chain[0] + L / 2, L))[0] < mind:
                continue                 # the chain's first bead overlaps an earlier chain
            while len(chain) < nbead and ok:
                for _t in range(200):
                    v = rng.standard_normal(3)
                    p = chain[-1] + r0 * v / np.linalg.norm(v)
                    p = _min_image(p, L)
                    d_own = np.linalg.norm(_min_image(np.array(chain[:-1]) - p, L), axis=1) if len(chain) > 1 else np.array([1e9])
                    if d_own.min() < mind:
                        continue
                    if tree is not None and tree.query(np.mod(p + L / 2, L))[0] < mind:
                        continue
                    chain.append(p)
                    break
                else:
                    ok = False
            if ok:
                beads.extend(chain)
                break
        else:
            raise RuntimeError("could not grow chain %d" % c)
    beads = np.array(beads)
    ions = place_uniform(rng, nb, L, mind, existing=beads, exist_mind=mind)
    s["ro"] = np.concatenate([beads, ions])
    s["rod"] = maxwell_velocities(rng, s["masspt"][s["iptpn"] - 1], temp)
    bij = []
    for c in range(nchain):
        for k in range(nbead - 1):
            bij.append((c * nbead + k + 1, c * nbead + k + 2))
    s["bond_ij"] = np.array(bij, np.int32)
    s["nbond"] = len(bij)
    s["bond_p"] = np.full(len(bij), 2, np.int32)
    s["bond_k"] = np.full(len(bij), bond_kT * kT(temp) / 2.0)   # k/p, Src/potential.F90:3561
    s["bond_eq"] = np.full(len(bij), r0)
    s["name"] = "polyelectrolyte_%d" % n
    return s


def colloid_bd(seed=0, n_macro=2000, z_macro=20.0, sigma_macro=40.0, n_salt_pairs=79000,
               L=1200.0, temp=298.0, relp=78.4, sigma=4.0, rcut=30.0, nmesh=128, order=4,
               tstep=1e-3, d_ion=1.0, d_macro=0.1, mass_ion=23.0, mass_macro=1.0e5, eps_kT=0.1):
    """Charged colloids for Brownian dynamics: 2000 macroions (+20e, sigma 40 A), 40000
    counterions (-1e) and 79000+79000 salt ions (sigma 4 A) in L=1200 A; SPME 128^3 order 4.
    Types: 1 macroion, 2 anion (counterion and salt anion), 3 cation.  dcoeff in units of
    1e-9 m^2/s (scldif)."""
    rng = np.random.default_rng(seed)
    n_ci = int(round(n_macro * z_macro))
    n_an = n_ci + n_salt_pairs
    n_cat = n_salt_pairs
    n = n_macro + n_an + n_cat
    s = _base(n, 3, L, rcut, temp, relp, order, nmesh, tstep)
    s["zat"] = np.array([z_macro, -1.0, 1.0])
    s["sigat"] = np.array([sigma_macro, sigma, sigma])
    s["epsat"] = np.array([eps_kT * kT(temp)] * 3)
    s["masspt"] = np.array([mass_macro, mass_ion, mass_ion])
    s["dcoeff"] = np.array([d_macro, d_ion, d_ion])
    s["iptpn"] = np.array([1] * n_macro + [2] * n_an + [3] * n_cat, np.int32)
    s["az"] = s["zat"][s["iptpn"] - 1].copy()
    macro = place_uniform(rng, n_macro, L, sigma_macro)
    ions = place_uniform(rng, n_an + n_cat, L, 0.8 * sigma, existing=macro,
                         exist_mind=0.5 * (sigma_macro + sigma), batch=32768)
    s["ro"] = np.concatenate([macro, ions])
    s["rod"] = np.zeros((n, 3))
    s["name"] = "colloid_bd_%d" % n
    return s


def bd_factors(s):
    """fac1/fac2 of BDStep, Src/bd.F90:135-140, per particle type."""
    dt, T, D = s["tstep"], s["temp"], np.asarray(s["dcoeff"], np.float64)
    fac1 = dt * SCLTIM * D * SCLDIF * SCLFOR / (GAS_CONSTANT * T * 1.0) / SCLLEN
    fac2 = np.sqrt(2.0 * D * SCLDIF * dt * SCLTIM) / SCLLEN
    return fac1, fac2


def replica_electrolyte(rng, n, rho_red, temp, sigma=4.0, mass=23.0, order=4, nmesh=32,
                        tstep=0.005, drnlist=2.0, eps_kT=0.1, relp=78.4):
    """One member of the batched ensemble: N ions (N/2 of each sign) at reduced density
    rho*sigma^3, temperature T; rc = min(30 A, L/2 - drnlist)."""
    rho = rho_red / sigma ** 3
    L = (n / rho) ** (1.0 / 3.0)
    rcut = min(30.0, L / 2.0 - drnlist)
    s = _base(n, 2, L, rcut, temp, relp, order, nmesh, tstep, drnlist=drnlist)
    s["zat"] = np.array([1.0, -1.0])
    s["sigat"] = np.array([sigma, sigma])
    s["epsat"] = np.array([eps_kT * kT(temp)] * 2)
    s["masspt"] = np.array([mass, mass])
    s["iptpn"] = np.array([1] * (n // 2) + [2] * (n // 2), np.int32)
    s["az"] = s["zat"][s["iptpn"] - 1].copy()
    s["ro"] = place_uniform(rng, n, L, 0.8 * sigma)
    s["rod"] = maxwell_velocities(rng, s["masspt"][s["iptpn"] - 1], temp)
    s["name"] = "replica_%d" % n
    return s


def batched_ensemble(seed=0, nsys=512, nmin=200, nmax=4000):
    """512 electrolytes with N ~ U{200..4000} (even), rho*sigma^3 ~ U[0.01, 0.3],
    T ~ U[250, 400] K; the SPME grid edge is chosen later by the autotuner."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nsys):
        n = 2 * int(rng.integers(nmin // 2, nmax // 2 + 1))
        rho_red = float(rng.uniform(0.01, 0.3))
        T = float(rng.uniform(250.0, 400.0))
        out.append(replica_electrolyte(rng, n, rho_red, T))
    return out


def scaled_job(rng, n, kind, order=4):
    """A serving job: the electrolyte generator at its density, or the polyelectrolyte
    generator at its density with chains of up to 200 beads, scaled to N particles."""
    if kind == "electrolyte":
        L = 100.0 * (n / 1000.0) ** (1.0 / 3.0)
        s = electrolyte(seed=int(rng.integers(1 << 30)), n_pairs=n // 2, L=L,
                        rcut=min(30.0, L / 2 - 2.0), nmesh=_grid_for(L), order=order)
    else:
        nb = n // 2
        nbead = min(200, max(2, nb))
        nchain = max(1, nb // nbead)
        nb = nchain * nbead
        L = 250.0 * (2 * nb / 16000.0) ** (1.0 / 3.0)
        s = polyelectrolyte(seed=int(rng.integers(1 << 30)), nchain=nchain, nbead=nbead, L=L,
                            rcut=min(25.0, L / 2 - 2.0), nmesh=_grid_for(L), order=order)
    return s


def _grid_for(L, spacing=3.9):
    for g in (16, 24, 32, 48, 64, 96, 128):
        if L / g <= spacing:
            return g
    return 128


def _random_rotations(rng, n):
    """n uniformly random rotation matrices (from normalised random quaternions)."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)


def particle_list(ro, box, rlist):
    """MOLSIM's particle list over positions ro (SetVListMD's rule, Src/nlist.F90:724-759):
    every pair within rlist stored once, in row ip (1-based) when (ip < jp and ip + jp odd)
    or (ip > jp and ip + jp even).  Returns nneighpn [np], jpnlist [np][maxnneigh] (1-based)."""
    from scipy.spatial import cKDTree

    L = float(box)
    t = cKDTree(np.mod(np.asarray(ro) + L / 2, L), boxsize=L)
    pairs = t.query_pairs(rlist, output_type="ndarray")
    n = len(ro)
    rows = [[] for _ in range(n)]
    for a, b in pairs:
        ip, jp = int(a) + 1, int(b) + 1
        lo, hi = min(ip, jp), max(ip, jp)
        own = lo if (lo + hi) % 2 == 1 else hi
        rows[own - 1].append(hi if own == lo else lo)
    maxn = max(1, max(len(r) for r in rows))
    nn = np.array([len(r) for r in rows], np.int32)
    jp = np.zeros((n, maxn), np.int32)
    for i, r in enumerate(rows):
        jp[i, :len(r)] = sorted(r)
    return nn, jp


def rigid_molecules(seed=0, nmol=400, nsolute=200, L=50.0, rcut=12.0, drnlist=1.0, temp=298.0, relp=78.4):
    """Polyatomic test system for UTwoBodyP: rigid three-site molecules (particle type 1:
    an A site at the centre and two B sites 1 A away, 109.47 degrees apart; charges -0.8,
    +0.4, +0.4) and one-site solutes (particle type 2: a neutral C site), random
    orientations, centres uniform without overlap.  Atom types A, B, C carry the (1,6,12)
    parameters of the site-site table.  Returns the particle and atom arrays in MOLSIM's
    layout (1-based) with the particle list."""
    rng = np.random.default_rng(seed)
    npart = nmol + nsolute
    ro = place_uniform(rng, npart, L, 4.0)
    ang = np.deg2rad(109.47)
    frame = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [np.cos(ang), np.sin(ang), 0.0]])
    rot = _random_rotations(rng, nmol)
    r_mol = ro[:nmol, None, :] + np.einsum("nij,kj->nki", rot, frame)
    r = np.concatenate([r_mol.reshape(-1, 3), ro[nmol:]])
    iptpn = np.array([1] * nmol + [2] * nsolute, np.int32)
    napt = np.array([3, 1], np.int32)
    ianpn = np.concatenate([1 + 3 * np.arange(nmol), 1 + 3 * nmol + np.arange(nsolute)]).astype(np.int32)
    iatan = np.array([1, 2, 2] * nmol + [3] * nsolute, np.int32)
    s = dict(np=npart, na=len(r), npt=2, nat=3, boxlen=[float(L)] * 3, rcut=float(rcut), drnlist=float(drnlist),
             temp=float(temp), relpermitt=float(relp), epsi_four_pi=EPSI0_FOUR_PI / relp, ro=ro, r=r, iptpn=iptpn,
             napt=napt, ianpn=ianpn, iatan=iatan, zat=np.array([-0.8, 0.4, 0.0]), sigat=np.array([3.0, 1.0, 4.0]),
             epsat=np.array([0.6, 0.05, 0.5]) * kT(temp), lewald=False, lljcut=False, **POT_DEFAULTS)
    s["nneighpn"], s["jpnlist"] = particle_list(ro, L, rcut + drnlist)
    s["name"] = "rigid_molecules_%d" % npart
    return s


def site_table_params(s):
    """Parameters of the site-site (atom-type) table of a rigid_molecules system: the table
    reaches past rcut by the largest site distance from a centre (twice), as MOLSIM's
    rumax = 1.1 (rcut + racom) does."""
    d = dict(s)
    d["npt"] = s["nat"]
    d["rcut"] = s["rcut"] + 2.0
    return d


def qua_to_ori(q):
    """QuaToOri (Src/mollib.F90:2221-2255) for quaternions q [n][4]: ori [n][3][3], which takes
    a particle's principal-frame vectors to the lab frame."""
    q = np.asarray(q, np.float64)
    q0, q1, q2, q3 = q.T
    o = np.empty((len(q), 3, 3))
    o[:, 0, 0] = -q2 * q2 + q1 * q1 - q3 * q3 + q0 * q0
    o[:, 1, 0] = 2 * (q0 * q3 - q1 * q2)
    o[:, 2, 0] = 2 * (q1 * q3 + q0 * q2)
    o[:, 0, 1] = -2 * (q1 * q2 + q0 * q3)
    o[:, 1, 1] = q2 * q2 - q1 * q1 - q3 * q3 + q0 * q0
    o[:, 2, 1] = 2 * (q0 * q1 - q2 * q3)
    o[:, 0, 2] = 2 * (q1 * q3 - q0 * q2)
    o[:, 1, 2] = -2 * (q2 * q3 + q0 * q1)
    o[:, 2, 2] = -q2 * q2 - q1 * q1 + q3 * q3 + q0 * q0
    return o


def rigid_bodies(seed=0, nmol=300, nsolute=100, L=40.0, rcut=10.0, drnlist=1.5, temp=298.0, relp=78.4,
                 tstep=0.001):
    """Rigid-body MD test system: three-site molecules (an O-like site of mass 16 and two H-like
    sites of mass 1, 1 A bonds at 109.47 degrees; charges -0.8, +0.4, +0.4) and one-site solutes
    (mass 23, neutral), with centres of mass, principal frames (sites `ra` in them, masses and
    principal moments `momp` per particle type), random orientations (quaternions `qua`) and
    Maxwell-Boltzmann centre velocities; quaternion velocities and accelerations start at zero.
    The site positions r = ro + ori(qua) ra and the particle list are included."""
    rng = np.random.default_rng(seed)
    s = rigid_molecules(seed=seed, nmol=nmol, nsolute=nsolute, L=L, rcut=rcut, drnlist=drnlist, temp=temp,
                        relp=relp)
    ang = np.deg2rad(109.47)
    sites = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [np.cos(ang), np.sin(ang), 0.0]])
    m = np.array([16.0, 1.0, 1.0])
    com = (m[:, None] * sites).sum(0) / m.sum()
    x = sites - com
    inertia = (m[:, None, None] * ((x * x).sum(1)[:, None, None] * np.eye(3) - x[:, :, None] * x[:, None, :])).sum(0)
    mom, axes = np.linalg.eigh(inertia)
    ra = np.zeros((2, 3, 3))
    ra[0] = x @ axes                                   # principal-frame sites
    momp = np.array([mom, [1.0, 1.0, 1.0]])            # a one-site solute: no torque, any moment
    masspt = np.array([m.sum(), 23.0])
    q = rng.standard_normal((s["np"], 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    ori = qua_to_ori(q)
    ro = np.asarray(s["ro"])
    ipt = np.asarray(s["iptpn"]) - 1
    r = np.concatenate([(ro[:nmol, None, :] + np.einsum("nij,kj->nki", ori[:nmol], ra[0])).reshape(-1, 3),
                        ro[nmol:]])
    s.update(ra=ra, maxsite=3, masspt=masspt, momp=momp, qua=q, quad=np.zeros_like(q), quadd=np.zeros_like(q),
             r=r, rod=maxwell_velocities(rng, masspt[ipt], temp), rodd=np.zeros((s["np"], 3)), tstep=float(tstep),
             nvvite=2, tvvite=0.0)
    s["name"] = "rigid_bodies_%d" % s["np"]
    return s
