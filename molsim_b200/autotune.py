"""Autotuner for batched ensembles: SPME grid per system and pair-kernel lanes.

SPME grid (per system).  MOLSIM takes the grid edge from the input
(nmesh, Src/energy.F90:6855-7019) and alpha from the real-space tolerance
(RcutToAlpha, Src/energy.F90:7090-7105).  For an ensemble of systems of
different sizes and densities the edge is chosen here instead: for each system,
the cheapest edge among the candidates whose reciprocal-space force error does
not exceed the real-space truncation error at the system's alpha and cutoff.

* The reciprocal-space error is MEASURED: forces of every system with each
  candidate edge (FP64 path, same alpha and table) against a reference solve
  on a fine grid at spline order 6.  Real-space, self and bonded terms are the
  same in both, so the difference is the reciprocal-space error alone.
* The real-space error is the Kolafa-Perram estimate (J. Kolafa, J. W. Perram,
  Mol. Simul. 9 (1992) 351): for random charges the RMS force error of
  truncating erfc(alpha r)/r at rc is
      dF = 2 sqrt(<q^2>) sqrt(sum_j q_j^2 / (rc V)) exp(-alpha^2 rc^2) * EpsiFourPi
  (kJ/(mol A)), from integrating the squared large-r erfc force over the
  particles beyond rc.
* A system no candidate satisfies gets the largest candidate.

Pair kernel shape (per handle).  The pair kernel gives each particle G lanes,
G set from the expected row length; the tuner times a few steps for G scaled
by 2^shift, for 1, 2 or 4 row entries in flight per lane, and for all SMs or
2 blocks per SM (room for the SPME chain running beside it), and keeps the
fastest.  In FP64 the results do not depend on G beyond
FP64 rounding; in mixed precision a lane adds its few pair terms in FP32
before rounding them to fixed point, so G moves results by FP32 rounding
(relative 1e-7 level) while each setting stays deterministic and independent
of which other systems share the handle.  Timing advances the systems by
len(shifts) * (steps + 2) MD steps.
"""
import time

import numpy as np

CANDIDATES = (16, 24, 32, 48)


def kolafa_perram_force_error(system, alpha):
    q = np.asarray(system["az"], np.float64)
    vol = float(np.prod(system["boxlen"]))
    rc = float(system["rcut"])
    return 2.0 * np.sqrt(np.mean(q * q)) * np.sqrt(np.sum(q * q) / (rc * vol)) * \
        np.exp(-(alpha * rc) ** 2) * float(system["epsi_four_pi"])


def _forces(systems, tables, nmesh, order, chunk):
    """FP64 forces of every system with the given grid edge(s) and order."""
    from .engine import Engine

    out = []
    for a in range(0, len(systems), chunk):
        sub = []
        for k in range(a, min(len(systems), a + chunk)):
            d = dict(systems[k])
            d["nmesh"] = int(nmesh[k] if np.ndim(nmesh) else nmesh)
            d["order"] = int(order)
            sub.append(d)
        e = Engine(sub, tables[a:a + len(sub)], precision="fp64")
        e.UTotal(0)
        out.extend(e.forces(k)[0] for k in range(len(sub)))
        del e
    return out


def tune_grids(systems, tables, candidates=CANDIDATES, order=4, ref_mesh=None, ref_order=6, chunk=128):
    """Grid edge per system.  Returns (edges, report) where report[k] holds the
    measured RMS reciprocal error per candidate and the real-space target."""
    cands = sorted(candidates)
    if ref_mesh is None:
        ref_mesh = 2 * cands[-1]
    ref = _forces(systems, tables, ref_mesh, ref_order, chunk)
    err = {c: [] for c in cands}
    for c in cands:
        fc = _forces(systems, tables, c, order, chunk)
        for k in range(len(systems)):
            err[c].append(float(np.sqrt(np.mean(np.sum((fc[k] - ref[k]) ** 2, axis=1)))))
    edges, report = [], []
    for k, s in enumerate(systems):
        target = kolafa_perram_force_error(s, tables[k]["ualpha"])
        pick = next((c for c in cands if err[c][k] <= target), cands[-1])
        edges.append(pick)
        report.append(dict(target=target, met=err[pick][k] <= target, err={c: err[c][k] for c in cands}))
    return edges, report


def apply_grids(systems, edges, order=4):
    out = []
    for s, g in zip(systems, edges):
        d = dict(s)
        d["nmesh"] = int(g)
        d["order"] = int(order)
        out.append(d)
    return out


def _time_steps(engine, steps, repeats=3, run=None):
    """Milliseconds per MD step: the best of `repeats` runs of `steps` steps, each from the
    systems' initial state, so that every setting is timed over the same stretch of the
    same trajectory (the systems relax from their start and rebuild their lists more or
    less often as they go, which would otherwise favour whichever setting is timed
    first); a run that happens to meet a busy moment of the host does not decide.  `run`,
    when given, times the steps instead: run(engine, steps) -> ms per step (for instance
    device-timed steps with the caller's cache conditions); by default the wall clock
    times them."""
    import torch

    best = float("inf")
    for _ in range(repeats):
        engine.reset_states()
        engine.UTotal(0)
        engine.GetLinAcc()
        if run is not None:
            best = min(best, run(engine, steps))
            continue
        engine.VelVer(2, energies=False)           # (re)capture the graph for this layout
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        engine.VelVer(steps, energies=False)
        torch.cuda.synchronize()
        best = min(best, 1000.0 * (time.perf_counter() - t0) / steps)
    return best


def tune_pair_lanes(engine, shifts=(-1, 0, 1), steps=10):
    """Time `steps` MD steps per lane scaling; leave the engine on the fastest.
    Returns (best shift, {shift: ms per step})."""
    times = {}
    for sh in shifts:
        engine.tune_pair_lanes(sh)
        times[sh] = _time_steps(engine, steps)
    best = min(times, key=times.get)
    engine.tune_pair_lanes(best)
    return best, times


def tune_pair_kernel(engine, steps=10, shifts=(-3, -2, -1, 0, 1), unrolls=(1, 2, 4), blocks=(0, 2), kinds=(2, 3),
                     overlaps=(1, 0), run=None):
    """Shape of the pair kernel for this handle, by timing MD steps: the list layout
    (kind 2: half list with partner atomics, 3: full list), lanes per particle
    (2^shift times the default), row entries in flight per lane (unroll), whether the
    pair kernel runs beside the SPME chain or after it (overlap 1 or 0), and pair blocks
    per SM (0: as many as fit; 2: room for the SPME chain beside it).  Layout and lanes
    are searched together (which lane count suits a system depends on the layout), then
    entries in flight and the overlap together (more entries in flight hold more of an
    SM's registers, which the SPME chain beside the kernel also needs), then the blocks;
    each setting is timed from the systems' initial state (by `run` when given, see
    _time_steps).  Leaves the engine on the best; returns ({knob: value},
    {setting: ms per step}).  Mixed precision only (the knobs belong to its pair kernel).  Every
    setting gives the same results to FP32 rounding of the forces."""
    from . import _lib

    setk = engine.tune
    best = {"kind": 2, "shift": 0, "unroll": 2, "overlap": 1, "blocks": 0}
    log = {}
    res = {}
    for kd in kinds:
        setk(_lib.MSG_TUNE_PAIR_KERNEL, kd)
        for sh in shifts:
            engine.tune_pair_lanes(sh)
            res[(kd, sh)] = _time_steps(engine, steps, run=run)
            log["kind=%s,shift=%s" % (kd, sh)] = res[(kd, sh)]
    best["kind"], best["shift"] = min(res, key=res.get)
    setk(_lib.MSG_TUNE_PAIR_KERNEL, best["kind"])
    engine.tune_pair_lanes(best["shift"])
    res = {}
    for un in unrolls:
        setk(_lib.MSG_TUNE_PAIR_UNROLL, un)
        for ov in overlaps:
            setk(_lib.MSG_TUNE_OVERLAP, ov)
            res[(un, ov)] = _time_steps(engine, steps, run=run)
            log["unroll=%s,overlap=%s" % (un, ov)] = res[(un, ov)]
    best["unroll"], best["overlap"] = min(res, key=res.get)
    setk(_lib.MSG_TUNE_PAIR_UNROLL, best["unroll"])
    setk(_lib.MSG_TUNE_OVERLAP, best["overlap"])
    for name, vals, key in (("blocks", blocks, _lib.MSG_TUNE_PAIR_BLOCKS),):
        res = {}
        for v in vals:
            setk(key, v)
            res[v] = _time_steps(engine, steps, run=run)
            log["%s=%s" % (name, v)] = res[v]
        best[name] = min(res, key=res.get)
        setk(key, best[name])
    return best, log
