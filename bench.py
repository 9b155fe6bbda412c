#!/usr/bin/env python
"""Throughput of MOLSIM's per-step force/energy path on B200.

Workload (one GPU): the polyelectrolyte solution -- 40 chains x 200 beads
(-1e, sigma 4 A, harmonic bonds k = 0.4 kT/A^2, r0 = 5 A) plus 8000 counterions,
16000 particles in a 250 A box; SPME 64^3, order 5, rc = 25 A; tabulated LJ +
Coulomb; velocity Verlet, dt = 0.005 ps.  A step is one MD step (VelVer + UTotal
+ NList skin test / rebuild).  Synthetic, seeded inputs.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank advances its own replica (seed = rank): the path does
not shard, so N>1 runs N independent replicas ("weak" scaling, no collective
on the data path).  `--impl reference` times MOLSIM's serial algorithm (the
FP64 CPU restatement in oracle/, compiled -O2) on the host cores, one replica
per core.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
WORKLOAD = "polyelectrolyte_16000"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--replicas", type=int, default=32,
                    help="replicas of the workload in one handle for the batched figure (0: skip)")
    ap.add_argument("--ensemble", type=int, default=512,
                    help="systems in the batched ensemble (0: skip)")
    ap.add_argument("--bd", type=int, default=1, help="time the 200,000-particle BD system (0: skip)")
    ap.add_argument("--serve-wait", type=float, default=0.0,
                    help="serving: batching window in seconds before a cohort forms")
    ap.add_argument("--serve-ahead", type=int, default=2, help="serving: step chunks enqueued per cohort")
    ap.add_argument("--poly", type=int, default=1,
                    help="time UTwoBodyP on 50000 rigid molecules and solutes (0: skip)")
    ap.add_argument("--mc", type=int, default=1,
                    help="time Monte Carlo sweeps of the 1000-ion electrolyte, one chain and an ensemble (0: skip)")
    ap.add_argument("--ewald-std", type=int, default=1,
                    help="time the 1000-ion electrolyte with standard Ewald reciprocal space (0: skip)")
    ap.add_argument("--serve-jobs", type=int, default=200,
                    help="jobs in the serving stream (Poisson arrivals at 200/s; 0: skip)")
    ap.add_argument("--serve-budget-gib", type=float, default=4.0)
    ap.add_argument("--serve-refill", type=int, default=0,
                    help="serving: iteration-level admission (re-form a running cohort with waiting jobs)")
    ap.add_argument("--serve-low-rate", type=float, default=50.0,
                    help="serving: the same stream again at this arrival rate (jobs/s; 0: skip)")
    ap.add_argument("--profile", default=None, choices=["single", "batched", "bd"],
                    help="profiling target for ncu: build that workload (mixed precision), run a "
                         "UTotal and three steps, print one line of per-kernel times, no JSON line")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_workload(seed):
    from molsim_b200 import systems as S
    return S.polyelectrolyte(seed=seed)


# --------------------------------------------------------------------------
# CPU reference: the oracle, one replica per process
# --------------------------------------------------------------------------
def _oracle_worker(args):
    seed, steps, warm = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import pyoracle as O
    from molsim_b200 import systems as S
    s = S.polyelectrolyte(seed=seed)
    q2 = float(np.mean(s["az"] ** 2))
    alpha = O.rcut_to_alpha(s["uewaldtol"], q2, s["epsi_four_pi"], min(s["boxlen"]), s["rcut"])
    pot = dict(npt=s["npt"], zat=s["zat"], sigat=s["sigat"], epsat=s["epsat"], rcut=s["rcut"], ualpha=alpha,
               epsi_four_pi=s["epsi_four_pi"], lewald=1, lljcut=1,
               **{k: s[k] for k in ("ljrcut", "ljushift", "r2uminin", "utoltab", "ftoltab", "umaxtab", "fmaxtab",
                                    "rumaxfac")})
    t = O.pot_tab(pot)
    t["r2atat"] = np.zeros(3)
    d = dict(s)
    d["ualpha"] = alpha
    o = O.System(d, t, maxnneigh=512, lcellbuild=True)
    o.set_state(s["ro"], s["rod"])
    o.set_vlist()
    o.utotal()
    st = o.get_state()
    fo = o.utotal()["forceo"]
    o.set_state(st["ro"], st["rod"], fo / s["masspt"][s["iptpn"] - 1][:, None])
    for _ in range(warm):
        o.velver_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.velver_step()
    return s["np"] * steps, time.perf_counter() - t0


def cpu_reference(steps, warm, procs):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_oracle_worker, [(1000 + k, steps, warm) for k in range(procs)])
    # all replicas run concurrently: aggregate = sum of work / longest replica time
    work = sum(r[0] for r in res)
    tmax = max(r[1] for r in res)
    return work / tmax, tmax


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    steps = max(1, min(a.steps, 20))
    warm = max(0, min(a.warmup, 2))
    value, tmax = cpu_reference(steps, warm, procs)
    sample = "%d concurrent replicas x %d velocity-Verlet steps of the 16000-particle polyelectrolyte" % (procs, steps)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": 1000.0 * tmax / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "particles": 16000, "spme": "64^3 order 5", "rcut_A": 25.0,
                       "integrator": "velocity Verlet", "replicas": procs},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def read_profile_traffic(name="pair_kernel_polyelectrolyte_16000.md"):
    """Per-launch DRAM bytes of the pair kernel from a committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class L2Flush:
    """Evicts the step's data from the 126 MB L2 before a timed step: a 256 MB write,
    then a 256 MB read of a second buffer, so the write's dirty lines are written back
    before the step starts instead of during it."""

    def __init__(self):
        import torch

        self.w = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        self.r = torch.zeros(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def __call__(self):
        self.w.zero_()
        self.r.sum()


def tuner_run(flush):
    """Step timer for the pair-kernel tuner: ms per step of `steps` device-timed MD steps
    with the L2 flushed before each, as the timed legs run them."""
    return lambda e, steps: timed_md_steps(e, steps, flush, 0) / steps


def timed_md_steps(e, K, flush, warmup):
    """K MD steps of every system of engine e, L2 flushed before each; device time
    summed over the steps (ms), CUDA events on the engine's stream."""
    import torch

    from molsim_b200 import _lib

    Lx = _lib.lib()
    extx = torch.cuda.ExternalStream(e.stream())
    for _ in range(max(3, warmup)):
        with torch.cuda.stream(extx):
            flush()
        if Lx.msg_velver_async(e.h, 1):
            raise RuntimeError(Lx.msg_last_error(e.h).decode())
    e.VelVer(1, energies=False)
    torch.cuda.synchronize()
    st = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    en = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    for k in range(K):
        with torch.cuda.stream(extx):
            flush()
            st[k].record(extx)
        if Lx.msg_velver_async(e.h, 1):
            raise RuntimeError(Lx.msg_last_error(e.h).decode())
        with torch.cuda.stream(extx):
            en[k].record(extx)
    torch.cuda.synchronize()
    return sum(x.elapsed_time(y) for x, y in zip(st, en))


def hbm_peak():
    """(peak GB/s, source) for the roofline denominators."""
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
        if "hbm_gbs" in peaks:
            return float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6650 GB/s"


def pair_bytes(e, s_pos, s_f=24):
    """Algorithmic bytes of one pair-kernel launch over every system of engine e:
    sum of N (s_pos + s_f) + 4 P_half, with P_half each system's half-list pair count
    (the reference's SetVListMD rule, from a fresh list build)."""
    tot = pairs = 0
    for k, sd in enumerate(e.systems):
        _, _, npair = e.SetVList(k, export=False)
        tot += int(sd["np"]) * (s_pos + s_f) + 4 * int(npair)
        pairs += int(npair)
    return tot, pairs


def pair_roofline(e, step, K, flush, b_pair, traffic=None):
    """Roofline object of the pair kernel of engine e: its mean CUDA-event duration over K
    steps (the library's per-kernel timers, which serialise the step's two branches), with
    the L2 flushed before each step; `step` advances e by one step."""
    import torch

    ext = torch.cuda.ExternalStream(e.stream())
    e.set_timing(True)
    for _ in range(K):
        with torch.cuda.stream(ext):
            flush()
        step()
    kt = e.kernel_times()
    e.set_timing(False)
    tot, cnt = kt.get("pair", (0.0, 0))
    t_pair = tot / cnt / 1000.0 if cnt else 0.0
    peak, src = hbm_peak()
    achieved = b_pair / t_pair / 1e9 if t_pair > 0 else 0.0
    return {"kernel": "pair", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if peak else None, "traffic": traffic, "algorithmic_bytes_per_launch": b_pair,
            "pair_ms_per_launch": 1000.0 * t_pair, "peak_source": src}


def run_ensemble(a, flush, rank=0, world=1):
    """The batched ensemble: electrolytes with N ~ U{200..4000}, rho*sigma^3 ~ U[0.01, 0.3],
    T ~ U[250, 400] K, SPME order 4 with the grid edge of each system chosen by the
    autotuner from {16, 24, 32, 48}; all systems in one handle, one CUDA-graph replay
    per step.  Mixed precision, beside the same ensemble on the FP64 path.  Under torchrun
    the systems are partitioned across the ranks (longest-work-first, no exchange on the
    data path): each rank advances its share in its own handle, and the whole-job figure
    is all particle-steps over the slowest rank's device time."""
    import torch

    from molsim_b200 import Engine, prepare
    from molsim_b200.autotune import apply_grids, tune_grids, tune_pair_kernel
    from molsim_b200.shard import combine_ensemble, ensemble_share, gather_metrics
    from molsim_b200.systems import batched_ensemble

    t0 = time.perf_counter()
    systems_all = batched_ensemble(seed=0, nsys=a.ensemble)
    tables_all = [prepare(s) for s in systems_all]
    if world > 1:
        from molsim_b200.engine import estimate_bytes
        nb = [estimate_bytes(s_, t_) for s_, t_ in zip(systems_all, tables_all)]
        mine = ensemble_share([int(s_["np"]) for s_ in systems_all], nb, rank, world)
    else:
        mine = list(range(len(systems_all)))
    systems = [systems_all[k] for k in mine]
    tables = [tables_all[k] for k in mine]
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    edges, rep = tune_grids(systems, tables)
    t_tune = time.perf_counter() - t0
    sy = apply_grids(systems, edges)
    ntot = sum(int(s["np"]) for s in sy)
    eng = Engine(sy, tables, precision="mixed")
    eng.UTotal(0)
    eng.GetLinAcc()
    best, lane_ms = tune_pair_kernel(eng, steps=25, run=tuner_run(flush))
    eng.reset_states()
    eng.UTotal(0)
    eng.GetLinAcc()
    K = max(10, a.steps // 4)
    if world > 1:
        torch.distributed.barrier()
    ms = timed_md_steps(eng, K, flush, a.warmup)
    del eng
    e64 = Engine(sy, tables, precision="fp64")
    e64.UTotal(0)
    e64.GetLinAcc()
    if world > 1:
        torch.distributed.barrier()
    ms64 = timed_md_steps(e64, K, flush, a.warmup)
    del e64
    torch.cuda.synchronize()
    # the same systems with the SPME reciprocal-space chain as one persistent kernel
    # (MSG_SPME_CONV=1) and the pair kernel shaped as tuned above; a failure is recorded,
    # not raised, so that it cannot cost the legs that follow
    ms_conv, conv_err = None, None
    try:
        from molsim_b200 import _lib

        os.environ["MSG_SPME_CONV"] = "1"
        try:
            ec = Engine(sy, tables, precision="mixed")
        finally:
            os.environ.pop("MSG_SPME_CONV", None)
        Lc = _lib.lib()
        for key, val in ((_lib.MSG_TUNE_PAIR_KERNEL, best["kind"]), (_lib.MSG_TUNE_PAIR_UNROLL, best["unroll"]),
                         (_lib.MSG_TUNE_OVERLAP, best["overlap"]), (_lib.MSG_TUNE_PAIR_BLOCKS, best["blocks"])):
            if Lc.msg_tune(ec.h, key, int(val)):
                raise RuntimeError(Lc.msg_last_error(ec.h).decode())
        ec.tune_pair_lanes(best["shift"])
        ec.UTotal(0)
        ec.GetLinAcc()
        ms_conv = timed_md_steps(ec, K, flush, a.warmup)
        del ec
        torch.cuda.synchronize()
    except Exception as ex:                                  # noqa: BLE001
        conv_err = str(ex)[:200]
    per = gather_metrics({"systems": len(sy), "particles": ntot, "steps": K, "device_ms": ms,
                          "device_ms_fp64": ms64, "device_ms_conv": ms_conv, "conv_error": conv_err,
                          "edges": list(edges), "met": int(sum(r["met"] for r in rep))})
    comb = combine_ensemble(per)
    comb64 = combine_ensemble([dict(m, device_ms=m["device_ms_fp64"]) for m in per])
    conv = None
    if all(m["device_ms_conv"] is not None for m in per):
        cc = combine_ensemble([dict(m, device_ms=m["device_ms_conv"]) for m in per])
        conv = {"value": cc["value"], "ms_per_step": cc["device_ms_max"] / K,
                "vs_graph_cufft": cc["value"] / comb["value"]}
    else:
        conv = {"error": next((m["conv_error"] for m in per if m["conv_error"]), "not measured")}
    all_edges = [e_ for m in per for e_ in m["edges"]]
    hist = {g: all_edges.count(g) for g in sorted(set(all_edges))}
    return {"systems": comb["systems"], "particles": comb["particles"], "value": comb["value"], "unit": METRIC,
            "steps": K, "ms_per_step": comb["device_ms_max"] / K, "precision": "mixed",
            "fp64_batched_value": comb64["value"], "vs_fp64_batched": comb["value"] / comb64["value"],
            "ranks": world, "partition": "longest-work-first over ranks, no collective on the data path",
            "autotune": {"grid_edges": hist, "target_met": int(sum(m["met"] for m in per)),
                         "rule": "cheapest edge with measured reciprocal RMS force error <= Kolafa-Perram "
                                 "real-space estimate (reference 96^3 order 6)",
                         "pair_kernel": best, "pair_kernel_ms_per_step": lane_ms, "tune_s": t_tune},
            "spme_conv_kernel": conv, "generate_s": t_gen}


def run_bd(a, flush):
    """The 200,000-particle charged-colloid Brownian dynamics (2000 macroions +20e, 40000
    counterions, 79000 salt pairs; L = 1200 A; SPME 128^3 order 4; rc = 30 A; Ermak-McCammon,
    dt = 1e-3 ps, FP32 Philox noise): device time per BD step, L2 flushed before each, mixed
    precision beside the FP64 path."""
    import torch

    from molsim_b200 import Engine, _lib
    from molsim_b200 import systems as S

    s = S.colloid_bd(seed=0)
    s["bd_fac"] = S.bd_factors(s)
    n = int(s["np"])
    L = _lib.lib()
    out = {"particles": n, "spme": "128^3 order 4", "rcut_A": 30.0, "unit": METRIC}
    for prec in ("mixed", "fp64"):
        e = Engine(s, precision=prec)
        e.UTotal()
        ext = torch.cuda.ExternalStream(e.stream())
        K = max(10, a.steps // 10)
        for _ in range(3):
            e.BDStep(1, seed=7, energies=False)
        torch.cuda.synchronize()
        st = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        en = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        for k in range(K):
            with torch.cuda.stream(ext):
                flush()
                st[k].record(ext)
            if L.msg_bd_step(e.h, 1, 7, 0, None, None, None):
                raise RuntimeError(L.msg_last_error(e.h).decode())
            with torch.cuda.stream(ext):
                en[k].record(ext)
        torch.cuda.synchronize()
        ms = sum(x.elapsed_time(y) for x, y in zip(st, en))
        out["value" if prec == "mixed" else "fp64_value"] = n * K / (ms / 1000.0)
        out["ms_per_step" if prec == "mixed" else "fp64_ms_per_step"] = ms / K
        out["steps"] = K
        if prec == "mixed":
            b_pair, pairs = pair_bytes(e, 16)
            e.BDStep(1, seed=7, energies=False)

            def bd_step():
                if L.msg_bd_step(e.h, 1, 7, 0, None, None, None):
                    raise RuntimeError(L.msg_last_error(e.h).decode())
            out["roofline"] = pair_roofline(e, bd_step, K, flush, b_pair,
                                            traffic=read_profile_traffic("pair_kernel_bd_200000.md"))
            out["half_list_pairs"] = pairs
        del e
    out["vs_fp64"] = out["value"] / out["fp64_value"]
    return out


def _std_nkv(ncut, cube=False):
    """k-vectors of the standard Ewald sum (0 <= n_i <= ncut, |n|^2 within the region, n != 0)."""
    c2 = 3 * ncut * ncut if cube else ncut * ncut
    r = range(ncut + 1)
    return sum(1 for x in r for y in r for z in r if 0 < x * x + y * y + z * z <= c2)


# FP64 operations per (k-vector, particle) as k_ew_sk (44) and k_ew_force (67) issue them
STD_FLOP_PER_KP = 111


def run_ewald_std(a, flush):
    """The 1000-ion electrolyte (500 + 500 ions, L = 100 A, rc = 30 A) with standard Ewald
    reciprocal space (txewaldrec 'std', sphere, ncut from AlphaToNcut at uewaldtol = 1e-5):
    device time per MD step with the L2 flushed before each, FP64 drop-in and mixed, beside
    the same system on SPME (32^3 order 4) and the oracle on one host core."""
    import torch

    from molsim_b200 import Engine, prepare
    from molsim_b200 import systems as S

    s = S.electrolyte(0)
    d = dict(s)
    d["ewaldrec"] = "std"
    d["ncutregion"] = "sphere"
    t = prepare(d)
    n, ncut = int(s["np"]), int(t["ncut"])
    nkv = _std_nkv(ncut)
    K = max(10, a.steps // 10)
    out = {"workload": "electrolyte_1000 (L = 100 A, rc = 30 A)", "ncut": ncut, "k_vectors": nkv,
           "unit": METRIC, "steps": K}
    for prec in ("fp64", "mixed"):
        e = Engine(d, t, precision=prec)
        e.UTotal()
        e.GetLinAcc()
        ms = timed_md_steps(e, K, flush, a.warmup)
        out["value" if prec == "fp64" else "mixed_value"] = n * K / (ms / 1000.0)
        out["ms_per_step" if prec == "fp64" else "mixed_ms_per_step"] = ms / K
        if prec == "fp64":
            ext = torch.cuda.ExternalStream(e.stream())
            e.set_timing(True)
            for _ in range(K):
                with torch.cuda.stream(ext):
                    flush()
                e.VelVer(1, energies=False)
            kt = e.kernel_times()
            e.set_timing(False)
            tot, cnt = kt.get("ewald_std", (0.0, 0))
            if cnt:
                ms_ew = tot / cnt
                out["ewald_std_ms_per_step"] = ms_ew
                out["ewald_std_fp64_tflops"] = STD_FLOP_PER_KP * nkv * n / (ms_ew / 1000.0) / 1e12
        del e
    es = Engine(s, precision="fp64")
    es.UTotal()
    es.GetLinAcc()
    out["spme_fp64_value"] = n * K / (timed_md_steps(es, K, flush, a.warmup) / 1000.0)
    del es
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np
        import pyoracle as O
        q2 = float(np.mean(s["az"] ** 2))
        pot = dict(npt=s["npt"], zat=s["zat"], sigat=s["sigat"], epsat=s["epsat"], rcut=s["rcut"],
                   ualpha=t["ualpha"], epsi_four_pi=s["epsi_four_pi"], lewald=1, lljcut=1,
                   **{k: s[k] for k in ("ljrcut", "ljushift", "r2uminin", "utoltab", "ftoltab", "umaxtab",
                                        "fmaxtab", "rumaxfac")})
        ot = O.pot_tab(pot)
        ot["r2atat"] = np.zeros(3)
        od = dict(d)
        od["ualpha"] = t["ualpha"]
        od["ncut"] = O.alpha_to_ncut(s["uewaldtol"], q2, s["epsi_four_pi"], min(s["boxlen"]), t["ualpha"])
        o = O.System(od, ot, maxnneigh=n)
        o.set_state(s["ro"], s["rod"])
        o.set_vlist()
        fo = o.utotal()["forceo"]
        st = o.get_state()
        o.set_state(st["ro"], st["rod"], fo / s["masspt"][s["iptpn"] - 1][:, None])
        steps = 3
        t0 = time.perf_counter()
        for _ in range(steps):
            o.velver_step()
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n * steps / cpu_s, "unit": METRIC, "cores": 1, "kind": "port",
                               "sample": "%d velocity-Verlet steps of the same system, oracle (FP64 C "
                                         "restatement of UEwaldRecStd and the rest of the serial path), "
                                         "1 thread" % steps}
    return out


def run_mc(a):
    """Monte Carlo single-particle translations (MCPass/SPartMove/DUTotal/Metropolis) of the
    1000-ion electrolyte with standard Ewald (ncut from AlphaToNcut at 1e-5, sphere), displacement
    2 A, at 298 K: trial moves per second for one chain and for an ensemble of 592 chains (four per
    SM, one seed each), device time around each call (a UTotal, the sweeps and the list rebuild),
    beside the oracle's chain on one host core."""
    import torch

    from molsim_b200 import Engine, prepare
    from molsim_b200 import systems as S

    s = S.electrolyte(0)
    d = dict(s)
    d["ewaldrec"] = "std"
    t = prepare(d)
    n = int(s["np"])
    beta = 1.0 / S.kT(s["temp"])
    dtran = [2.0] * s["npt"]
    out = {"workload": "electrolyte_1000, standard Ewald (ncut %d), dtran 2 A, 298 K" % t["ncut"],
           "unit": "trial moves/s"}

    def timed(e, npass):
        ext = torch.cuda.ExternalStream(e.stream())
        e.MCPass(1, dtran, beta)                       # warm-up
        torch.cuda.synchronize()
        st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st.record(ext)
        acc, _, _ = e.MCPass(npass, dtran, beta)
        en.record(ext)
        torch.cuda.synchronize()
        return st.elapsed_time(en) / 1000.0, acc

    e1 = Engine(d, t, precision="fp64")
    e1.mc_seed(1)
    sweeps = 5
    sec, acc = timed(e1, sweeps)
    out["single"] = {"value": n * sweeps / sec, "sweeps": sweeps, "acceptance": float(acc[0]) / (n * sweeps)}
    del e1
    nrep = 4 * 148
    er = Engine([dict(d) for _ in range(nrep)], [t] * nrep, precision="fp64")
    for k in range(nrep):
        er.mc_seed(1 + k, isys=k)
    sec, acc = timed(er, sweeps)
    out["ensemble"] = {"value": nrep * n * sweeps / sec, "chains": nrep, "sweeps": sweeps,
                       "acceptance": float(acc.sum()) / (nrep * n * sweeps)}
    del er
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np
        import pyoracle as O
        q2 = float(np.mean(s["az"] ** 2))
        pot = dict(npt=s["npt"], zat=s["zat"], sigat=s["sigat"], epsat=s["epsat"], rcut=s["rcut"],
                   ualpha=t["ualpha"], epsi_four_pi=s["epsi_four_pi"], lewald=1, lljcut=1,
                   **{k: s[k] for k in ("ljrcut", "ljushift", "r2uminin", "utoltab", "ftoltab", "umaxtab",
                                        "fmaxtab", "rumaxfac")})
        ot = O.pot_tab(pot)
        ot["r2atat"] = np.zeros(3)
        od = dict(d)
        od["ualpha"] = t["ualpha"]
        od["ncut"] = O.alpha_to_ncut(s["uewaldtol"], q2, s["epsi_four_pi"], min(s["boxlen"]), t["ualpha"])
        o = O.System(od, ot, maxnneigh=n)
        o.set_state(s["ro"], s["rod"])
        o.set_vlist()
        u = o.utotal()
        o.mc_seed(1)
        t0 = time.perf_counter()
        o.mc_pass(1, dtran, beta, u)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": n / cpu_s, "unit": "trial moves/s", "cores": 1, "kind": "port",
                               "sample": "one sweep (1000 trial moves) of the same chain, oracle (FP64 C "
                                         "restatement of SPartMove/DUTotal/Metropolis/MCUpdate), 1 thread"}
    # the same chain with SPME reciprocal space (32^3, order 4): the trial's energy difference from
    # the spectrum and the two stencils' transforms
    ds = dict(s)
    tsp = prepare(ds)
    e2 = Engine(ds, tsp, precision="fp64")
    e2.mc_seed(1)
    sec, acc = timed(e2, sweeps)
    sp = {"workload": "electrolyte_1000, SPME %d^3 order %d, dtran 2 A, 298 K" % (s["nmesh"], s["order"]),
          "value": n * sweeps / sec, "unit": "trial moves/s", "sweeps": sweeps,
          "acceptance": float(acc[0]) / (n * sweeps)}
    del e2
    if not a.no_cpu_baseline:
        ods = dict(ds)
        ods["ualpha"] = tsp["ualpha"]
        o2 = O.System(ods, ot, maxnneigh=n)
        o2.set_state(s["ro"], s["rod"])
        o2.set_vlist()
        u2 = o2.utotal()
        o2.mc_seed(1)
        t0 = time.perf_counter()
        o2.mc_pass(1, dtran, beta, u2)
        sp["cpu_baseline"] = {"value": n / (time.perf_counter() - t0), "unit": "trial moves/s", "cores": 1,
                              "kind": "port", "sample": "one sweep of the same SPME chain, oracle (the "
                                                        "reference's way: the mesh re-transformed per trial), "
                                                        "1 thread"}
    out["spme"] = sp
    # MCAllPass on the 16000-particle polyelectrolyte: all particles displaced at once per trial
    # (draws jumped ahead on the device), list rebuild, UTotal, Metropolis
    pe = S.polyelectrolyte(seed=0)
    tpe = prepare(pe)
    ea = Engine(pe, tpe, precision="fp64")
    ea.mc_seed(1)
    dta = [0.05] * pe["npt"]
    ext = torch.cuda.ExternalStream(ea.stream())
    ea.MCAllPass(2, dta)                               # warm-up
    torch.cuda.synchronize()
    ntr = 20
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record(ext)
    acc, _ = ea.MCAllPass(ntr, dta)
    en.record(ext)
    torch.cuda.synchronize()
    sec = st.elapsed_time(en) / 1000.0
    ma = {"workload": "polyelectrolyte_16000 (SPME 64^3), MCAll dtranall 0.05 A", "trials": ntr,
          "value": pe["np"] * ntr / sec, "unit": "particle moves/s", "ms_per_trial": 1000.0 * sec / ntr,
          "acceptance": float(acc[0]) / ntr}
    del ea
    if not a.no_cpu_baseline:
        qpe = float(np.mean(pe["az"] ** 2))
        ape = O.rcut_to_alpha(pe["uewaldtol"], qpe, pe["epsi_four_pi"], min(pe["boxlen"]), pe["rcut"])
        ppe = dict(npt=pe["npt"], zat=pe["zat"], sigat=pe["sigat"], epsat=pe["epsat"], rcut=pe["rcut"],
                   ualpha=ape, epsi_four_pi=pe["epsi_four_pi"], lewald=1, lljcut=1,
                   **{k: pe[k] for k in ("ljrcut", "ljushift", "r2uminin", "utoltab", "ftoltab", "umaxtab",
                                         "fmaxtab", "rumaxfac")})
        otp = O.pot_tab(ppe)
        otp["r2atat"] = np.zeros(len(otp["r2umin"]))
        dpe = dict(pe)
        dpe["ualpha"] = ape
        op = O.System(dpe, otp, maxnneigh=512, lcellbuild=True)
        op.set_state(pe["ro"], pe["rod"])
        op.set_vlist()
        upe = op.utotal()
        op.mc_seed(1)
        t0 = time.perf_counter()
        op.mcall_pass(2, dta, 1.0 / S.kT(pe["temp"]), upe)
        ma["cpu_baseline"] = {"value": pe["np"] * 2 / (time.perf_counter() - t0), "unit": "particle moves/s",
                              "cores": 1, "kind": "port", "sample": "two MCAll trials of the same system, oracle, "
                                                                    "1 thread"}
    out["mcall_16000"] = ma
    return out


def run_poly(a):
    """UTwoBodyP (polyatomic particles) on 40000 rigid three-site molecules and 10000 one-site
    solutes (L = 185 A, rc = 10 A): the device time of the site-site pair computation, the whole
    call (host arrays in and out), and the oracle on one host core."""
    import numpy as np

    from molsim_b200 import systems as S
    from molsim_b200.engine import pot_tab
    from molsim_b200.polyatomic import utwobody_p

    s = S.rigid_molecules(seed=0, nmol=40000, nsolute=10000, L=185.0, rcut=10.0)
    d = S.site_table_params(s)
    t = pot_tab(d, 0.0)
    # site pairs of the particle pairs within rcut
    ro = np.asarray(s["ro"])
    npairs = 0
    napt = np.asarray(s["napt"])
    ipt = np.asarray(s["iptpn"]) - 1
    L = s["boxlen"][0]
    for i in range(s["np"]):
        js = s["jpnlist"][i, :s["nneighpn"][i]] - 1
        dd = ro[i] - ro[js]
        dd -= L * np.round(dd / L)
        ok = (dd * dd).sum(1) <= s["rcut"] ** 2
        npairs += int((napt[ipt[i]] * napt[ipt[js[ok]]]).sum())
    utwobody_p(s, t)                                  # warm-up
    reps = 5
    kms, calls = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        kms.append(utwobody_p(s, t)["kernel_ms"])
        calls.append((time.perf_counter() - t0) * 1000.0)
    call_ms = float(np.median(calls))
    out = {"workload": "40000 rigid 3-site molecules + 10000 solutes, L = 185 A, rc = 10 A",
           "site_pairs": npairs, "kernel_ms": float(np.median(kms)), "call_ms": call_ms,
           "site_pairs_per_s": npairs / (float(np.median(kms)) / 1000.0), "unit": "site pairs/s"}
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as O
        t0 = time.perf_counter()
        O.utwobody_p(s, t)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": npairs / cpu_s, "unit": "site pairs/s", "cores": 1, "kind": "port",
                               "sample": "one UTwoBodyP evaluation of the same system, oracle, 1 thread"}
    # the rigid-body MD step (quaternion velocity Verlet) on 16000 molecules + 4000 solutes
    import copy

    from molsim_b200.polyatomic import velver_p

    rb = S.rigid_bodies(seed=0, nmol=16000, nsolute=4000, L=136.0, rcut=10.0, drnlist=2.0, tstep=0.001)
    tb = pot_tab(S.site_table_params(rb), 0.0)
    velver_p(copy.deepcopy(rb), tb, 2)                 # warm-up
    k = 20
    ms = velver_p(copy.deepcopy(rb), tb, k)["kernel_ms"]
    md = {"workload": "16000 rigid 3-site molecules + 4000 solutes, L = 136 A, rc = 10 A, dt = 1 fs",
          "steps": k, "ms_per_step": ms / k, "value": rb["np"] * k / (ms / 1000.0), "unit": METRIC}
    if not a.no_cpu_baseline:
        ro = copy.deepcopy(rb)
        t0 = time.perf_counter()
        O.velver_p(ro, tb, 2)
        md["cpu_baseline"] = {"value": rb["np"] * 2 / (time.perf_counter() - t0), "unit": METRIC, "cores": 1,
                              "kind": "port", "sample": "two rigid-body steps of the same system, oracle, 1 thread"}
    # the same rigid bodies with SPME over the sites (order 5, 96^3 mesh)
    db = S.site_table_params(rb)
    db["lewald"] = 1
    tbs = pot_tab(db, 0.35)
    ewb = dict(az=np.asarray(rb["zat"], np.float64)[np.asarray(rb["iatan"]) - 1], ualpha=0.35, order=5, nmesh=96)
    velver_p(copy.deepcopy(rb), tbs, 2, ewald=ewb)    # warm-up
    ms = velver_p(copy.deepcopy(rb), tbs, k, ewald=ewb)["kernel_ms"]
    mds = {"workload": "16000 rigid 3-site molecules + 4000 solutes (52000 sites), L = 136 A, rc = 10 A, "
                       "SPME over sites alpha = 0.35, order 5, 96^3, dt = 1 fs",
           "steps": k, "ms_per_step": ms / k, "value": rb["np"] * k / (ms / 1000.0), "unit": METRIC}
    if not a.no_cpu_baseline:
        ro = copy.deepcopy(rb)
        t0 = time.perf_counter()
        O.velver_p(ro, tbs, 1, ewald=ewb)
        mds["cpu_baseline"] = {"value": rb["np"] / (time.perf_counter() - t0), "unit": METRIC, "cores": 1,
                               "kind": "port", "sample": "one rigid-body step with SPME over sites of the same "
                                                         "system, oracle, 1 thread"}
    md["rigid_md_spm_20000"] = mds
    out["rigid_md_20000"] = md
    # SPME over the 130000 sites of the UTwoBodyP system (order 5, 128^3 mesh, alpha 0.35)
    from molsim_b200.polyatomic import uewald_sites as _uew

    azs = np.asarray(s["zat"], np.float64)[np.asarray(s["iatan"]) - 1]
    _uew(s, azs, 0.35, order=5, nmesh=128)             # warm-up
    kms, calls = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        kms.append(_uew(s, azs, 0.35, order=5, nmesh=128)["kernel_ms"])
        calls.append((time.perf_counter() - t0) * 1000.0)
    km = float(np.median(kms))
    sp = {"workload": "SPME over the 130000 sites of the system above, alpha = 0.35, order 5, 128^3",
          "kernel_ms": km, "call_ms": float(np.median(calls)), "value": s["na"] / (km / 1000.0), "unit": "sites/s"}
    if not a.no_cpu_baseline:
        t0 = time.perf_counter()
        O.uewald_sites(s, azs, 0.35, order=5, nmesh=128)
        sp["cpu_baseline"] = {"value": s["na"] / (time.perf_counter() - t0), "unit": "sites/s", "cores": 1,
                              "kind": "port", "sample": "one SPME site sum of the same system, oracle, 1 thread"}
    out["uewald_sites_spm_130000"] = sp
    # UEwald over sites: 4000 rigid 3-site molecules (12000 sites), standard Ewald, alpha 0.35
    from molsim_b200.polyatomic import uewald_sites

    se = S.rigid_molecules(seed=5, nmol=4000, nsolute=0, L=75.0, rcut=11.0)
    az = np.asarray(se["zat"], np.float64)[np.asarray(se["iatan"]) - 1]
    ncut = 40
    nkv = _std_nkv(ncut)
    uewald_sites(se, az, 0.35, ncut)                   # warm-up
    kms, calls = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        kms.append(uewald_sites(se, az, 0.35, ncut)["kernel_ms"])
        calls.append((time.perf_counter() - t0) * 1000.0)
    km = float(np.median(kms))
    ew = {"workload": "4000 rigid 3-site molecules (12000 sites), L = 75 A, alpha = 0.35, ncut = 40 (sphere)",
          "k_vectors": nkv, "kernel_ms": km, "call_ms": float(np.median(calls)),
          "value": se["na"] * nkv / (km / 1000.0), "unit": "site k-vector terms/s",
          "fp64_tflops": STD_FLOP_PER_KP * nkv * se["na"] / (km / 1000.0) / 1e12}
    if not a.no_cpu_baseline:
        sm = S.rigid_molecules(seed=5, nmol=1000, nsolute=0, L=47.0, rcut=11.0)
        azm = np.asarray(sm["zat"], np.float64)[np.asarray(sm["iatan"]) - 1]
        nc = 25
        t0 = time.perf_counter()
        O.uewald_sites(sm, azm, 0.35, nc)
        ew["cpu_baseline"] = {"value": sm["na"] * _std_nkv(nc) / (time.perf_counter() - t0),
                              "unit": "site k-vector terms/s", "cores": 1, "kind": "port",
                              "sample": "one site Ewald sum of 1000 molecules (3000 sites, L = 47 A, ncut = 25), "
                                        "oracle, 1 thread"}
    # the rigid-body MD step with the site Ewald sum: 4000 molecules + 1000 solutes (13000 sites)
    re_ = S.rigid_bodies(seed=0, nmol=4000, nsolute=1000, L=85.0, rcut=10.0, drnlist=2.0, tstep=0.001)
    dre = S.site_table_params(re_)
    dre["lewald"] = 1
    tre = pot_tab(dre, 0.35)
    ewp = dict(az=np.asarray(re_["zat"], np.float64)[np.asarray(re_["iatan"]) - 1], ualpha=0.35, ncut=45)
    velver_p(copy.deepcopy(re_), tre, 2, ewald=ewp)     # warm-up
    k = 10
    ms = velver_p(copy.deepcopy(re_), tre, k, ewald=ewp)["kernel_ms"]
    mde = {"workload": "4000 rigid 3-site molecules + 1000 solutes (13000 sites), L = 85 A, rc = 10 A, "
                       "site Ewald alpha = 0.35, ncut = 45, dt = 1 fs",
           "steps": k, "ms_per_step": ms / k, "value": re_["np"] * k / (ms / 1000.0), "unit": METRIC}
    if not a.no_cpu_baseline:
        rs = S.rigid_bodies(seed=0, nmol=1000, nsolute=250, L=52.0, rcut=10.0, drnlist=2.0, tstep=0.001)
        drs = S.site_table_params(rs)
        drs["lewald"] = 1
        trs = pot_tab(drs, 0.35)
        ews = dict(az=np.asarray(rs["zat"], np.float64)[np.asarray(rs["iatan"]) - 1], ualpha=0.35, ncut=28)
        t0 = time.perf_counter()
        O.velver_p(rs, trs, 2, ewald=ews)
        mde["cpu_baseline"] = {"value": rs["np"] * 2 / (time.perf_counter() - t0), "unit": METRIC, "cores": 1,
                               "kind": "port",
                               "sample": "two rigid-body steps with site Ewald of 1000 molecules + 250 solutes "
                                         "(L = 52 A, ncut = 28), oracle, 1 thread"}
    ew["rigid_md_ewald_5000"] = mde
    out["uewald_sites_12000"] = ew
    return out


def run_serving(a, rank=0, world=1):
    """The serving stream: Poisson arrivals at 200 jobs/s, N log-uniform over 100-20000,
    half electrolytes and half polyelectrolytes, 1000 MD steps each, mixed precision,
    admitted by device-memory budget into concurrent cohorts; the same jobs again at a
    rate the GPU keeps up with (a.serve_low_rate jobs/s), so that latency shows service
    time rather than queueing.  Beside them: a sample of the same jobs run alone, one after
    another, on the plain FP64 path.  Under torchrun each rank serves its share of the
    stream (jobs partitioned by work, longest first; no exchange on the data path), and
    the metrics of all ranks are combined: particle-steps over the longest rank's span,
    latency percentiles over all jobs."""
    import torch

    from molsim_b200 import Engine
    from molsim_b200.serve import Server, poisson_stream
    from molsim_b200.shard import combine_serving, gather_metrics, my_share

    # load the library and fill the cuFFT plan cache outside the measured stream
    warm = poisson_stream(seed=12, rate=1e6, njobs=4, nmin=100, nmax=400, nsteps=20)
    Server(1 << 30, precision="mixed", chunk=10).run(warm, realtime=False)
    out = None
    for rate in (200.0, a.serve_low_rate):
        if rate <= 0:
            continue
        jobs = poisson_stream(seed=11, rate=rate, njobs=a.serve_jobs, nmin=100, nmax=20000, nsteps=1000)
        if world > 1:
            jobs = my_share(jobs, [j.n * j.nsteps for j in jobs], [1] * len(jobs), rank, world)
        srv = Server(int(a.serve_budget_gib * (1 << 30)), precision="mixed", max_cohorts=8, max_jobs=64, chunk=50,
                     batch_wait_s=a.serve_wait, ahead=a.serve_ahead, refill=bool(a.serve_refill))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        m = srv.run(jobs)
        per = gather_metrics(m)
        comb = combine_serving(per) if world > 1 else dict(m)
        comb.pop("latencies", None)
        comb["jobs_per_s_offered"] = rate
        if out is None:
            out = comb
            out["jobs_all"] = jobs
        else:
            out["low_rate"] = comb
    jobs = out.pop("jobs_all")
    # the plain FP64 path, each job alone: a sample across sizes, 200 steps each
    smp = sorted(jobs, key=lambda j: j.n)[:: max(1, len(jobs) // 12)][:12]
    work = tsum = 0.0
    ks = 200
    for j in smp:
        e = Engine(j.system, j.table, precision="fp64")
        e.UTotal()
        e.GetLinAcc()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.VelVer(ks, energies=False)
        torch.cuda.synchronize()
        tsum += (time.perf_counter() - t0) * j.nsteps / ks
        work += j.n * j.nsteps
        del e
    alone = work / tsum if tsum else None
    out.update({"unit": METRIC, "nsteps_per_job": 1000, "ranks": world,
                "precision": "mixed", "fp64_alone_value": alone,
                "fp64_alone_sample": "%d jobs across the size range, %d steps each, scaled to 1000" % (len(smp), ks),
                "vs_fp64_alone": (out["value"] / alone) if alone else None})
    return out


def run_gpu(a):
    import ctypes as C

    import numpy as np
    import torch

    from molsim_b200 import Engine, _lib

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    s = make_workload(seed=rank)
    n = int(s["np"])
    eng = Engine(s, precision=a.precision)
    eng.UTotal()
    eng.GetLinAcc()
    flush = L2Flush()
    tuned = None
    if a.precision == "mixed":
        from molsim_b200.autotune import tune_pair_kernel
        # the tuner times steps as this bench does: on the device, L2 flushed before each
        tuned, _ = tune_pair_kernel(eng, steps=40, run=tuner_run(flush))
        # the timed steps start from the seeded initial state, however long the tuning ran
        eng.reset_states()
        eng.UTotal()
        eng.GetLinAcc()
    _, _, npair = eng.SetVList(0, export=False)
    ext = torch.cuda.ExternalStream(eng.stream())
    L = _lib.lib()

    def step_async(k):
        rc = L.msg_velver_async(eng.h, k)
        if rc:
            raise RuntimeError(L.msg_last_error(eng.h).decode())

    def timed_steps(e, K):
        return timed_md_steps(e, K, flush, a.warmup)

    # warm-up (also captures the step graph)
    for _ in range(max(3, a.warmup)):
        with torch.cuda.stream(ext):
            flush()
        step_async(1)
    eng.VelVer(1, energies=False)
    torch.cuda.synchronize()

    # ---- timed region: K steps, L2 flushed before each, device time per step ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    clocks = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = eng.launch_count()
    nb0 = eng.nrebuild(0)
    for k in range(a.steps):
        with torch.cuda.stream(ext):
            flush()
            starts[k].record(ext)
        step_async(1)
        with torch.cuda.stream(ext):
            ends[k].record(ext)
    torch.cuda.synchronize()
    launches = eng.launch_count() - l0
    rebuilds = eng.nrebuild(0) - nb0
    clk = clocks.stop()
    t_ms = sum(st.elapsed_time(en) for st, en in zip(starts, ends))
    if world > 1:
        tt = torch.tensor([t_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.barrier()
        t_ms = float(tt.item())
    value = n * a.steps * world / (t_ms / 1000.0)

    # ---- the plain FP64 path on the same system (the drop-in and the comparison base) ----
    fp64_value = None
    errs = None
    if a.precision != "fp64":
        e64 = Engine(s, precision="fp64")
        e64.UTotal()
        e64.GetLinAcc()
        fp64_value = n * a.steps / (timed_steps(e64, a.steps) / 1000.0)
        # the metric's accuracy condition: mixed forces against the plain FP64 GPU path, same state
        st_m = eng.get_state(0)
        e64.put_state(0, st_m["ro"], st_m["rod"], st_m["rodd"], keep_list=False)
        r64, rmx = e64.UTotal(), eng.UTotal()
        f64v, fmx = np.asarray(r64["force"]), np.asarray(rmx["force"])
        errs = {"force_rms_rel": float(np.sqrt(((fmx - f64v) ** 2).sum() / (f64v ** 2).sum()))}
        for k in ("utot", "urec", "virial", "ubond"):
            errs[k + "_rel"] = abs(rmx[k] - r64[k]) / max(abs(r64[k]), 1e-300)
        errs["utwob_rel"] = [abs(x - y) / max(abs(y), 1e-300) for x, y in zip(rmx["utwob"], r64["utwob"])]
        del e64
    # ---- batched: replicas of the workload advanced together in one handle ----
    batched = None
    if a.replicas > 1:
        eb = Engine([dict(s) for _ in range(a.replicas)], precision=a.precision)
        eb.UTotal(0)
        eb.GetLinAcc()
        tuned_b = None
        if a.precision == "mixed":
            from molsim_b200.autotune import tune_pair_kernel
            tuned_b, _ = tune_pair_kernel(eb, steps=5, run=tuner_run(flush))
            eb.reset_states()
            eb.UTotal(0)
            eb.GetLinAcc()
        kb = max(10, a.steps // 4)
        tb = timed_steps(eb, kb)
        batched = {"replicas": a.replicas, "pair_kernel": tuned_b, "value": n * a.replicas * kb / (tb / 1000.0), "unit": METRIC,
                   "steps": kb, "ms_per_step": tb / kb,
                   "vs_fp64_single": (n * a.replicas * kb / (tb / 1000.0)) / fp64_value if fp64_value else None}
        b_pair_b, _ = pair_bytes(eb, 32 if a.precision == "fp64" else 16)
        eb.VelVer(1, energies=False)
        batched["roofline"] = pair_roofline(eb, lambda: eb.VelVer(1, energies=False), kb, flush, b_pair_b,
                                            traffic=read_profile_traffic("pair_kernel_batched_32x16000.md"))
        del eb
        if a.precision != "fp64":
            # the same replicas on the FP64 path: the like-for-like comparison of the batched figure
            e64b = Engine([dict(s) for _ in range(a.replicas)], precision="fp64")
            e64b.UTotal(0)
            e64b.GetLinAcc()
            tb64 = timed_steps(e64b, kb)
            del e64b
            batched["fp64_value"] = n * a.replicas * kb / (tb64 / 1000.0)
            batched["vs_fp64_batched"] = tb64 / tb

    # ---- per-kernel device times: the same K steps with the library's CUDA-event timers ----
    eng.set_timing(True)
    for k in range(a.steps):
        with torch.cuda.stream(ext):
            flush()
        eng.VelVer(1, energies=False)
    kt = eng.kernel_times()
    eng.set_timing(False)
    total_k = sum(v[0] for v in kt.values()) or 1.0
    breakdown = {k: {"ms_per_launch": (v[0] / v[1]) if v[1] else 0.0, "share": v[0] / total_k}
                 for k, v in kt.items() if v[1]}

    # ---- end to end through the C-ABI with host buffers (the drop-in call pattern) ----
    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    st0 = eng.get_state(0)
    ro, rod, rodd = pinned((n, 3)), pinned((n, 3)), pinned((n, 3))
    ro[:], rod[:], rodd[:] = st0["ro"], st0["rod"], st0["rodd"]
    e = _lib.MsgEnergy()
    f64 = C.POINTER(C.c_double)
    pr = [x.ctypes.data_as(f64) for x in (ro, rod, rodd)]
    ke = max(10, a.steps // 2) if not a.no_e2e else 1
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke):
        # the drop-in step with host-held state: send, step, return (msg_velver_host)
        assert L.msg_velver_host(eng.h, 0, 1, pr[0], pr[1], pr[2], C.byref(e)) == 0
    t_e2e = time.perf_counter() - t0
    if world > 1:
        tt = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_e2e = float(tt.item())
    e2e = n * ke * world / t_e2e

    # ---- roofline of the pair kernel ----
    s_pos = 32 if a.precision == "fp64" else 16
    s_f = 24
    b_pair = n * (s_pos + s_f) + 4 * npair
    t_pair = breakdown.get("pair", {}).get("ms_per_launch", 0.0) / 1000.0
    peak, peak_src = hbm_peak()
    achieved = b_pair / t_pair / 1e9 if t_pair > 0 else 0.0
    traffic = read_profile_traffic()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu_steps = 3
        v, tmax = cpu_reference(cpu_steps, 1, 1)
        cpu = {"value": v, "unit": METRIC, "cores": 1, "kind": "port",
               "sample": "%d velocity-Verlet steps of the same 16000-particle polyelectrolyte, "
                         "oracle (FP64 C restatement of MOLSIM's serial path, -O2), 1 thread" % cpu_steps}

    ensemble = serving = bd = ewstd = mc = poly = None
    if rank == 0 and world == 1 and a.bd:
        bd = run_bd(a, flush)
    if rank == 0 and world == 1 and a.ewald_std:
        ewstd = run_ewald_std(a, flush)
    if rank == 0 and world == 1 and a.mc:
        mc = run_mc(a)
    if rank == 0 and world == 1 and a.poly:
        poly = run_poly(a)
    # independent systems shard across ranks: every rank runs these legs on its share
    if a.ensemble > 0:
        ensemble = run_ensemble(a, flush, rank, world)
    if a.serve_jobs > 0:
        serving = run_serving(a, rank, world)

    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t_ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f32+i64",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD, "particles": n, "half_list_pairs": int(npair),
                       "spme": "64^3 order 5", "rcut_A": 25.0, "skin_A": 2.0, "precision": a.precision,
                       "integrator": "velocity Verlet", "parallelism": "replicas" if world > 1 else "single",
                       "l2": "flushed before every timed step (256 MB write, then 256 MB read)",
                       "start": "timed steps start from the seeded initial state (reset after the pair-kernel tuning)",
                       "rebuilds_in_timed_steps": int(rebuilds), "pair_kernel": tuned},
            "fp64_value": fp64_value, "batched": batched, "ensemble": ensemble, "serving": serving,
            "bd_200k": bd, "ewald_std_1000": ewstd, "mc_1000": mc, "utwobody_p_50000": poly,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": 3 * 24 * n,
                    "d2h_bytes_per_step": 3 * 24 * n + C.sizeof(_lib.MsgEnergy)},
            "roofline": {"kernel": "pair", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "algorithmic_bytes_per_launch": b_pair, "pair_ms_per_launch": 1000.0 * t_pair,
                         "peak_source": peak_src},
            "kernels": breakdown, "gpu_launches": int(launches), "clocks": clk,
            "cpu_baseline": cpu, "errors_vs_fp64_gpu": errs}
    # like-for-like mixed/FP64 ratios and the other legs' headline figures as top-level scalars
    def g(d, *ks):
        for k in ks:
            if not isinstance(d, dict):
                return None
            d = d.get(k)
        return d
    line.update({
        "vs_fp64_single": value / fp64_value if fp64_value else None,
        "batched_value": g(batched, "value"), "batched_fp64_value": g(batched, "fp64_value"),
        "vs_fp64_batched": g(batched, "vs_fp64_batched"),
        "batched_roofline_frac": g(batched, "roofline", "frac"),
        "ensemble_value": g(ensemble, "value"), "ensemble_fp64_value": g(ensemble, "fp64_batched_value"),
        "vs_fp64_ensemble": g(ensemble, "vs_fp64_batched"),
        "ensemble_spme_conv_value": g(ensemble, "spme_conv_kernel", "value"),
        "bd_200k_value": g(bd, "value"), "bd_200k_fp64_value": g(bd, "fp64_value"),
        "vs_fp64_bd_200k": g(bd, "vs_fp64"), "bd_200k_roofline_frac": g(bd, "roofline", "frac"),
        "serving_value": g(serving, "value"), "serving_p50_s": g(serving, "p50_s"),
        "serving_p99_s": g(serving, "p99_s"), "serving_low_rate_p50_s": g(serving, "low_rate", "p50_s"),
        "serving_low_rate_p99_s": g(serving, "low_rate", "p99_s"),
        "force_rms_err_vs_fp64_gpu": g(errs, "force_rms_rel"),
    })
    print(json.dumps(line), flush=True)


def run_profile(a):
    """A small fixed workload for ncu captures: the 16000-particle polyelectrolyte alone
    or as 32 replicas in one handle, or the 200000-particle BD system; mixed precision with
    the default pair kernel; one UTotal and three steps (launched directly when the
    environment sets MSG_NO_GRAPHS=1, which ncu needs), then the library's per-kernel
    timers over three more steps."""
    import torch

    from molsim_b200 import Engine
    from molsim_b200 import systems as S

    if a.profile == "bd":
        s = S.colloid_bd(seed=0)
        s["bd_fac"] = S.bd_factors(s)
        e = Engine(s, precision="mixed")
        step = lambda: e.BDStep(1, seed=7, energies=False)          # noqa: E731
    else:
        s = S.polyelectrolyte(seed=0)
        e = Engine([dict(s) for _ in range(32 if a.profile == "batched" else 1)], precision="mixed")
        step = lambda: e.VelVer(1, energies=False)                  # noqa: E731
    e.UTotal(0)
    if a.profile != "bd":
        e.GetLinAcc()
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e.set_timing(True)
    for _ in range(3):
        step()
    kt = e.kernel_times()
    print(a.profile, {k: round(v[0] / v[1], 4) for k, v in kt.items() if v[1]})


def main():
    a = parse()
    if a.profile:
        run_profile(a)
        return
    if a.impl == "reference":
        run_reference(a)
    else:
        run_gpu(a)


if __name__ == "__main__":
    main()
