"""Partition independent systems (an ensemble or a job stream) across GPUs.

The systems of a batched ensemble or a serving stream are independent, so
they shard across ranks with no exchange on the data path: each rank runs its
share in its own handles and only metrics are gathered at the end.  (A single
system does not shard: ranks run replicas.)

`assign` is greedy longest-processing-time bin packing: systems in decreasing
order of work (particles x steps) go to the rank with the least work so far
among the ranks whose memory budget still fits the system.  It is a pure
function of its inputs, so every rank computes the same assignment without
communicating.
"""
import numpy as np


def assign(work, nbytes, world, budget_bytes=None):
    """Rank of each system.  work[k]: particle-steps of system k; nbytes[k]: its
    device bytes; budget_bytes: per-rank memory budget (None: unlimited).
    Raises ValueError if a system fits no rank."""
    work = np.asarray(work, np.float64)
    nbytes = np.asarray(nbytes, np.int64)
    load = np.zeros(world)
    used = np.zeros(world, np.int64)
    out = np.full(len(work), -1, np.int64)
    # decreasing work; ties by index so the order is deterministic
    order = sorted(range(len(work)), key=lambda k: (-work[k], k))
    for k in order:
        ok = np.ones(world, bool) if budget_bytes is None else used + nbytes[k] <= budget_bytes
        if not ok.any():
            raise ValueError("system %d (%d bytes) fits no rank's budget" % (k, nbytes[k]))
        cand = np.where(ok)[0]
        r = int(cand[np.argmin(load[cand])])
        out[k] = r
        load[r] += work[k]
        used[r] += nbytes[k]
    return out


def my_share(items, work, nbytes, rank, world, budget_bytes=None):
    """The items this rank runs, in their original order."""
    a = assign(work, nbytes, world, budget_bytes)
    return [it for it, r in zip(items, a) if r == rank]


def gather_metrics(local, group=None):
    """All ranks' metric dicts on every rank (torch.distributed object gather); the
    only collective, after the data path has finished."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [local]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, local, group=group)
    return out


def ensemble_share(n_particles, nbytes, rank, world, budget_bytes=None):
    """Indices of the ensemble systems rank `rank` advances: every system takes the same
    number of steps, so its work is its particle count.  Every rank computes the same
    partition from the same (seeded) ensemble, without communicating."""
    idx = list(range(len(n_particles)))
    return my_share(idx, [float(n) for n in n_particles], nbytes, rank, world, budget_bytes)


def combine_ensemble(per_rank):
    """Whole-job ensemble throughput from per-rank results {particles, steps, device_ms}:
    all ranks' particle-steps over the slowest rank's device time (ranks start together
    after a barrier and run no collective until they finish)."""
    work = float(sum(m["particles"] * m["steps"] for m in per_rank))
    tmax = max(m["device_ms"] for m in per_rank)
    return dict(systems=int(sum(m["systems"] for m in per_rank)), particles=int(sum(m["particles"] for m in per_rank)),
                particle_steps=work, device_ms_max=tmax, value=work / (tmax / 1000.0) if tmax > 0 else 0.0,
                ranks=len(per_rank))


def combine_serving(per_rank):
    """Whole-job serving metrics from per-rank ones: particle-steps over the longest
    rank's span; latency percentiles over all jobs."""
    lat = np.concatenate([np.asarray(m["latencies"], np.float64) for m in per_rank]) if per_rank else np.zeros(1)
    work = float(sum(m["particle_steps"] for m in per_rank))
    span = max(m["makespan_s"] for m in per_rank)
    return dict(jobs=int(sum(m["jobs"] for m in per_rank)), particle_steps=work, makespan_s=span,
                value=work / span if span > 0 else 0.0, p50_s=float(np.percentile(lat, 50)),
                p99_s=float(np.percentile(lat, 99)), ranks=len(per_rank))
