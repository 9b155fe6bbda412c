"""Sharding independent systems across ranks: the assignment on its own, and a
world-size-2 gloo run of the serving loop (simulated cohorts) on the CPU."""
import os
import socket

import numpy as np
import pytest

from molsim_b200.shard import assign, combine_serving, my_share


def test_assignment_balances_and_covers():
    rng = np.random.default_rng(0)
    work = rng.integers(100, 20000, size=200) * 1000
    nb = rng.integers(1, 100, size=200)
    a = assign(work, nb, 4)
    assert set(a.tolist()) == {0, 1, 2, 3}
    loads = np.array([work[a == r].sum() for r in range(4)])
    # LPT is within 4/3 of optimal; the mean is a lower bound of the optimum
    assert loads.max() <= 4.0 / 3.0 * max(loads.mean(), work.max()) + 1
    # deterministic: same inputs, same answer on every rank
    assert np.array_equal(a, assign(work, nb, 4))


def test_assignment_respects_budget():
    work = [10, 9, 8, 7, 6, 5]
    nb = [60, 50, 40, 30, 20, 10]
    a = assign(work, nb, 2, budget_bytes=110)
    for r in range(2):
        assert sum(b for b, x in zip(nb, a) if x == r) <= 110
    with pytest.raises(ValueError):
        assign([1, 1], [200, 1], 2, budget_bytes=100)


def test_shares_are_disjoint_and_complete():
    items = list(range(37))
    work = [(k * 7919) % 101 + 1 for k in items]
    nb = [1] * len(items)
    shares = [my_share(items, work, nb, r, 3) for r in range(3)]
    flat = sorted(x for s in shares for x in s)
    assert flat == items


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from molsim_b200.serve import Job, Server
    from molsim_b200.shard import gather_metrics
    from test_serve import FakeCohort, TickClock

    rng = np.random.default_rng(7)
    jobs = []
    for k in range(24):
        j = Job(k, dict(np=int(rng.integers(100, 2000)), order=4), {}, 20, 0.001 * k)
        j.nbytes = int(j.n) * 10
        jobs.append(j)
    mine = my_share(jobs, [j.n * j.nsteps for j in jobs], [j.nbytes for j in jobs], rank, world)
    srv = Server(1 << 20, backend=FakeCohort, clock=TickClock(), estimate=lambda j: j.nbytes, chunk=5)
    m = srv.run(mine, poll_s=0)
    m["ids"] = sorted(j.jid for j in mine)
    allm = gather_metrics(m)
    if rank == 0:
        ids = sorted(i for mm in allm for i in mm["ids"])
        comb = combine_serving(allm)
        out.put((ids, comb["jobs"], comb["particle_steps"], sum(j.n * 20 for j in jobs)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_serving_partition():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ids, njobs, work, want = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert ids == list(range(24))
    assert njobs == 24
    assert work == want


def _ensemble_rank_main(rank, world, port, out):
    """One rank of the bench's ensemble partition: its share of a seeded ensemble, a
    simulated device time proportional to its particles, metrics gathered and combined."""
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from molsim_b200.shard import combine_ensemble, ensemble_share, gather_metrics

    rng = np.random.default_rng(3)
    npart = [int(x) for x in rng.integers(100, 2000, size=40) * 2]
    nbytes = [n * 1000 for n in npart]
    mine = ensemble_share(npart, nbytes, rank, world)
    steps = 10
    local = {"systems": len(mine), "particles": sum(npart[k] for k in mine), "steps": steps,
             "device_ms": 1e-3 * sum(npart[k] for k in mine), "ids": mine}
    per = gather_metrics(local)
    if rank == 0:
        out.put((sorted(i for m in per for i in m["ids"]), combine_ensemble(per), npart,
                 [m["device_ms"] for m in per]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_ensemble_partition():
    """The ensemble leg of bench.py under torchrun: the ranks' shares cover every system
    once, the loads balance, and the whole-job value is all particle-steps over the
    slowest rank's time."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ensemble_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ids, comb, npart, times = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert ids == list(range(40))
    assert comb["systems"] == 40 and comb["particles"] == sum(npart) and comb["ranks"] == 2
    assert max(times) <= 1.05 * min(times)
    assert abs(comb["value"] - sum(npart) * 10 / (max(times) / 1000.0)) <= 1e-6 * comb["value"]
