"""Continuous-batching service for MD jobs of different sizes.

MOLSIM runs one system per process (Src/molsim.F90 main loop: one
configuration, MDDriver per step).  This module serves a stream of such jobs
on one GPU.  A job is one system (any size) with its pair table and a step
count.  Jobs arrive over time; the server admits them while the device-memory
budget allows, keeps their state resident, and advances them batched:

* A *cohort* is the set of jobs admitted together.  It lives in one library
  handle (`msg_create_batch`), so every step of all its systems is one CUDA
  graph replay (one launch per kernel for all systems).
* Cohorts run concurrently, each on its own stream, so jobs that arrive while
  others are on the GPU start as soon as a cohort slot and memory free up;
  their work overlaps on the device with the running cohorts.
* Memory: each job's footprint comes from `msg_estimate_bytes` (a dry set-up)
  when it arrives; a cohort is admitted when the sum fits the free budget.
  Handles allocate and free stream-ordered, so creating or retiring a cohort
  does not wait for the others.
* Steps are enqueued in chunks (`msg_velver_async`), at most two chunks ahead
  per cohort, so the host never blocks on a full launch queue.

Results (final positions, velocities and energies) are the same as running the
job alone: every per-system quantity is computed from that system's data
only, and the mixed-precision path sums in 64-bit fixed point, so the order in
which systems share a kernel does not change a bit.

The `backend` argument lets the host logic (admission, grouping, budget
accounting, latency bookkeeping) run without a GPU: tests pass a simulated
cohort class with the same methods.
"""
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Job:
    jid: int
    system: dict
    table: dict
    nsteps: int
    arrival: float                     # seconds after the stream starts
    nbytes: int = 0                    # device bytes estimated for the job alone
    admitted: float = None
    done: float = None
    cohort: int = -1
    result: dict = field(default_factory=dict)
    error: str = ""

    @property
    def n(self):
        return int(self.system["np"])

    @property
    def order(self):
        return int(self.system["order"])

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


class GpuCohort:
    """A cohort on the device: one batch handle, stepped asynchronously."""

    def __init__(self, jobs, precision, chunk, ahead=2):
        from .engine import Engine

        self.jobs = jobs
        self.chunk = chunk
        self.ahead = ahead
        self.eng = Engine([j.system for j in jobs], [j.table for j in jobs], precision=precision)
        self.eng.UTotal(0)            # forces and energies of every system
        self.eng.GetLinAcc()
        self.left = jobs[0].nsteps
        self.nbytes = self.eng.device_bytes()

    def pump(self):
        """Keep up to `ahead` chunks in flight; True once every step has run."""
        pend = self.eng.pending()
        while self.left > 0 and pend < self.ahead:
            k = min(self.chunk, self.left)
            self.eng.velver_async(k)
            self.left -= k
            pend += 1
        return self.left == 0 and pend == 0

    def harvest(self):
        out = []
        for k, _j in enumerate(self.jobs):
            st = self.eng.get_state(k)
            out.append(dict(ro=st["ro"], rod=st["rod"], energy=self.eng.energy(k)))
        return out

    def close(self):
        self.eng = None


class Server:
    """Admission by memory budget, cohorts of queued jobs, concurrent cohorts.

    budget_bytes: device bytes the server may hold across all resident jobs.
    max_cohorts:  cohorts resident at once (streams in use).
    max_jobs:     jobs per cohort.
    chunk:        steps per asynchronous enqueue.
    batch_wait_s: batching window: a cohort is formed once the queue holds max_jobs
                  jobs, its head job has waited this long, or no arrivals remain (0: at once).
    ahead:        step chunks each cohort keeps enqueued.
    headroom:     factor on each job's set-up estimate reserved at admission; the
                  Verlet rows may grow past their initial capacity (x1.5 of the longest
                  row) when the first list is built.  Once a cohort exists its reservation
                  is the larger of that and the bytes its handle really holds.
    """

    def __init__(self, budget_bytes, precision="mixed", max_cohorts=8, max_jobs=64, chunk=50,
                 backend=None, clock=None, estimate=None, headroom=1.5, batch_wait_s=0.0, ahead=2):
        self.budget = int(budget_bytes)
        self.precision = precision
        self.max_cohorts = max_cohorts
        self.max_jobs = max_jobs
        self.chunk = chunk
        self.backend = backend or GpuCohort
        self.clock = clock or time.perf_counter
        if estimate is None:
            from .engine import estimate_bytes

            def estimate(job):
                return estimate_bytes(job.system, job.table, precision)
        self.estimate = estimate
        self.headroom = headroom
        self.batch_wait_s = batch_wait_s
        self.ahead = ahead
        self.used = 0
        self.device_now = 0
        self.peak_device = 0
        self.peak_used = 0
        self.ncohorts = 0
        self.cohort_sizes = []
        self.max_concurrent = 0

    def _form(self, queue, free):
        """FIFO cohort: the head job and the queued jobs that can share its handle
        (same step count and spline order), while the estimates fit `free`."""
        head = queue[0]
        take, tot = [], 0
        for j in queue:
            if len(take) >= self.max_jobs:
                break
            if j.nsteps != head.nsteps or j.order != head.order:
                continue
            if tot + j.nbytes > free:
                if not take:
                    return [], 0
                continue
            take.append(j)
            tot += j.nbytes
        return take, tot

    def run(self, jobs, realtime=True, poll_s=2e-4):
        """Serve `jobs` (arrival times relative to the start); returns the metrics dict.
        realtime=False admits every job at t=0 (a closed batch)."""
        pending = sorted(jobs, key=lambda j: j.arrival)
        queue, running, finished = [], [], []
        t0 = self.clock()
        now = 0.0
        ia = 0
        while ia < len(pending) or queue or running:
            now = self.clock() - t0
            while ia < len(pending) and (not realtime or pending[ia].arrival <= now):
                j = pending[ia]
                ia += 1
                j.nbytes = int(self.headroom * self.estimate(j))
                if j.nbytes > self.budget:
                    j.error = "job needs %d bytes, budget is %d" % (j.nbytes, self.budget)
                    j.done = now
                    finished.append(j)
                    continue
                queue.append(j)
            # admission
            while queue and len(running) < self.max_cohorts:
                if (self.batch_wait_s > 0 and ia < len(pending) and len(queue) < self.max_jobs
                        and now - queue[0].arrival < self.batch_wait_s):
                    break                           # batching window still open
                take, tot = self._form(queue, self.budget - self.used)
                if not take:
                    break
                ids = set(id(j) for j in take)
                queue = [j for j in queue if id(j) not in ids]
                tadm = self.clock() - t0
                try:
                    c = self.backend(take, self.precision, self.chunk, self.ahead) \
                        if self.backend is GpuCohort else self.backend(take, self.precision, self.chunk)
                except Exception as exc:          # set-up failed: these jobs fail, the server goes on
                    self._fail(take, exc, self.clock() - t0, finished)
                    continue
                c.cid = self.ncohorts
                c.reserved = max(tot, getattr(c, "nbytes", 0))
                self.device_now += getattr(c, "nbytes", 0)
                self.peak_device = max(self.peak_device, self.device_now)
                self.ncohorts += 1
                self.cohort_sizes.append(len(take))
                self.used += c.reserved
                self.peak_used = max(self.peak_used, self.used)
                for j in take:
                    j.admitted = tadm
                    j.cohort = c.cid
                running.append(c)
            self.max_concurrent = max(self.max_concurrent, len(running))
            # progress and completion
            still = []
            progressed = False
            for c in running:
                try:
                    complete = c.pump()
                except Exception as exc:          # a device error in this cohort: fail its jobs
                    self._fail(c.jobs, exc, self.clock() - t0, finished)
                    c.close()
                    self.used -= c.reserved
                    self.device_now -= getattr(c, "nbytes", 0)
                    progressed = True
                    continue
                if complete:
                    res = c.harvest()
                    tdone = self.clock() - t0
                    for j, r in zip(c.jobs, res):
                        j.result = r
                        j.done = tdone
                        finished.append(j)
                    c.close()
                    self.used -= c.reserved
                    self.device_now -= getattr(c, "nbytes", 0)
                    progressed = True
                else:
                    still.append(c)
            running = still
            if not progressed and poll_s:
                time.sleep(poll_s)
        return self.metrics(finished)

    @staticmethod
    def _fail(jobs, exc, now, finished):
        for j in jobs:
            j.error = "%s: %s" % (type(exc).__name__, exc)
            j.done = now
            finished.append(j)

    def metrics(self, finished):
        ok = [j for j in finished if not j.error]
        lat = np.array([j.latency for j in ok]) if ok else np.zeros(1)
        t_first = min(j.arrival for j in finished) if finished else 0.0
        t_last = max(j.done for j in finished) if finished else 0.0
        work = float(sum(j.n * j.nsteps for j in ok))
        span = max(t_last - t_first, 1e-12)
        return dict(jobs=len(finished), failed=len(finished) - len(ok),
                    p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                    mean_s=float(lat.mean()), makespan_s=span, particle_steps=work,
                    value=work / span, cohorts=self.ncohorts,
                    mean_cohort_jobs=float(np.mean(self.cohort_sizes)) if self.cohort_sizes else 0.0,
                    latencies=[float(x) for x in lat] if ok else [],
                    max_concurrent_cohorts=self.max_concurrent, peak_reserved_bytes=self.peak_used,
                    peak_device_bytes=self.peak_device, budget_bytes=self.budget)


def poisson_stream(seed=0, rate=200.0, njobs=200, nmin=100, nmax=20000, nsteps=1000, order=4):
    """Seeded job stream: Poisson arrivals at `rate` jobs/s, N log-uniform over [nmin, nmax],
    half electrolytes and half polyelectrolytes (the two generators scaled to N)."""
    from .engine import prepare
    from .systems import scaled_job

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=njobs))
    t -= t[0]
    jobs = []
    tabcache = {}
    for k in range(njobs):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        n = max(nmin, n + (n & 1))
        kind = "electrolyte" if rng.uniform() < 0.5 else "polyelectrolyte"
        s = scaled_job(rng, n, kind, order=order)
        key = (kind, round(s["rcut"], 9), round(float(np.mean(np.asarray(s["az"]) ** 2)), 9), s["boxlen"][0])
        tab = tabcache.get(key)
        if tab is None:
            tab = prepare(s)
            tabcache[key] = tab
        jobs.append(Job(k, s, tab, nsteps, float(t[k])))
    return jobs
