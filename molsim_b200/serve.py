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
* Iteration-level admission (`refill=True`): jobs in one cohort may have
  different step counts; a chunk never runs past the step at which one of them
  finishes, and that job's state is read out at that boundary (the handle keeps
  stepping it unread until the cohort is re-formed).  When jobs wait and every
  cohort slot is taken, one running cohort is drained to a chunk boundary and
  re-formed: a new handle holds its unfinished jobs (positions, velocities and
  accelerations carried over exactly) plus queued jobs that fit, and the old
  handle is retired.  So a finished job's place is refilled and a new job joins
  running work at the next boundary instead of waiting for a whole cohort.

Results (final positions, velocities and energies) are the same as running the
job alone: every per-system quantity is computed from that system's data
only, and the mixed-precision path sums in 64-bit fixed point, so the order in
which systems share a kernel does not change a bit.  A job carried into a
re-formed cohort gets a freshly built Verlet list and skin count there, so its
later steps sum its pairs in another order: its result then agrees with the
job alone to rounding (FP32 rounding in the mixed path), not bit for bit.

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
    left: int = None                   # steps still to run (None: nsteps)
    carry: dict = None                 # state carried into a re-formed cohort (ro, rod, rodd)

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
    """A cohort on the device: one batch handle, stepped asynchronously.

    Jobs may have different step counts: a chunk never runs past the step at which
    one of them finishes, and that job's state is read out at that boundary."""

    def __init__(self, jobs, precision, chunk, ahead=2):
        from .engine import Engine

        self.jobs = jobs
        self.chunk = chunk
        self.ahead = ahead
        systems = []
        for j in jobs:
            if j.left is None:
                j.left = j.nsteps
            st = j.carry
            systems.append(j.system if st is None else dict(j.system, ro=st["ro"], rod=st["rod"], rodd=st["rodd"]))
        self.eng = Engine(systems, [j.table for j in jobs], precision=precision)
        self.eng.UTotal(0)            # forces and energies of every system
        self.eng.GetLinAcc()
        for k, j in enumerate(jobs):
            if j.carry is not None:
                # the carried accelerations are the ones its last step left (not recomputed)
                self.eng.put_state(k, j.carry["ro"], j.carry["rod"], j.carry["rodd"], keep_list=True)
                j.carry = None
        self.unsent = [j.left for j in jobs]      # steps not yet enqueued, per job
        self.done = [False] * len(jobs)
        self.drain = False                        # stop enqueuing (a re-form is waiting)
        self.chunks_sent = 0
        self.nbytes = self.eng.device_bytes()
        self.finished = []

    def _boundary(self):
        """A job's steps are all enqueued but its state is not read out yet."""
        return any(u == 0 and not d for u, d in zip(self.unsent, self.done))

    def pump(self):
        """Keep up to `ahead` chunks in flight; read out jobs at their last step.  True
        once every job is read out."""
        pend = self.eng.pending()
        if pend == 0 and self._boundary():
            for k, j in enumerate(self.jobs):
                if self.unsent[k] == 0 and not self.done[k]:
                    st = self.eng.get_state(k)
                    j.left = 0
                    j.result = dict(ro=st["ro"], rod=st["rod"], energy=self.eng.energy(k))
                    self.done[k] = True
                    self.finished.append(j)
        while pend < self.ahead and not self.drain and not self._boundary():
            live = [u for u in self.unsent if u > 0]
            if not live:
                break
            k = min(self.chunk, min(live))
            self.eng.velver_async(k)
            self.unsent = [max(0, u - k) for u in self.unsent]
            self.chunks_sent += 1
            pend += 1
        return all(self.done) and pend == 0

    def idle(self):
        return self.eng.pending() == 0

    def take_finished(self):
        out, self.finished = self.finished, []
        return out

    def carry_out(self):
        """Unfinished jobs with their current state and remaining steps (the cohort is idle)."""
        out = []
        for k, j in enumerate(self.jobs):
            if self.done[k]:
                continue
            st = self.eng.get_state(k)
            j.left = self.unsent[k]
            j.carry = dict(ro=st["ro"], rod=st["rod"], rodd=st["rodd"])
            out.append(j)
        return out

    def harvest(self):
        return [j.result for j in self.jobs]

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
                 backend=None, clock=None, estimate=None, headroom=1.5, batch_wait_s=0.0, ahead=2,
                 refill=False):
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
        self.refill = refill
        self.reforms = 0
        self.joined = 0                 # queued jobs that joined a running cohort's work

    def _form(self, queue, free, head=None, room=None):
        """FIFO cohort: the head job and the queued jobs that can share its handle
        (same spline order; same step count unless cohorts refill), while the estimates
        fit `free`.  head/room: a re-formed cohort's first job and free job places."""
        head = head or queue[0]
        room = self.max_jobs if room is None else room
        take, tot = [], 0
        for j in queue:
            if len(take) >= room:
                break
            if j.order != head.order or (not self.refill and j.nsteps != head.nsteps):
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
                    c = self._make(take)
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
            # iteration-level admission: with jobs waiting and every slot taken, drain one
            # cohort to a chunk boundary and re-form it with the waiting jobs
            if self.refill and queue and len(running) >= self.max_cohorts:
                if not any(getattr(c, "drain", False) for c in running):
                    cand = [c for c in running if self._can_take(c, queue)]
                    if cand:
                        min(cand, key=lambda c: sum(1 for d in c.done if not d)).drain = True
            # progress and completion
            still = []
            progressed = False
            for c in running:
                try:
                    complete = c.pump()
                except Exception as exc:          # a device error in this cohort: fail its jobs
                    self._fail([j for j in c.jobs if j.done is None], exc, self.clock() - t0, finished)
                    c.close()
                    self.used -= c.reserved
                    self.device_now -= getattr(c, "nbytes", 0)
                    progressed = True
                    continue
                if hasattr(c, "take_finished"):
                    tdone = self.clock() - t0
                    for j in c.take_finished():
                        j.done = tdone
                        finished.append(j)
                        progressed = True
                if complete:
                    tdone = self.clock() - t0
                    if not hasattr(c, "take_finished"):
                        for j, r in zip(c.jobs, c.harvest()):
                            j.result = r
                            j.done = tdone
                            finished.append(j)
                    c.close()
                    self.used -= c.reserved
                    self.device_now -= getattr(c, "nbytes", 0)
                    progressed = True
                elif getattr(c, "drain", False) and c.idle():
                    c2, queue = self._reform(c, queue, finished, t0)
                    progressed = True
                    if c2 is not None:
                        still.append(c2)
                else:
                    still.append(c)
            running = still
            if not progressed and poll_s:
                time.sleep(poll_s)
        return self.metrics(finished)

    def _can_take(self, c, queue):
        """Whether re-forming cohort c would admit a queued job: it has run at least one
        chunk since it was formed, has a free job place, and the first queued job of its
        spline order fits the budget its finished jobs free."""
        if not hasattr(c, "carry_out") or getattr(c, "chunks_sent", 1) < 1:
            return False
        live = [j for j, d in zip(c.jobs, c.done) if not d]
        if len(live) >= self.max_jobs:
            return False
        free = self.budget - self.used + c.reserved - sum(j.nbytes for j in live)
        head = live[0] if live else queue[0]
        for j in queue:
            if j.order == head.order:
                return j.nbytes <= free
        return False

    def _make(self, jobs):
        """A cohort of the backend; backends that step jobs of different lengths and can be
        re-formed (GpuCohort, or one marked `refillable`) also take the enqueue depth."""
        if self.backend is GpuCohort or getattr(self.backend, "refillable", False):
            return self.backend(jobs, self.precision, self.chunk, self.ahead)
        return self.backend(jobs, self.precision, self.chunk)

    def _reform(self, c, queue, finished, t0):
        """Replace the idle cohort c by a new handle holding its unfinished jobs (state
        carried over) and queued jobs that fit the freed budget and job places.
        Returns (new cohort or None, queue)."""
        keep = c.carry_out()
        self.used -= c.reserved
        self.device_now -= getattr(c, "nbytes", 0)
        c.close()
        tot = sum(j.nbytes for j in keep)
        take = []
        if queue:
            head = keep[0] if keep else queue[0]
            take, t_new = self._form(queue, self.budget - self.used - tot, head=head,
                                     room=self.max_jobs - len(keep))
            tot += t_new
            ids = set(id(j) for j in take)
            queue = [j for j in queue if id(j) not in ids]
        members = keep + take
        if not members:
            return None, queue
        tadm = self.clock() - t0
        try:
            c2 = self._make(members)
        except Exception as exc:
            self._fail(members, exc, self.clock() - t0, finished)
            return None, queue
        c2.cid = self.ncohorts
        c2.reserved = max(tot, getattr(c2, "nbytes", 0))
        self.device_now += getattr(c2, "nbytes", 0)
        self.peak_device = max(self.peak_device, self.device_now)
        self.ncohorts += 1
        self.cohort_sizes.append(len(members))
        self.used += c2.reserved
        self.peak_used = max(self.peak_used, self.used)
        self.reforms += 1
        self.joined += len(take)
        for j in take:
            j.admitted = tadm
        for j in members:
            j.cohort = c2.cid
        return c2, queue

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
                    peak_device_bytes=self.peak_device, budget_bytes=self.budget, reforms=self.reforms,
                    joined_running=self.joined)


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
