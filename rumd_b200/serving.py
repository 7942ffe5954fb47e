"""Continuous-batching MD job server on one GPU.

Jobs (independent MD systems of any size and step count) arrive over time.
The server keeps every admitted job's state resident in HBM as a replica of
one engine and advances all resident jobs together in chunks: each chunk is
one `run_queued_async` launch in which every replica advances by up to the
chunk's step count of its own remaining steps.  Two chunks are kept in
flight, so the GPU never waits for the host:

  * arrivals: a job's initial configuration is built on a worker thread as
    soon as it arrives (the stand-in for a client uploading it), off the
    serving loop;
  * admission, FIFO: the head of the queue is admitted when its configuration
    is ready and the engine's reported memory (`usage`) plus the job's
    `footprint` fits the HBM budget.  `add` only queues the upload behind the
    running chunks and returns; the job joins the next chunk launched;
  * completion: each chunk leaves a snapshot of every replica's state in
    pinned host memory; when the oldest chunk finishes the server reads it,
    retires the jobs it shows finished (results from the snapshot) and
    removes them, which returns their memory at once, and launches the next
    chunk.

Because a replica's arithmetic does not depend on which other replicas share
the launches, every job's result is the same alone and in the mix.

`MDServer` takes the engine as an argument, so the scheduling logic runs
unchanged against a fake engine in the CPU tests.
"""
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import initconf

DENSITY = {"KA": 1.2, "LJ": 0.8442}
# snapshot columns (capi.CHUNK_FIELDS)
SNAP = {k: i for i, k in enumerate(["active", "steps", "steps_left", "pe", "virial", "ke", "xi", "rebuilds",
                                     "overflow"])}


@dataclass
class Job:
    id: int
    kind: str            # "KA" or "LJ"
    n: int
    T: float
    steps: int
    arrival: float       # seconds after the start of the stream
    seed: int = 0
    admitted: float = -1.0
    done: float = -1.0
    result: dict = field(default_factory=dict)

    @property
    def latency(self):
        return self.done - self.arrival


def poisson_stream(njobs, rate=50.0, seed=0, n_range=(256, 32768), steps_range=(1000, 100000),
                   T_range=(0.5, 2.0)):
    """Seeded job stream: Poisson arrivals at `rate` jobs/s, KA or LJ 50/50,
    N and steps log-uniform, T uniform."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, njobs))
    kinds = np.where(rng.random(njobs) < 0.5, "KA", "LJ")
    ns = np.floor(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]), njobs))).astype(int)
    steps = np.floor(np.exp(rng.uniform(np.log(steps_range[0]), np.log(steps_range[1]), njobs))).astype(int)
    Ts = rng.uniform(T_range[0], T_range[1], njobs)
    return [Job(id=k, kind=str(kinds[k]), n=int(ns[k]), T=float(Ts[k]), steps=int(steps[k]), arrival=float(t[k]),
                seed=seed * 100003 + k) for k in range(njobs)]


def job_params(job):
    if job.kind == "KA":
        return initconf.lj_params(2, initconf.KA), 2
    return initconf.lj_params(1, initconf.LJ), 1


def job_config(job):
    """Initial configuration and parameter table of a job."""
    params, ntypes = job_params(job)
    if job.kind == "KA":
        return initconf.ka_config(job.n, T=job.T, seed=job.seed), params, ntypes
    return initconf.lj_config(job.n, T=job.T, seed=job.seed), params, ntypes


def job_box(job):
    """The job's cubic box (the configuration's density)."""
    L = (job.n / DENSITY[job.kind]) ** (1.0 / 3.0)
    return np.array([L, L, L], np.float32)


class _Ready:
    """A finished result in the shape of a Future (configurations built inline)."""

    def __init__(self, value):
        self.value = value

    def done(self):
        return True

    def result(self):
        return self.value


@dataclass
class _Resident:
    job: Job
    left: int                  # steps left, from the latest snapshot that includes the job
    first_ticket: int = 0      # the first chunk launched after the admission (0: none yet)


class MDServer:
    """chunk_steps: steps per chunk, or "auto": about `chunk_seconds` of GPU
    time at `rate_hint` particle-steps/s over the resident particles (between
    min_chunk_steps and max_chunk_steps).  workers: threads that build
    arriving jobs' configurations (0: inline).  max_resident: replicas at
    once (the batched kernel's limit)."""

    def __init__(self, engine, hbm_budget=150e9, chunk_steps="auto", dt=0.005, skin=0.3, tau=0.2,
                 clock=time.perf_counter, sleep=time.sleep, workers=2, max_resident=1024, chunk_seconds=0.05,
                 rate_hint=1.5e9, min_chunk_steps=16, max_chunk_steps=2000, poll_seconds=2e-4, in_flight=2):
        self.engine = engine
        self.budget = float(hbm_budget)
        self.chunk = chunk_steps
        self.dt, self.skin, self.tau = dt, skin, tau
        self.clock, self.sleep = clock, sleep
        self.workers = int(workers)
        self.max_resident = int(max_resident)
        self.chunk_seconds, self.rate_hint = chunk_seconds, rate_hint
        self.min_chunk, self.max_chunk = int(min_chunk_steps), int(max_chunk_steps)
        self.poll_seconds = poll_seconds
        self.in_flight = int(in_flight)
        self.max_used = 0
        self.running = {}      # replica id -> _Resident
        # after each chunk: (t, jobs waiting, jobs resident, backlog particle-steps,
        # resident particles with steps left, steps the chunk ran)
        self.timeline = []
        self.chunks = 0

    # ---- memory ----
    @property
    def used(self):
        return self.engine.usage()[0]

    def job_footprint(self, job):
        """Device bytes the engine reports for the job (box from its density)."""
        params, ntypes = job_params(job)
        return self.engine.footprint(job.n, job_box(job), params, ntypes, cutoff="SF", skin=self.skin)

    # ---- jobs ----
    def admit(self, job, conf, now):
        c, params, ntypes = conf
        rid = self.engine.add(c["pos4"], c["box"], params, ntypes, cutoff="SF", skin=self.skin, dt=self.dt,
                              T=job.T, tau=self.tau, vel4=c["vel4"])
        self.engine.queue(rid, job.steps)
        job.admitted = now
        self.running[rid] = _Resident(job, job.steps)
        self.max_used = max(self.max_used, self.used)

    def retire(self, rid, row, now):
        job = self.running.pop(rid).job
        job.result = {"pe": float(row[SNAP["pe"]]), "ke": float(row[SNAP["ke"]]), "xi": float(row[SNAP["xi"]]),
                      "steps": int(row[SNAP["steps"]]), "rebuilds": int(row[SNAP["rebuilds"]])}
        job.done = now
        self.engine.remove(rid)

    def chunk_length(self):
        if self.chunk != "auto":
            return int(self.chunk)
        parts = sum(r.job.n for r in self.running.values() if r.left > 0)
        k = int(self.chunk_seconds * self.rate_hint / max(parts, 1))
        return max(self.min_chunk, min(self.max_chunk, k))

    def _after_chunk(self, ticket, snap, now, waiting, ran=0):
        parts = sum(r.job.n for r in self.running.values() if r.left > 0)
        for rid, r in list(self.running.items()):
            if r.first_ticket == 0 or ticket < r.first_ticket:
                continue  # admitted after this chunk was launched
            row = snap[rid]
            r.left = int(row[SNAP["steps_left"]])
            if r.left <= 0:
                self.retire(rid, row, now)
        backlog = sum(r.left * r.job.n for r in self.running.values()) + sum(j.n * j.steps for j in waiting)
        self.timeline.append((now, len(waiting), len(self.running), float(backlog), parts, int(ran)))

    @property
    def queue_depth(self):
        """Jobs waiting for admission, after each chunk."""
        return [row[1] for row in self.timeline]

    def serve(self, jobs, realtime=True):
        """Runs the whole stream; returns the jobs with admitted/done times set."""
        pending = sorted(jobs, key=lambda j: j.arrival)
        for j in pending:
            if self.job_footprint(j) > self.budget:
                raise ValueError(f"job {j.id} needs more memory than the whole budget")
        pool = ThreadPoolExecutor(self.workers) if self.workers > 0 else None
        confs = {}
        waiting = deque()
        inflight = deque()
        t0 = self.clock()
        k = 0
        try:
            while k < len(pending) or waiting or self.running or inflight:
                now = self.clock() - t0 if realtime else float("inf")
                while k < len(pending) and pending[k].arrival <= now:
                    j = pending[k]
                    k += 1
                    waiting.append(j)
                    confs[j.id] = pool.submit(job_config, j) if pool else _Ready(job_config(j))
                # FIFO admission: the head waits for its configuration and for room
                while waiting and len(self.running) < self.max_resident and confs[waiting[0].id].done():
                    j = waiting[0]
                    conf = confs[j.id].result()
                    c, params, ntypes = conf
                    need = self.engine.footprint(len(c["pos4"]), c["box"], params, ntypes, cutoff="SF",
                                                 skin=self.skin)
                    if self.used + need > self.budget:
                        break
                    waiting.popleft()
                    del confs[j.id]
                    self.admit(j, conf, self.clock() - t0)
                # keep the GPU fed: chunks in flight while any resident job has steps left
                while len(inflight) < self.in_flight and any(r.left > 0 for r in self.running.values()):
                    t = self.engine.run_queued_async(self.chunk_length())
                    self.chunks += 1
                    inflight.append(t)
                    for r in self.running.values():
                        if r.first_ticket == 0:
                            r.first_ticket = t
                if inflight:
                    if self.engine.poll(inflight[0]):
                        t = inflight.popleft()
                        ran, snap = self.engine.wait(t)
                        self._after_chunk(t, snap, self.clock() - t0, waiting, ran)
                    else:
                        self.sleep(self.poll_seconds)
                elif waiting:
                    self.sleep(self.poll_seconds)  # the head's configuration is still being built
                elif k < len(pending):
                    self.sleep(max(0.0, pending[k].arrival - (self.clock() - t0)))
        finally:
            if pool:
                pool.shutdown(wait=True)
        return jobs


def shard(jobs, rank, world):
    """Deterministic split of independent jobs over `world` GPUs (one process
    per GPU, no data exchange): longest-processing-time-first by n*steps,
    ties by job id.  Returns this rank's jobs."""
    loads = [0.0] * world
    mine = []
    for j in sorted(jobs, key=lambda j: (-j.n * j.steps, j.id)):
        r = min(range(world), key=lambda q: (loads[q], q))
        loads[r] += j.n * j.steps
        if r == rank:
            mine.append(j)
    return sorted(mine, key=lambda j: j.arrival)


def latency_summary(jobs):
    lat = np.array([j.latency for j in jobs])
    ps = float(sum(j.n * j.steps for j in jobs))
    span = max(j.done for j in jobs) - min(j.arrival for j in jobs)
    return {"jobs": len(jobs), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "particle_steps": ps, "makespan_s": span,
            "throughput": ps / span if span > 0 else 0.0}


def timeline_summary(server, jobs, step_s=1.0):
    """Load over time: per `step_s` window, the largest number of jobs waiting
    for admission and resident, the backlog (particle-steps still to run) at
    the window's end, the resident particles with steps left and the mean
    time of a step of the chunks that ended in the window; with the offered
    load."""
    tl = server.timeline
    if not tl:
        return {}
    end = tl[-1][0]
    rows = []
    i = 0
    for w in range(int(np.ceil(end / step_s)) + 1):
        hi = (w + 1) * step_s
        sel = []
        while i < len(tl) and tl[i][0] < hi:
            sel.append(tl[i])
            i += 1
        if sel:
            steps = sum(s[5] for s in sel)
            t_lo = tl[i - len(sel) - 1][0] if i - len(sel) - 1 >= 0 else 0.0
            step_us = (sel[-1][0] - t_lo) / steps * 1e6 if steps else None
            rows.append([round(hi, 3), max(s[1] for s in sel), max(s[2] for s in sel), sel[-1][3],
                         max(s[4] for s in sel), None if step_us is None else round(step_us, 1)])
    arrivals = [j.arrival for j in jobs]
    span = max(arrivals) - min(arrivals)
    work = float(sum(j.n * j.steps for j in jobs))
    return {"window_s": step_s, "columns": ["t_s", "max_waiting", "max_resident", "backlog_particle_steps",
                                            "max_resident_particles", "us_per_step"],
            "rows": rows, "arrival_span_s": span, "offered_particle_steps_per_s": work / span if span > 0 else None,
            "max_waiting": max(s[1] for s in tl), "max_resident": max(s[2] for s in tl), "chunks": server.chunks}


def serve_one_at_a_time(engine_factory, jobs, dt=0.005, skin=0.3, tau=0.2, clock=time.perf_counter,
                        sleep=time.sleep):
    """The plain loop: one job on the GPU at a time, in arrival order."""
    t0 = clock()
    for job in sorted(jobs, key=lambda j: j.arrival):
        now = clock() - t0
        if job.arrival > now:
            sleep(job.arrival - now)
        e = engine_factory()
        c, params, ntypes = job_config(job)
        job.admitted = clock() - t0
        rid = e.add(c["pos4"], c["box"], params, ntypes, cutoff="SF", skin=skin, dt=dt, T=job.T, tau=tau,
                    vel4=c["vel4"])
        e.queue(rid, job.steps)
        e.run_queued(0)
        st = e.stats(rid)
        job.result = {"pe": st["pe"], "ke": st["ke"], "xi": st["xi"], "steps": st["steps"],
                      "rebuilds": st["rebuilds"]}
        job.done = clock() - t0
        e.close()
    return jobs
