"""Continuous-batching MD job server on one GPU.

Jobs (independent MD systems of any size and step count) arrive over time.
The server keeps every admitted job's state resident in HBM as a replica of
one engine, admits queued jobs as soon as the memory budget allows, and
advances all resident jobs together: each round is one `run_queued` call of
`chunk_steps` steps in which every replica advances by up to that many of its
own remaining steps.  Jobs that finish leave between rounds, which frees
their slot and memory for the next queued jobs.  Because a replica's
arithmetic does not depend on which other replicas share the launches, every
job's result is the same alone and in the mix.

`MDServer` takes the engine as an argument, so the scheduling logic runs
unchanged against a fake engine in the CPU tests.
"""
import time
from dataclasses import dataclass, field

import numpy as np

from . import initconf

# Device bytes per particle held by an engine replica: positions/velocities/
# images/ids double-buffered, forces, virials, stresses, last-build positions,
# list length, sort scratch.
BYTES_PER_PARTICLE = 2 * (16 + 16 + 16 + 4) + 16 * 4 + 4 * 4


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


def job_bytes(job, skin=0.3):
    """HBM needed by a job: particle arrays + neighbour list + cell arrays."""
    density = 1.2 if job.kind == "KA" else 0.8442
    rc = 2.5
    max_nbrs = int(np.ceil(1.5 * 4.0 / 3.0 * np.pi * (rc + skin) ** 3 * density)) + 1
    cells = (job.n / density) / ((rc + skin) / 2) ** 3
    return int(job.n * (BYTES_PER_PARTICLE + 4 * max_nbrs) + 8 * cells + 4096)


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


def job_config(job):
    """Initial configuration and parameter table of a job."""
    if job.kind == "KA":
        c = initconf.ka_config(job.n, T=job.T, seed=job.seed)
        return c, initconf.lj_params(2, initconf.KA), 2
    c = initconf.lj_config(job.n, T=job.T, seed=job.seed)
    return c, initconf.lj_params(1, initconf.LJ), 1


class MDServer:
    def __init__(self, engine, hbm_budget=150e9, chunk_steps=200, dt=0.005, skin=0.3, tau=0.2,
                 clock=time.perf_counter, sleep=time.sleep):
        self.engine = engine
        self.budget = float(hbm_budget)
        self.chunk = int(chunk_steps)
        self.dt, self.skin, self.tau = dt, skin, tau
        self.clock, self.sleep = clock, sleep
        self.used = 0
        self.max_used = 0
        self.running = {}     # replica id -> (job, remaining steps)
        self.queue_depth = []

    def admit(self, job, now):
        c, params, ntypes = job_config(job)
        rid = self.engine.add(c["pos4"], c["box"], params, ntypes, cutoff="SF", skin=self.skin, dt=self.dt,
                              T=job.T, tau=self.tau, vel4=c["vel4"])
        self.engine.queue(rid, job.steps)
        self.used += job_bytes(job, self.skin)
        self.max_used = max(self.max_used, self.used)
        job.admitted = now
        self.running[rid] = [job, job.steps]

    def retire(self, rid, now):
        job, _ = self.running.pop(rid)
        st = self.engine.stats(rid)
        job.result = {"pe": st["pe"], "ke": st["ke"], "xi": st["xi"], "steps": st["steps"],
                      "rebuilds": st["rebuilds"]}
        job.done = now
        self.engine.remove(rid)
        self.used -= job_bytes(job, self.skin)

    def serve(self, jobs, realtime=True):
        """Runs the whole stream; returns the jobs with admitted/done times set."""
        pending = sorted(jobs, key=lambda j: j.arrival)
        for j in pending:
            if job_bytes(j, self.skin) > self.budget:
                raise ValueError(f"job {j.id} needs more memory than the whole budget")
        t0 = self.clock()
        k = 0
        waiting = []
        while k < len(pending) or waiting or self.running:
            now = self.clock() - t0 if realtime else float("inf")
            while k < len(pending) and pending[k].arrival <= now:
                waiting.append(pending[k])
                k += 1
            # FIFO admission while the budget allows
            while waiting and self.used + job_bytes(waiting[0], self.skin) <= self.budget:
                self.admit(waiting.pop(0), self.clock() - t0)
            self.queue_depth.append(len(waiting))
            if not self.running:
                if k < len(pending):
                    self.sleep(max(0.0, pending[k].arrival - (self.clock() - t0)))
                continue
            ran = self.engine.run_queued(self.chunk)
            now = self.clock() - t0
            for rid in list(self.running):
                self.running[rid][1] -= ran
                if self.running[rid][1] <= 0:
                    if self.engine.stats(rid)["steps_left"] <= 0:
                        self.retire(rid, now)
                    else:
                        self.running[rid][1] = int(self.engine.stats(rid)["steps_left"])
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
