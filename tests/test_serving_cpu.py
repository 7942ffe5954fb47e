"""Serving scheduler and multi-GPU sharding host logic, on the CPU.

The engine is replaced by a fake that advances step counters; the clock is a
virtual clock driven by the fake's work, so the tests are deterministic."""
import os

import numpy as np
import pytest


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, s):
        self.t += max(0.0, s)


class FakeEngine:
    """The engine calls the server makes, on a virtual clock.  A chunk runs
    when it is launched: every replica advances by up to its step count, and
    the clock advances by a fixed launch cost per step (what a small system
    alone is bound by) plus the particle-steps of all replicas at `rate`.
    Memory: 600 bytes per particle."""

    BYTES_PER_PARTICLE = 600

    def __init__(self, clock, rate=1e9):
        self.clock, self.rate = clock, rate
        self.reps, self.free = {}, []
        self.max_live = 0
        self.tickets = 0
        self.snaps = {}

    def footprint(self, n, box, params, ntypes, **kw):
        return n * self.BYTES_PER_PARTICLE

    def usage(self):
        return sum(r["n"] for r in self.reps.values()) * self.BYTES_PER_PARTICLE, 0

    def add(self, pos4, box, params, ntypes, **kw):
        rid = min(self.free) if self.free else len(self.reps)
        if rid in self.free:
            self.free.remove(rid)
        self.reps[rid] = {"n": len(pos4), "left": 0, "steps": 0}
        self.max_live = max(self.max_live, len(self.reps))
        return rid

    def queue(self, rid, k):
        self.reps[rid]["left"] += k

    def run_queued(self, k):
        todo = min(max([r["left"] for r in self.reps.values()] + [0]), k if k else 1 << 62)
        work = 0
        for r in self.reps.values():
            s = min(r["left"], todo)
            r["left"] -= s
            r["steps"] += s
            work += s * r["n"]
        self.clock.t += todo * 10e-6 + work / self.rate
        return todo

    def run_queued_async(self, k):
        ran = self.run_queued(k)
        self.tickets += 1
        cap = max(self.reps) + 1 if self.reps else 0
        snap = np.zeros((cap, 9))
        snap[:, 2] = -1
        for rid, r in self.reps.items():
            snap[rid, [0, 1, 2, 3, 5, 6, 7]] = [1, r["steps"], r["left"], -5.0, 1.0, 0.0, 1]
        self.snaps[self.tickets] = (ran, snap)
        return self.tickets

    def poll(self, ticket):
        return True

    def wait(self, ticket):
        ran, snap = self.snaps.pop(ticket)
        cap = max(list(self.reps) + [len(snap) - 1]) + 1
        out = np.zeros((cap, 9))
        out[:, 2] = -1
        out[:len(snap)] = snap
        return ran, out

    def stats(self, rid):
        r = self.reps[rid]
        return {"pe": -5.0, "ke": 1.0, "xi": 0.0, "steps": r["steps"], "rebuilds": 1, "steps_left": r["left"]}

    def remove(self, rid):
        del self.reps[rid]
        self.free.append(rid)


def small_stream(n=40, rate=50.0):
    from rumd_b200 import serving
    return serving.poisson_stream(n, rate=rate, seed=3, n_range=(256, 1024), steps_range=(100, 2000))


def test_stream_is_seeded_and_has_requested_shape():
    from rumd_b200 import serving
    a = serving.poisson_stream(500, seed=1)
    b = serving.poisson_stream(500, seed=1)
    assert [(j.n, j.steps, j.kind) for j in a] == [(j.n, j.steps, j.kind) for j in b]
    ns = np.array([j.n for j in a])
    assert ns.min() >= 256 and ns.max() <= 32768
    rate = len(a) / a[-1].arrival
    assert 40 < rate < 60
    assert 0.4 < np.mean([j.kind == "KA" for j in a]) < 0.6


def test_all_jobs_complete_with_exact_step_counts():
    from rumd_b200 import serving
    clk = FakeClock()
    eng = FakeEngine(clk)
    srv = serving.MDServer(eng, hbm_budget=150e9, chunk_steps=100, clock=clk, sleep=clk.sleep, workers=0)
    jobs = srv.serve(small_stream())
    assert all(j.done >= j.admitted >= j.arrival for j in jobs)
    assert all(j.result["steps"] == j.steps for j in jobs)
    assert not eng.reps and srv.used == 0
    s = serving.latency_summary(jobs)
    assert s["p99_s"] >= s["p50_s"] > 0


def test_budget_limits_concurrency_and_keeps_fifo():
    from rumd_b200 import serving
    jobs = small_stream(30, rate=1e6)  # everything arrives at once
    budget = 3 * max(j.n for j in jobs) * FakeEngine.BYTES_PER_PARTICLE
    clk = FakeClock()
    eng = FakeEngine(clk)
    srv = serving.MDServer(eng, hbm_budget=budget, chunk_steps=50, clock=clk, sleep=clk.sleep, workers=0)
    srv.serve(jobs)
    assert srv.max_used <= budget
    assert 3 <= eng.max_live < len(jobs)
    order = sorted(jobs, key=lambda j: j.admitted)
    assert [j.id for j in order] == sorted(j.id for j in jobs)  # FIFO admission
    assert max(srv.queue_depth) > 0


def test_job_larger_than_budget_is_rejected():
    from rumd_b200 import serving
    jobs = small_stream(3)
    clk = FakeClock()
    srv = serving.MDServer(FakeEngine(clk), hbm_budget=1000, clock=clk, sleep=clk.sleep, workers=0)
    with pytest.raises(ValueError):
        srv.serve(jobs)


def test_continuous_batching_beats_one_at_a_time_on_latency():
    """With the fake's cost model (work of the busiest round), batching
    overlaps jobs, so the mix finishes sooner than the sequential loop."""
    from rumd_b200 import serving
    clk = FakeClock()
    srv = serving.MDServer(FakeEngine(clk, rate=2e8), chunk_steps=100, clock=clk, sleep=clk.sleep, workers=0)
    mix = serving.latency_summary(srv.serve(small_stream()))
    clk2 = FakeClock()
    seq = serving.latency_summary(serving.serve_one_at_a_time(lambda: _closing(FakeEngine(clk2, rate=2e8)),
                                                               small_stream(), clock=clk2, sleep=clk2.sleep))
    assert mix["p50_s"] <= seq["p50_s"]


def _closing(e):
    e.close = lambda: None
    return e


def test_shard_partitions_jobs():
    from rumd_b200 import serving
    jobs = serving.poisson_stream(100, seed=5)
    parts = [serving.shard(jobs, r, 4) for r in range(4)]
    ids = sorted(j.id for p in parts for j in p)
    assert ids == list(range(100))
    loads = [sum(j.n * j.steps for j in p) for p in parts]
    assert max(loads) / min(loads) < 1.2


def _gloo_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from rumd_b200 import serving
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    jobs = serving.poisson_stream(64, seed=9)
    mine = serving.shard(jobs, rank, world)
    t = torch.tensor([len(mine)], dtype=torch.int64)
    dist.all_reduce(t)
    gathered = [None] * world
    dist.all_gather_object(gathered, [j.id for j in mine])
    # max-over-ranks timing reduction as bench.py does it
    tm = torch.tensor([float(rank + 1)])
    dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    dist.destroy_process_group()
    q.put((rank, int(t.item()), gathered, float(tm.item())))


def test_two_rank_gloo_sharding():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    for rank, total, gathered, tmax in out:
        assert total == 64
        assert sorted(gathered[0] + gathered[1]) == list(range(64))
        assert not set(gathered[0]) & set(gathered[1])
        assert tmax == 2.0


def test_snapshot_of_a_chunk_launched_before_admission_is_ignored():
    """A replica id can be reused by a job admitted after a chunk was
    launched; that chunk's snapshot shows the previous owner (done) and must
    not retire the new job."""
    from rumd_b200 import serving
    clk = FakeClock()
    eng = FakeEngine(clk)
    srv = serving.MDServer(eng, clock=clk, sleep=clk.sleep, workers=0)
    job = serving.Job(id=0, kind="KA", n=256, T=1.0, steps=100, arrival=0.0)
    rid = eng.add(np.zeros((256, 4), np.float32), None, None, 2)
    srv.running[rid] = serving._Resident(job, 100, first_ticket=5)
    snap = np.zeros((1, 9))
    snap[0, serving.SNAP["active"]] = 1
    snap[0, serving.SNAP["steps"]] = 100
    srv._after_chunk(4, snap, 1.0, [])
    assert rid in srv.running and job.done < 0
    srv._after_chunk(5, snap, 2.0, [])
    assert rid not in srv.running and job.done == 2.0 and job.result["steps"] == 100


def test_configurations_built_on_worker_threads_keep_fifo():
    from rumd_b200 import serving
    jobs = small_stream(20, rate=1e6)
    clk = FakeClock()
    eng = FakeEngine(clk)
    budget = 4 * max(j.n for j in jobs) * FakeEngine.BYTES_PER_PARTICLE
    srv = serving.MDServer(eng, hbm_budget=budget, chunk_steps=80, clock=clk, sleep=clk.sleep, workers=2)
    srv.serve(jobs)
    assert all(j.result["steps"] == j.steps for j in jobs)
    order = sorted(jobs, key=lambda j: (j.admitted, j.id))
    assert [j.id for j in order] == sorted(j.id for j in jobs)
    assert srv.max_used <= budget and not eng.reps


def test_auto_chunk_length_follows_the_resident_particles():
    from rumd_b200 import serving
    clk = FakeClock()
    srv = serving.MDServer(FakeEngine(clk), clock=clk, sleep=clk.sleep, workers=0, chunk_seconds=0.05,
                           rate_hint=1e9, min_chunk_steps=16, max_chunk_steps=2000)
    for rid, n in enumerate([100000, 400000]):
        srv.running[rid] = serving._Resident(serving.Job(rid, "LJ", n, 1.0, 10, 0.0), 10)
    assert srv.chunk_length() == 100  # 0.05 s * 1e9 / 5e5 particles
    srv.running.pop(1)
    srv.running[0].left = 0
    assert srv.chunk_length() == 2000  # nothing left to run: the cap


def test_timeline_summary_reports_backlog_and_offered_load():
    from rumd_b200 import serving
    clk = FakeClock()
    srv = serving.MDServer(FakeEngine(clk, rate=1e8), chunk_steps=100, clock=clk, sleep=clk.sleep, workers=0)
    jobs = srv.serve(small_stream(30, rate=200.0))
    s = serving.timeline_summary(srv, jobs, step_s=0.05)
    assert s["rows"] and s["columns"][0] == "t_s"
    assert s["offered_particle_steps_per_s"] > 0 and s["chunks"] == srv.chunks > 0
    assert s["rows"][-1][3] == 0.0  # drained at the end
