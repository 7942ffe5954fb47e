#!/usr/bin/env python
"""Benchmark: RUMD's LJ/NVT time step on B200 (particle-steps/s).

Headline workload (one JSON line on rank 0): plain method, single large
system -- Kob-Andersen 80:20 LJ, N=65536, density 1.2, T=0.45, Nose-Hoover
NVT (tau=0.2), dt=0.005, skin 0.3, shifted-force cut-off 2.5 sigma_ij, FP32
forces with FP64 reductions.  A "step" is one MD time step (momentum reset,
neighbour-list check/rebuild, forces, integration).  The line also carries the
batched form (256 mixed-size KA replicas in one launch sequence) against
sequential plain runs of a sample of the same replicas, and the served form
(a Poisson stream of KA/LJ jobs through the continuous-batching server, with
p50/p99 job latency) against the one-job-at-a-time loop.

  python bench.py [--gpus N --steps K --warmup W]        # this implementation
  python bench.py --impl reference ...                   # reference CPU path

--gpus N > 1 runs under torchrun: every rank advances its own independent
replica of the workload (the path has no data exchange); value is the sum.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_PLAIN = 65536
KA_DENSITY = 1.2
T_PLAIN = 0.45
DT = 0.005
SKIN = 0.3
TAU = 0.2
METRIC = "particle-steps/s at 1 B200 (plain vs batched/served); p50/p99 job latency"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20000)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--pb", type=int, default=64)
    p.add_argument("--tp", type=int, default=2)
    p.add_argument("--batch-steps", type=int, default=10000)
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--served-jobs", type=int, default=400, help="jobs in the served stream (0: skip)")
    p.add_argument("--served-only", action="store_true",
                   help="only the served stream (one JSON line, not the headline)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--force-mode", type=int, default=None, help="kernel variant: 0 streamed, 1 staged, 2 window")
    p.add_argument("--build-lanes", type=int, default=None, help="kernel variant: list-build lanes per particle")
    p.add_argument("--sm-tiles", type=int, default=None, help="kernel variant: 1 = SM-region tile claiming")
    p.add_argument("--persistent", type=int, default=None,
                   help="kernel variant: 1 = one cooperative kernel runs the steps between list rebuilds")
    p.add_argument("--profile-launches", action="store_true",
                   help="small plain run only (for the ncu launch list)")
    p.add_argument("--profile-batched", action="store_true",
                   help="the 256-replica batch only, eager launches of --steps steps between "
                        "cudaProfilerStart/Stop (for the ncu launch list)")
    p.add_argument("--batched-only", action="store_true",
                   help="only the 256-replica batch (one JSON line, not the headline)")
    p.add_argument("--lj1m", action="store_true",
                   help="only the HBM-scale plain workload: single-component LJ, N=1,048,576 (one JSON line)")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Barrier and max-over-ranks for timings (NCCL when launched by torchrun)."""

    def __init__(self, world, local):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
            self.dist = dist
            self.torch = torch

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        t = self.torch.tensor([float(x)], device="cuda")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if self.world == 1:
            return x
        t = self.torch.tensor([float(x)], device="cuda")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ka_in_range_ratio(skin=SKIN, fractions=(0.8, 0.2), sig=((1.0, 0.8), (0.8, 0.88)), rcut=2.5):
    """Model ratio (pairs within rc) / (pairs within rc + skin) for KA: the
    density of each partner type times (4/3) pi r^3, averaged over the
    particle's type.  Scales the measured mean list length to the in-range
    neighbour count of the FLOP model."""
    n_in = n_list = 0.0
    for a in range(2):
        for b in range(2):
            rc = rcut * sig[a][b]
            n_in += fractions[a] * fractions[b] * rc ** 3
            n_list += fractions[a] * fractions[b] * (rc + skin) ** 3
    return n_in / n_list


def profiled_traffic():
    """DRAM bytes of the persistent step kernel per step, copied from the
    committed ncu capture (profiles/traffic.json)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return None


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

# kernel variants for every engine the bench makes (None: the engine's default)
KERNEL_VARIANTS = {}


def new_engine(capi, **kw):
    e = capi.Engine(**kw)
    for which, value in KERNEL_VARIANTS.items():
        if value is not None:
            e.set_variant(which, value)
    return e


def ka_params():
    from rumd_b200 import initconf as I
    return I.lj_params(2, I.KA)


def prepare_plain(capi, device, pb, tp, seed):
    """KA N=65536 melted at T=2 then brought to T=0.45 (untimed preparation)."""
    from rumd_b200 import initconf as I
    c = I.ka_config(N_PLAIN, density=KA_DENSITY, T=2.0, seed=seed)
    params = ka_params()
    e = new_engine(capi, device=device, pb=pb, tp=tp)
    rid = e.add(c["pos4"], c["box"], params, 2, cutoff="SF", skin=SKIN, dt=DT, T=2.0, tau=TAU, vel4=c["vel4"])
    e.run(1000)
    e.set_integrator(rid, DT, T_PLAIN, TAU)
    e.run(2000)
    return e, rid, c["box"], params


def flush_l2(device):
    import torch
    buf = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{device}")
    buf.fill_(1)
    torch.cuda.synchronize(device)
    del buf


def time_run(capi, e, steps, device):
    """Device time of Run(steps) with CUDA events on the engine's stream."""
    import torch
    stream = torch.cuda.ExternalStream(e.stream(), device=f"cuda:{device}")
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    t0.record(stream)
    e.run(steps)
    t1.record(stream)
    torch.cuda.synchronize(device)
    return t0.elapsed_time(t1) / 1e3


def launches_in_run(steps, rebuilds, per_rebuild=8, persistent=False):
    # run start: steps + momentum; run end: rebuild sequence + force kernel.
    # Per-step graphs: a fused kernel per step, a gate per graph launch and
    # the rebuild kernels (8, 9 with position windows) per rebuild.
    # Persistent graph: one loop gate, then per loop pass (a pass ends at each
    # rebuild) the rebuild kernels, which exit at once when none is due, and
    # one k_steps launch.
    if persistent:
        core = 1 + (rebuilds + 1) * (per_rebuild + 1)
    else:
        core = steps + steps // 32 + steps % 32 + per_rebuild * rebuilds
    return int(core + 2 + per_rebuild + 1)


def _timed_oracle_steps(O, pos4, vel4, im3, kw, seconds):
    t = time.perf_counter()
    O.md_run(pos4, vel4, im3, nsteps=2, **kw)
    one = max((time.perf_counter() - t) / 2, 1e-4)
    steps = int(max(2, min(2000, seconds / one)))
    t = time.perf_counter()
    O.md_run(pos4, vel4, im3, nsteps=steps, **kw)
    return steps, time.perf_counter() - t


def cpu_baseline_sample(e, rid, box, params, seconds=15.0, seconds_1core=5.0):
    """The oracle's FP32 step (cell list + full list + forces + NVT) on all
    host cores, and on one core, from the GPU arm's own equilibrated state."""
    from oracle import oracle as O
    n = N_PLAIN
    pos4, vel4, im3 = e.read(rid, n)
    kw = dict(L=box, ntypes=2, params=params, cutoff=O.SF, skin=SKIN, dt=DT, T=T_PLAIN, tau=TAU)
    cores = O.num_threads()
    steps, dt = _timed_oracle_steps(O, pos4, vel4, im3, kw, seconds)
    O.set_num_threads(1)
    try:
        steps1, dt1 = _timed_oracle_steps(O, pos4, vel4, im3, kw, seconds_1core)
    finally:
        O.set_num_threads(cores)
    return {"value": n * steps / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "cpu_model": cpu_model(), "value_1core": n * steps1 / dt1,
            "sample": f"KA N={n} from the equilibrated T=0.45 state, {steps} FP32 steps (cell sort, full list, "
                      f"SF forces, NVT) with OpenMP over particles on {cores} threads; {steps1} steps on 1 thread "
                      f"for value_1core"}


def pinned(a):
    """A page-locked host copy of numpy array a (the caller's pinned buffers)."""
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out, t


def e2e_run(capi, device, pb, tp, pos4, vel4, im3, box, params, steps):
    """Public API end to end: upload (H2D from the caller's pinned arrays) +
    Run(steps) + read back (D2H) of positions, velocities, images and the
    energies.  The engine is created, with pools sized for the system (the way
    a serving process keeps one), before the timed region."""
    n = len(pos4)
    (p_in, t1), (v_in, t2) = pinned(np.ascontiguousarray(pos4)), pinned(np.ascontiguousarray(vel4))
    e = new_engine(capi, device=device, pb=pb, tp=tp, max_particles=n, max_list_entries=n * 256)
    e.run(0)
    t = time.perf_counter()
    rid = e.add(p_in, box, params, 2, cutoff="SF", skin=SKIN, dt=DT, T=T_PLAIN, tau=TAU, vel4=v_in, im3=im3)
    t_add = time.perf_counter()
    e.run(steps)
    t_run = time.perf_counter()
    p, v, im = e.read(rid, n)
    st = e.stats(rid)
    t_end = time.perf_counter()
    dt = t_end - t
    e.close()
    del t1, t2
    assert np.isfinite(p).all() and np.isfinite(st["pe"])
    h2d = n * (16 + 16 + 16)                   # r, v, images (last_r and ids are made on the device)
    d2h = n * (4 + 16 + 16 + 16 + 4) + 256     # ids, pos, vel, images, list lengths (stats), state
    return {"value": n * steps / dt, "unit": "particle-steps/s",
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
            "phases_ms": {"add": 1e3 * (t_add - t), "run": 1e3 * (t_run - t_add), "read_back": 1e3 * (t_end - t_run)}}


def batch_workload(seed=0):
    """The batching configuration: 256 KA replicas, N = floor(exp(U(ln 512,
    ln 8192))) (seeded), T log-spaced from 0.45 to 2.0."""
    from rumd_b200 import initconf as I
    return I.ka_batch_workload(seed)


def batch_tuning():
    """The autotuner's pick for the 256-replica batch from the library's
    autotune cache (rumd_b200/autotune_cache.json, profiles/autotune_batch256.md),
    or the plain defaults when the cache has no entry for it."""
    from rumd_b200 import autotune
    path = os.path.join(ROOT, "rumd_b200", "autotune_cache.json")
    key = autotune.signature(autotune.batch_replicas())
    cache = {}
    if os.path.exists(path):
        with open(path) as fh:
            cache = json.load(fh)
    if key in cache:
        e = cache[key]
        return {"pb": e["pb"], "tp": e["tp"], "skin": e["skin"], "persistent": e.get("persistent", 1),
                "source": "autotuner (rumd_b200/autotune_cache.json)"}
    return {"pb": 64, "tp": 2, "skin": SKIN, "persistent": 1, "source": "defaults (no autotune entry)"}


def batch_engine(capi, device, pb, tp, ns, Ts, confs, skin=SKIN):
    R = len(ns)
    params = ka_params()
    e = new_engine(capi, device=device, max_particles=int(ns.sum() + 64 * R), max_replicas=R, pb=pb, tp=tp)
    for c, T in zip(confs, Ts):
        e.add(c["pos4"], c["box"], params, 2, cutoff="SF", skin=skin, dt=DT, T=float(T), tau=TAU, vel4=c["vel4"])
    return e


def profile_batched(capi, device, args):
    """The batch with eager launches (b2md_run_timed) for ncu's launch list."""
    import torch
    ns, Ts, confs = batch_workload()
    tune = batch_tuning()
    e = batch_engine(capi, device, tune["pb"], tune["tp"], ns, Ts, confs, skin=tune["skin"])
    e.set_variant(capi.VARIANT_PERSISTENT, tune["persistent"])
    e.run_timed(300)  # warm-up with eager launches too (no graphs under the profiler)
    torch.cuda.synchronize(device)
    torch.cuda.profiler.start()
    ms, nl = e.run_timed(max(args.steps, 1))
    torch.cuda.synchronize(device)
    torch.cuda.profiler.stop()
    print(json.dumps({"profile_batched_steps": args.steps, "particles": int(ns.sum()),
                      "step_kernel_ms_avg": ms / max(args.steps, 1), "launches": nl}), flush=True)
    e.close()


def batched(capi, device, pb, tp, steps, seed=0):
    """256 KA replicas, N log-uniform in [512, 8192], T log-spaced 0.45..2.0,
    advanced together with the autotuner's launch shape and skin; against
    sequential plain runs of every 16th replica (the plain defaults)."""
    R = 256
    ns, Ts, confs = batch_workload(seed)
    params = ka_params()
    tune = batch_tuning()
    e = batch_engine(capi, device, tune["pb"], tune["tp"], ns, Ts, confs, skin=tune["skin"])
    e.set_variant(capi.VARIANT_PERSISTENT, tune["persistent"])
    e.run(500)
    t_b = time_run(capi, e, steps, device)
    rate_b = float(ns.sum()) * steps / t_b
    kind = e.get_variant(capi.VARIANT_PERSISTENT_ACTIVE)
    e.close()
    sample = list(range(0, R, 16))
    t_seq, ps_seq = 0.0, 0.0
    for k in sample:
        c = confs[k]
        s = new_engine(capi, device=device, pb=pb, tp=tp)
        s.add(c["pos4"], c["box"], params, 2, cutoff="SF", skin=SKIN, dt=DT, T=float(Ts[k]), tau=TAU, vel4=c["vel4"])
        s.run(500)
        t_seq += time_run(capi, s, steps, device)
        ps_seq += float(ns[k]) * steps
        s.close()
    rate_s = ps_seq / t_seq
    return {"value": rate_b, "unit": "particle-steps/s", "replicas": R, "particles": int(ns.sum()),
            "steps": steps, "ms_per_step": t_b / steps * 1e3, "tuning": tune,
            "persistent_kernel": {0: "none (one launch per step)", 1: "k_steps", 2: "k_batch",
                                  3: "k_flow"}.get(kind, kind),
            "sequential_plain_value": rate_s,
            "sequential_sample": f"{len(sample)} of the {R} replicas run alone, one after another",
            "speedup_vs_sequential": rate_b / rate_s}


def served(capi, device, pb, tp, njobs, seed=0):
    """Continuous batching: a seeded Poisson stream (50 jobs/s) of KA/LJ jobs,
    N log-uniform in [256, 32768], steps log-uniform in [1e3, 1e5], admitted
    against a 150 GB budget of engine-reported memory and advanced together
    in asynchronous chunks (rumd_b200.serving) with the batch's autotuned
    launch shape, skin and batched kernel.  Latencies are wall-clock from
    arrival to the host seeing the job's last step; throughput is all jobs'
    particle-steps over the makespan (first arrival to last completion).
    Against the plain one-job-at-a-time loop on a sample of the same jobs."""
    from rumd_b200 import serving
    jobs = serving.poisson_stream(njobs, rate=50.0, seed=seed)
    tune = batch_tuning()
    total_n = sum(j.n for j in jobs)
    # pre-sized for every job resident at once: no pool grows (and no graph
    # is rebuilt) while the stream runs; about 180 list entries per particle
    e = new_engine(capi, device=device, max_particles=total_n + 64 * njobs, max_replicas=min(njobs, 1024),
                   max_list_entries=180 * (total_n + 32 * njobs), pb=tune["pb"], tp=tune["tp"])
    e.set_variant(capi.VARIANT_PERSISTENT, 3)  # k_flow: replicas step on their own
    srv = serving.MDServer(e, hbm_budget=150e9, chunk_steps="auto", dt=DT, skin=tune["skin"], tau=TAU,
                           workers=2, max_resident=1024)
    srv.serve(jobs)
    reserved = e.memory()
    counters = e.counters()
    e.close()
    summ = serving.latency_summary(jobs)
    tl = serving.timeline_summary(srv, jobs)
    sample = [serving.Job(**{k: getattr(j, k) for k in ("id", "kind", "n", "T", "steps", "seed")}, arrival=0.0)
              for j in jobs[::max(1, njobs // 8)]]
    t0 = time.perf_counter()
    serving.serve_one_at_a_time(lambda: new_engine(capi, device=device, pb=pb, tp=tp), sample, dt=DT, skin=SKIN,
                                tau=TAU)
    t_one = time.perf_counter() - t0
    one_rate = sum(j.n * j.steps for j in sample) / t_one
    offered = tl.get("offered_particle_steps_per_s") or 0.0
    thr = summ["throughput"]
    if offered > thr:
        statement = (f"not sustainable: 50 jobs/s offers {offered:.3g} particle-steps/s, {offered / thr:.1f}x the "
                   f"measured capacity of {thr:.3g}; the backlog grows while jobs arrive and drains only after "
                   f"the arrivals stop (rows of load_over_time). The sustainable rate for this job mix is about "
                   f"{50.0 * thr / offered:.1f} jobs/s.")
    else:
        statement = (f"sustainable: 50 jobs/s offers {offered:.3g} particle-steps/s, below the measured capacity "
                   f"of {thr:.3g}")
    return {"value": thr, "unit": "particle-steps/s", "jobs": summ["jobs"],
            "p50_latency_s": summ["p50_s"], "p99_latency_s": summ["p99_s"], "makespan_s": summ["makespan_s"],
            "particle_steps": summ["particle_steps"], "hbm_max_used_bytes": srv.max_used,
            "hbm_reserved_bytes": reserved, "engine_counters": counters, "tuning": tune,
            "sustainability": statement, "load_over_time": tl,
            "one_at_a_time_value": one_rate,
            "one_at_a_time_sample": f"{len(sample)} of the {njobs} jobs run alone back to back (wall clock)",
            "speedup_vs_one_at_a_time": thr / one_rate,
            "stream": "Poisson 50 jobs/s, KA (rho 1.2) or LJ (rho 0.8442) 50/50, N 256-32768 and steps 1e3-1e5 "
                      f"log-uniform, T 0.5-2.0, seed {seed}; throughput = particle-steps / (last completion - first "
                      "arrival)"}


def lj_hbm_scale(capi, device, args):
    """The HBM-scale plain configuration: single-component LJ (SF rc = 2.5),
    N = 1,048,576 (4 x 64^3 FCC), density 0.8442, T = 0.722, NVT tau = 0.2,
    dt = 0.004, skin 0.3.  The list (about 320 MB) no longer fits in L2, so the
    force kernel's bytes come from HBM.  Prints one JSON line (not the
    headline)."""
    from rumd_b200 import initconf as I
    n = 1048576
    c = I.lj_config(n, density=0.8442, T=2.0, seed=3)
    params = I.lj_params(1, I.LJ)
    e = new_engine(capi, device=device, pb=args.pb, tp=args.tp)
    rid = e.add(c["pos4"], c["box"], params, 1, cutoff="SF", skin=SKIN, dt=0.004, T=2.0, tau=TAU, vel4=c["vel4"])
    e.run(500)
    e.set_integrator(rid, 0.004, 0.722, TAU)
    e.run(1000)
    steps = max(args.steps, 1)
    if args.profile_launches:
        # eager launches of `steps` steps between cudaProfilerStart/Stop (for ncu)
        import torch
        torch.cuda.synchronize(device)
        torch.cuda.profiler.start()
        ms, nl = e.run_timed(steps)
        torch.cuda.synchronize(device)
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_steps": steps, "step_kernel_ms_avg": ms / steps, "launches": nl}), flush=True)
        e.close()
        return
    r0 = e.stats(rid)["rebuilds"]
    flush_l2(device)
    t = time_run(capi, e, steps, device)
    rebuilds = e.stats(rid)["rebuilds"] - r0
    kms, _ = e.run_timed(200)
    st = e.stats(rid)
    per_launch_s = kms / 200 / 1e3
    bytes_alg = n * (168.0 + 4.0 * st["mean_nbrs"])
    peak, peak_kind = measured_peaks()
    achieved = bytes_alg / per_launch_s / 1e9
    accuracy = fp64_comparison(capi, device, e, rid, n, c["box"], params)
    print(json.dumps({"workload": "single-component LJ, N=1048576, rho=0.8442, T=0.722, NVT tau=0.2, dt=0.004, "
                                  "skin 0.3, SF rc=2.5 (plain method, HBM scale)",
                      "value": n * steps / t, "unit": "particle-steps/s", "steps": steps,
                      "ms_per_step": t / steps * 1e3, "rebuilds": rebuilds, "pb": args.pb, "tp": args.tp,
                      "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                   "frac": achieved / peak, "peak_source": peak_kind,
                                   "kernel_ms": per_launch_s * 1e3, "bytes_per_launch_alg": bytes_alg,
                                   "mean_list_length": st["mean_nbrs"]},
                      "fp64_oracle": accuracy}), flush=True)
    e.close()


def fp64_comparison(capi, device, e, rid, n, box, params, steps=5000):
    """The same state in the pure-FP64 GPU engine (b2md_f64_*): energy per
    particle and the configurational pressure W/V at that configuration, then
    `steps` NVT steps of each from it (FP32 engine and FP64 engine) with the
    run-averaged energy per particle over the second half (the trajectories
    decorrelate; the averages should not) and the FP64 run's own speed."""
    import torch
    pos4, vel4, im3 = e.read(rid, n)
    e.calc_f()
    s32 = e.stats(rid)
    V = float(np.prod(np.asarray(box, np.float64)))
    e64 = capi.F64Engine(pos4, box, params, 1, cutoff="SF", skin=SKIN, dt=0.004, T=0.722, tau=TAU, vel4=vel4,
                         im3=im3, device=device)
    e64.set_xi(s32["xi"])
    e64.calc_f()
    s64 = e64.stats()
    out = {"pe_per_particle_f32": s32["pe"] / n, "pe_per_particle_f64": s64["pe"] / n,
           "d_pe_per_particle": (s32["pe"] - s64["pe"]) / n,
           "W_over_V_f32": s32["virial"] / V, "W_over_V_f64": s64["virial"] / V,
           "d_pressure_configurational": (s32["virial"] - s64["virial"]) / V}
    e.set_energy_log(rid, 1, steps)
    e.run(steps)
    log = e.energy_log(rid)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    en = e64.run(steps, energies=True)
    torch.cuda.synchronize(device)
    t64 = time.perf_counter() - t0
    e64.close()
    half = steps // 2
    out.update({"nvt_steps": steps,
                "mean_pe_per_particle_f32": float(log[half:, 1].mean() / n),
                "mean_pe_per_particle_f64": float(en[half:, 0].mean() / n),
                "mean_W_over_V_f32": float(log[half:, 2].mean() / V),
                "mean_W_over_V_f64": float(en[half:, 1].mean() / V),
                "f64_value": n * steps / t64, "f64_unit": "particle-steps/s (wall clock)"})
    out["d_mean_pe_per_particle"] = out["mean_pe_per_particle_f32"] - out["mean_pe_per_particle_f64"]
    return out


def kernel_variants(engine):
    """The GPU arm's kernel variants (reported beside the config, not in it:
    the reference arm runs the same workload without them)."""
    from rumd_b200 import capi
    return {"pb_tp": list(engine.launch()), "force_mode": engine.get_variant(capi.VARIANT_FORCE_MODE),
            "build_lanes": engine.get_variant(capi.VARIANT_BUILD_LANES),
            "persistent": engine.get_variant(capi.VARIANT_PERSISTENT)}


def config_block(args, world):
    return {"workload": f"Kob-Andersen 80:20 LJ, N={N_PLAIN}, rho=1.2, T=0.45, NVT tau=0.2, dt=0.005, skin 0.3, "
                        "SF cut-off 2.5 sigma_ij (plain method, single large system)",
            "n_particles": N_PLAIN,
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "precision": "FP32 forces, FP64 reductions/thermostat, int32 images",
            "l2_policy": "L2 flushed (512 MiB write) before the timed Run; inside a Run every step reads the "
                         "state the previous step wrote, which stays L2-resident (30 MB) as in the reference"}


def run_reference(args):
    """The reference arm: the CPU implementation of the path (oracle port) on
    all host cores, same workload and metric.  The state is prepared with the
    GPU arm's recipe (seeded FCC start, 1000 steps at T=2, then 2000 at
    T=0.45, here on the CPU and untimed), then W warm-up steps and K timed
    steps (K capped so that the timed part stays near 60 s)."""
    rank, world, local = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    from rumd_b200 import initconf as I
    c = I.ka_config(N_PLAIN, density=KA_DENSITY, T=2.0, seed=1)
    params = ka_params()
    kw = dict(L=c["box"], ntypes=2, params=params, cutoff=O.SF, skin=SKIN, dt=DT, tau=TAU)
    st = O.md_run(c["pos4"], c["vel4"], c["im3"], nsteps=1000, T=2.0, **kw)
    st = O.md_run(st["pos4"], st["vel4"], st["im3"], nsteps=2000, xi=st["xi"], T=T_PLAIN, **kw)
    kw["T"] = T_PLAIN
    st = O.md_run(st["pos4"], st["vel4"], st["im3"], nsteps=max(args.warmup, 1), xi=st["xi"], **kw)
    t = time.perf_counter()
    st2 = O.md_run(st["pos4"], st["vel4"], st["im3"], nsteps=2, xi=st["xi"], **kw)
    one = (time.perf_counter() - t) / 2
    steps = int(max(2, min(args.steps, 60.0 / max(one, 1e-6))))
    t = time.perf_counter()
    O.md_run(st2["pos4"], st2["vel4"], st2["im3"], nsteps=steps, xi=st2["xi"], **kw)
    dt = time.perf_counter() - t
    v = N_PLAIN * steps / dt
    sample = (f"KA N={N_PLAIN} equilibrated with the GPU arm's recipe (seeded FCC, 1000 steps at T=2, 2000 at "
              f"T=0.45; untimed, on the CPU), then {steps} of the requested {args.steps} steps (capped at ~60 s), "
              "FP32 reference arithmetic, OpenMP over particles")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": dt / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_block(args, world),
            "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": O.num_threads(), "kind": "port",
                             "cpu_model": cpu_model(), "sample": sample},
            "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    dist = Dist(world, local)
    from rumd_b200 import capi
    capi.lib()
    KERNEL_VARIANTS[capi.VARIANT_FORCE_MODE] = args.force_mode
    KERNEL_VARIANTS[capi.VARIANT_BUILD_LANES] = args.build_lanes
    KERNEL_VARIANTS[capi.VARIANT_SM_TILES] = args.sm_tiles
    KERNEL_VARIANTS[capi.VARIANT_PERSISTENT] = args.persistent
    device = local
    if args.lj1m:
        lj_hbm_scale(capi, device, args)
        dist.close()
        return
    if args.profile_batched:
        profile_batched(capi, device, args)
        dist.close()
        return
    if args.batched_only:
        print(json.dumps({"batched": batched(capi, device, args.pb, args.tp, args.batch_steps)}), flush=True)
        dist.close()
        return
    if args.served_only:
        print(json.dumps({"served": served(capi, device, args.pb, args.tp, args.served_jobs)}), flush=True)
        dist.close()
        return
    if args.profile_launches:
        # Same workload driven with eager launches only (b2md_run_timed): the
        # kernels and their order are those of the graphs, but ncu sees plain
        # launches (it stalls on graphs with conditional nodes).
        from rumd_b200 import initconf as I
        c = I.ka_config(N_PLAIN, density=KA_DENSITY, T=2.0, seed=1)
        e = new_engine(capi, device=device, pb=args.pb, tp=args.tp)
        rid = e.add(c["pos4"], c["box"], ka_params(), 2, cutoff="SF", skin=SKIN, dt=DT, T=2.0, tau=TAU,
                    vel4=c["vel4"])
        e.run_timed(600)
        e.set_integrator(rid, DT, T_PLAIN, TAU)
        e.run_timed(400)
        # the profiled segment: ncu --profile-from-start off sees only these launches
        import torch
        torch.cuda.synchronize(device)
        torch.cuda.profiler.start()
        r0 = e.stats(rid)["rebuilds"]
        ms, nl = e.run_timed(max(args.steps, 1))
        torch.cuda.synchronize(device)
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_steps": args.steps, "step_kernel_ms_avg": ms / max(args.steps, 1),
                          "rebuilds": e.stats(rid)["rebuilds"] - r0, "launches": nl}), flush=True)
        e.close()
        dist.close()
        return
    e, rid, box, params = prepare_plain(capi, device, args.pb, args.tp, seed=1 + rank)
    e.run(max(args.warmup, 3))          # untimed warm-up steps (graphs instantiated)
    flush_l2(device)
    rb0 = e.stats(rid)["rebuilds"]
    clocks = ClockSampler(device)
    clocks.start()
    dist.barrier()
    t = time_run(capi, e, args.steps, device)
    dist.barrier()
    clk = clocks.stop()
    t_max = dist.max(t)
    st = e.stats(rid)
    rebuilds = st["rebuilds"] - rb0
    persistent_active = e.get_variant(capi.VARIANT_PERSISTENT_ACTIVE) == 1
    total_ps = dist.sum(N_PLAIN * args.steps)
    value = total_ps / t_max
    # live roofline of the dominant kernel: the persistent step kernel the
    # timed run uses (force + Nose-Hoover + reductions + grid barrier), timed
    # per launch with CUDA events in the eager form of the same loop
    # (b2md_run_timed), per step
    kms, _ = e.run_timed(2000)
    st2 = e.stats(rid)
    per_step_s = kms / 2000 / 1e3
    nlist = st2["mean_nbrs"]
    bytes_alg = N_PLAIN * (168.0 + 4.0 * nlist)            # HBM model: state + list stream
    l2_bytes_alg = N_PLAIN * (168.0 + 20.0 * nlist)        # + the 16-byte neighbour gathers
    flops_alg = N_PLAIN * (18.0 * nlist + 27.0 * nlist * ka_in_range_ratio())
    peak, peak_kind = measured_peaks()
    achieved = bytes_alg / per_step_s / 1e9
    l2_peak, fma_peak = capi.measure_peaks(5)
    tr = profiled_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tr or {}).get("bytes_per_step"),
                "traffic_source": "copied from the committed ncu capture (profiles/traffic.json), per step",
                "peak_source": peak_kind, "kernel": "k_steps<TP> (persistent fused step)",
                "kernel_ms_per_step": per_step_s * 1e3, "bytes_per_step_alg": bytes_alg,
                "mean_list_length": nlist, "step_share_of_run": per_step_s * args.steps / t,
                "limiter": "L1 neighbour gathers and their latency: the 30 MB working set is L2-resident at "
                           "this size, so the HBM fraction is a model figure",
                "l2": {"achieved": l2_bytes_alg / per_step_s / 1e9, "peak": l2_peak, "unit": "GB/s",
                       "frac": l2_bytes_alg / per_step_s / 1e9 / l2_peak, "bytes_per_step_alg": l2_bytes_alg,
                       "peak_source": "measured in this run (b2md_measure_peaks, 48 MiB read past L1)"},
                "fp32": {"achieved": flops_alg / per_step_s / 1e12, "peak": fma_peak, "unit": "TFLOP/s",
                         "frac": flops_alg / per_step_s / 1e12 / fma_peak, "flops_per_step_alg": flops_alg,
                         "peak_source": "measured in this run (b2md_measure_peaks, FP32 FMA chains)"}}
    extra = {}
    cfg = config_block(args, world)
    variants = kernel_variants(e)
    per_rebuild = 9 if variants.get("force_mode") == capi.FORCE_WINDOW else 8
    if rank == 0:
        pos4, vel4, im3 = e.read(rid, N_PLAIN)
        e2e = e2e_run(capi, device, args.pb, args.tp, pos4, vel4, im3, box, params, args.steps)
        if not args.no_cpu_baseline:
            extra["cpu_baseline"] = cpu_baseline_sample(e, rid, box, params)
        if not args.no_batched:
            extra["batched"] = batched(capi, device, args.pb, args.tp, args.batch_steps)
        if args.served_jobs > 0:
            extra["served"] = served(capi, device, args.pb, args.tp, args.served_jobs)
            if "batched" in extra:
                extra["served"]["vs_batched"] = extra["served"]["value"] / extra["batched"]["value"]
    e.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded FCC start, melted and equilibrated untimed)",
                "config": cfg, "variants": variants, "clocks": clk, "e2e": e2e,
                "gpu_launches": launches_in_run(args.steps, rebuilds, per_rebuild, persistent_active), "rebuilds": rebuilds,
                "roofline": roofline}
        line.update(extra)
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
