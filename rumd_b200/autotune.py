"""Autotuner for the launch shape and the rebuild cadence.

Modelled on RUMD's Autotune (Python/rumd/Autotune.py:156-161, 584-1000),
which times short runs over particles-per-block, threads-per-particle, skin
and neighbour-list method, and caches the winner in autotune.dat.  Here the
knobs are the engine's:
  pb   particles per block (tile size): 32, 64, 128
  tp   threads per particle: 1, 2, 4, 8   (pb*tp <= 512)
  skin neighbour-list skin, i.e. the rebuild cadence: 0.2 .. 0.5
and, in a second stage at the winning shape, the kernel variants
  force_mode    neighbours streamed (0), list tile staged (1) or position
                window staged (2) in shared memory
  build_lanes   lanes per particle in the list build: 0 (row scan, one thread
                per particle), 1, 2, 4, 8, or 32 (one warp per cell)
  sm_tiles      streamed mode: blocks claim tiles from their SM's region (1)
                or one block per tile (0)
  persistent    streamed mode, one block per tile: the steps between list
                rebuilds in one cooperative kernel (1) or one launch per step (0)
Each candidate is timed on the device (CUDA events around a short run of the
real workload, after a warm-up run).  As in RUMD's test mode
(Autotune.py:929-937), every candidate's potential energy after its run must
agree with the first candidate's within 0.005 per particle; a candidate that
fails this is rejected.  Results are cached in a JSON file keyed by the
workload signature.
"""
import itertools
import json
import os

DEFAULT_PB = (32, 64, 128)
DEFAULT_TP = (1, 2, 4, 8)
DEFAULT_SKIN = (0.2, 0.3, 0.4, 0.5)
VARIANT_KEYS = ("force_mode", "build_lanes", "sm_tiles", "persistent")
# kernel-variant candidates: (force_mode, sm_tiles, persistent) x build_lanes
VARIANTS = tuple(dict(force_mode=fm, sm_tiles=st, persistent=ps, build_lanes=bl)
                 for (fm, st, ps), bl in itertools.product(((0, 0, 1), (0, 0, 0), (0, 1, 0), (1, 0, 0), (2, 0, 0)),
                                                           (0, 1, 2, 4, 8, 32)))


def candidates(pbs=DEFAULT_PB, tps=DEFAULT_TP, skins=DEFAULT_SKIN, max_block=512):
    return [(pb, tp, sk) for pb, tp, sk in itertools.product(pbs, tps, skins) if pb * tp <= max_block]


def search(cands, measure, pe_tol=0.005):
    """measure(pb, tp, skin) -> (rate, pe_per_particle).  Returns the best
    candidate and the table of all measurements."""
    table = []
    ref_pe = None
    best = None
    for pb, tp, skin in cands:
        rate, pe = measure(pb, tp, skin)
        ok = True
        if ref_pe is None:
            ref_pe = pe
        elif abs(pe - ref_pe) > pe_tol:
            ok = False
        table.append({"pb": pb, "tp": tp, "skin": skin, "rate": rate, "pe": pe, "ok": ok})
        if ok and (best is None or rate > best["rate"]):
            best = table[-1]
    return best, table


def search_variants(shape, measure, variants=VARIANTS, pe_tol=0.005):
    """Second stage: the kernel variants at a fixed (pb, tp, skin).
    measure(pb, tp, skin, **variant) -> (rate, pe)."""
    table = []
    ref_pe = None
    best = None
    for var in variants:
        rate, pe = measure(shape["pb"], shape["tp"], shape["skin"], **var)
        ok = True
        if ref_pe is None:
            ref_pe = pe
        elif abs(pe - ref_pe) > pe_tol:
            ok = False
        table.append(dict(var, rate=rate, pe=pe, ok=ok))
        if ok and (best is None or rate > best["rate"]):
            best = table[-1]
    return best, table


def apply(engine, entry):
    """Sets a tuned entry's launch shape and kernel variants on an engine."""
    from . import capi
    engine.set_launch(entry["pb"], entry["tp"])
    codes = {"force_mode": capi.VARIANT_FORCE_MODE, "build_lanes": capi.VARIANT_BUILD_LANES,
             "sm_tiles": capi.VARIANT_SM_TILES, "persistent": capi.VARIANT_PERSISTENT}
    for k, code in codes.items():
        if k in entry:
            engine.set_variant(code, entry[k])


def signature(replicas):
    """Workload key: particle counts (binned), densities and types."""
    parts = sorted((int(round(r["n"], -2)), round(r["density"], 3), r["ntypes"]) for r in replicas)
    return json.dumps(parts)


class Autotune:
    def __init__(self, cache_path="autotune.json", **grid):
        self.cache_path = cache_path
        self.grid = grid

    def _load(self):
        if os.path.exists(self.cache_path):
            with open(self.cache_path) as fh:
                return json.load(fh)
        return {}

    def tune(self, replicas, measure, force=False, variants=False):
        """Stage 1 over (pb, tp, skin); with variants=True, stage 2 over the
        kernel variants at the winning shape (measure then takes the
        VARIANT_KEYS as keywords)."""
        key = signature(replicas)
        cache = self._load()
        if key in cache and not force:
            return cache[key]
        best, table = search(candidates(**self.grid), measure)
        entry = {"pb": best["pb"], "tp": best["tp"], "skin": best["skin"], "rate": best["rate"], "table": table}
        if variants:
            vbest, vtable = search_variants(entry, measure, variants=VARIANTS)
            entry.update({k: vbest[k] for k in VARIANT_KEYS if k in vbest})
            entry.update(rate=max(entry["rate"], vbest["rate"]), variant_table=vtable)
        cache[key] = entry
        with open(self.cache_path, "w") as fh:
            json.dump(cache, fh, indent=1)
        return cache[key]


def equilibrated_ka(capi, n, T, device=0, seed=1, melt_steps=1000, eq_steps=1000):
    """A KA liquid at temperature T: FCC start melted at T=2, then brought to T."""
    from . import initconf
    c = initconf.ka_config(n, T=2.0, seed=seed)
    params = initconf.lj_params(2, initconf.KA)
    e = capi.Engine(device=device)
    rid = e.add(c["pos4"], c["box"], params, 2, cutoff="SF", T=2.0, vel4=c["vel4"])
    e.run(melt_steps)
    e.set_integrator(rid, 0.005, T, 0.2)
    e.run(eq_steps)
    rep = dict(pos4=e.get(rid, "pos", n), vel4=e.get(rid, "vel", n), box=c["box"], params=params, ntypes=2, T=T,
               n=n, density=1.2)
    e.close()
    return rep


def device_measure(capi, replicas, device=0, steps=300, warmup=100):
    """measure() for `search`: builds an engine with all replicas at the given
    shape and skin and times `steps` device steps with CUDA events.

    replicas: list of dicts with pos4, vel4, box, params, ntypes, T, n, density."""
    import torch

    def measure(pb, tp, skin, force_mode=None, build_lanes=None, sm_tiles=None, persistent=None):
        e = capi.Engine(device=device, max_replicas=len(replicas), pb=pb, tp=tp)
        if persistent is not None:
            e.set_variant(capi.VARIANT_PERSISTENT, persistent)
        if force_mode is not None:
            e.set_variant(capi.VARIANT_FORCE_MODE, force_mode)
        if build_lanes is not None:
            e.set_variant(capi.VARIANT_BUILD_LANES, build_lanes)
        if sm_tiles is not None:
            e.set_variant(capi.VARIANT_SM_TILES, sm_tiles)
        ids = [e.add(r["pos4"], r["box"], r["params"], r["ntypes"], cutoff="SF", skin=skin, T=r["T"],
                     vel4=r["vel4"]) for r in replicas]
        e.calc_f()  # invariance check on the common starting configuration
        n = sum(r["n"] for r in replicas)
        pe = sum(e.stats(i)["pe"] for i in ids) / n
        e.run(warmup)
        stream = torch.cuda.ExternalStream(e.stream(), device=f"cuda:{device}")
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        t0.record(stream)
        e.run(steps)
        t1.record(stream)
        torch.cuda.synchronize(device)
        dt = t0.elapsed_time(t1) / 1e3
        e.close()
        return n * steps / dt, pe

    return measure


def batch_replicas(seed=0):
    """The 256-replica Kob-Andersen batch (initconf.ka_batch_workload) as
    autotuner replicas: FCC starts, each at its own temperature."""
    from . import initconf
    ns, Ts, confs = initconf.ka_batch_workload(seed)
    params = initconf.lj_params(2, initconf.KA)
    return [dict(pos4=c["pos4"], vel4=c["vel4"], box=c["box"], params=params, ntypes=2, T=float(T), n=int(n),
                 density=1.2) for n, T, c in zip(ns, Ts, confs)]


# kernel variants worth trying on a large batch (persistent kernel, list build)
BATCH_VARIANTS = tuple(dict(force_mode=0, sm_tiles=0, persistent=ps, build_lanes=bl) for ps in (1, 0) for bl in (0, 32))


def main(argv=None):
    """python -m rumd_b200.autotune --n 65536 --T 0.45 [--pbs 32,64 --tps 2,4 --skins 0.3]
    python -m rumd_b200.autotune --batch256 --skins 0.3,0.4,0.5   (the 256-replica batch)"""
    import argparse
    from . import capi
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=65536)
    p.add_argument("--T", type=float, default=0.45)
    p.add_argument("--batch256", action="store_true", help="tune on the 256-replica Kob-Andersen batch")
    p.add_argument("--pbs", default="32,64,128")
    p.add_argument("--tps", default="1,2,4,8")
    p.add_argument("--skins", default="0.3")
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--cache", default="autotune.json")
    p.add_argument("--no-variants", action="store_true", help="skip the kernel-variant stage")
    args = p.parse_args(argv)
    reps = batch_replicas() if args.batch256 else [equilibrated_ka(capi, args.n, args.T)]
    at = Autotune(cache_path=args.cache, pbs=tuple(int(x) for x in args.pbs.split(",")),
                  tps=tuple(int(x) for x in args.tps.split(",")),
                  skins=tuple(float(x) for x in args.skins.split(",")))
    if args.batch256:
        global VARIANTS
        VARIANTS = BATCH_VARIANTS
    best = at.tune(reps, device_measure(capi, reps, steps=args.steps, warmup=200), force=True,
                   variants=not args.no_variants)
    for r in best["table"]:
        print(f"pb={r['pb']:4d} tp={r['tp']} skin={r['skin']:.2f}  {r['rate']:.4e} particle-steps/s  "
              f"pe/N={r['pe']:.6f} {'ok' if r['ok'] else 'REJECTED'}")
    for r in best.get("variant_table", []):
        print(f"force_mode={r['force_mode']} sm_tiles={r['sm_tiles']} persistent={r['persistent']} "
              f"build_lanes={r['build_lanes']}  "
              f"{r['rate']:.4e} particle-steps/s  "
              f"pe/N={r['pe']:.6f} {'ok' if r['ok'] else 'REJECTED'}")
    print(json.dumps({k: best[k] for k in ("pb", "tp", "skin", "rate") + VARIANT_KEYS if k in best}))


if __name__ == "__main__":
    main()
