"""Serving on the GPU: jobs that arrive while others run are admitted into the
same launches (continuous batching), and every job's result is the same alone
and in the mix.  Stated tolerance: identical bits (the engine's per-replica
arithmetic and FP64 reduction trees do not depend on the other replicas).

Admission and removal do not wait for running work: the uploads queue behind
the chunks in flight, and the memory of a removed replica can be handed to a
new one while a chunk that still holds the old one runs.  The tests check
both that this stays bit-exact and that a batched graph survives it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stream():
    from rumd_b200 import serving
    return serving.poisson_stream(14, rate=400.0, seed=7, n_range=(256, 4096), steps_range=(200, 3000))


@pytest.mark.parametrize("persistent", [1, 2, 3])
def test_served_results_equal_results_alone(persistent):
    from rumd_b200 import capi, serving
    eng = capi.Engine(device=0, max_replicas=16, max_particles=1 << 16, pb=64, tp=4)
    eng.set_variant(capi.VARIANT_PERSISTENT, persistent)
    srv = serving.MDServer(eng, hbm_budget=2e9, chunk_steps=128)
    mix = srv.serve(_stream())
    assert srv.chunks > 2
    overlap = sum(1 for a in mix for b in mix if a.id < b.id and a.admitted < b.done and b.admitted < a.done)
    assert overlap > 0, "jobs should share the GPU"
    assert eng.usage()[0] == 0 and srv.max_used > 0
    eng.close()
    alone = serving.serve_one_at_a_time(lambda: capi.Engine(device=0, pb=64, tp=4), _stream())
    by_id = {j.id: j for j in alone}
    for j in mix:
        a = by_id[j.id]
        assert j.result["steps"] == j.steps == a.result["steps"]
        assert j.result["pe"] == a.result["pe"]
        assert j.result["ke"] == a.result["ke"]
        assert j.result["xi"] == a.result["xi"]
    s = serving.latency_summary(mix)
    assert np.isfinite(s["p99_s"]) and s["throughput"] > 0


def _ka(initconf, n, seed):
    c = initconf.ka_config(n, T=1.0, seed=seed)
    return c, initconf.lj_params(2, initconf.KA)


def _alone(capi, c, params, steps):
    e = capi.Engine(device=0, pb=128, tp=2)
    rid = e.add(c["pos4"], c["box"], params, 2, vel4=c["vel4"])
    e.queue(rid, steps)
    e.run_queued(0)
    st = e.stats(rid)
    pos = e.get(rid, "pos", len(c["pos4"]))
    e.close()
    return st, pos


@pytest.mark.parametrize("persistent", [2, 3])
def test_admission_and_removal_under_a_running_chunk(persistent):
    """k_batch (k_flow) engine: replicas A, B run; while a chunk holds A, A is
    removed and C admitted into A's id and memory; C and B must equal
    themselves alone, and the batched graph is built once."""
    from rumd_b200 import capi, initconf
    e = capi.Engine(device=0, max_replicas=8, max_particles=1 << 15, pb=128, tp=2)
    e.set_variant(capi.VARIANT_PERSISTENT, persistent)
    ca, p = _ka(initconf, 2048, 1)
    cb, _ = _ka(initconf, 3000, 2)
    cc, _ = _ka(initconf, 2048, 3)
    a = e.add(ca["pos4"], ca["box"], p, 2, vel4=ca["vel4"])
    b = e.add(cb["pos4"], cb["box"], p, 2, vel4=cb["vel4"])
    e.queue(a, 5000)
    e.queue(b, 1500)
    t1 = e.run_queued_async(400)
    assert e.get_variant(capi.VARIANT_PERSISTENT_ACTIVE) == persistent
    builds = e.get_variant(capi.VARIANT_GRAPH_BUILDS)
    e.remove(a)  # A is still being advanced by chunk t1
    c = e.add(cc["pos4"], cc["box"], p, 2, vel4=cc["vel4"])
    assert c == a  # the freed id (and particle range) is reused
    e.queue(c, 1200)
    ran1, snap1 = e.wait(t1)
    assert ran1 == 400
    assert snap1[b, 2] == 1100  # B's steps left after the chunk
    left = 1
    while left > 0:
        t = e.run_queued_async(300)
        ran, snap = e.wait(t)
        left = max(snap[b, 2], snap[c, 2])
    assert e.get_variant(capi.VARIANT_GRAPH_BUILDS) == builds
    sb, sc = e.stats(b), e.stats(c)
    pb_ = e.get(b, "pos", 3000)
    pc = e.get(c, "pos", 2048)
    e.close()
    for st, pos, conf, steps in ((sb, pb_, cb, 1500), (sc, pc, cc, 1200)):
        ref, rpos = _alone(capi, conf, p, steps)
        assert st["steps"] == ref["steps"] == steps
        assert st["pe"] == ref["pe"] and st["ke"] == ref["ke"] and st["xi"] == ref["xi"]
        assert np.array_equal(pos, rpos)


def test_footprint_matches_usage():
    from rumd_b200 import capi, initconf
    e = capi.Engine(device=0, max_replicas=4, pb=64, tp=4)
    c, p = _ka(initconf, 4000, 5)
    fp = e.footprint(4000, c["box"], p, 2)
    rid = e.add(c["pos4"], c["box"], p, 2, vel4=c["vel4"])
    assert e.usage()[0] == fp
    e.calc_f()  # the tile tables are laid out (and grown) before the first launch
    used, reserved = e.usage()
    assert used == fp and reserved >= used
    e.remove(rid)
    assert e.usage()[0] == 0
    e.close()


def test_list_repair_between_chunks_keeps_results_and_graph():
    """A replica whose list is too small overflows at its first build; the
    chunk's wait enlarges the list from the snapshot, without waiting for the
    chunk in flight and without rebuilding the step graph, and the replica
    then catches up: its result equals the same replica's queued steps run
    with b2md_run_queued (synchronous repair), bit for bit."""
    from rumd_b200 import capi, initconf
    c, p = _ka(initconf, 3000, 11)
    d, _ = _ka(initconf, 2000, 12)
    e = capi.Engine(device=0, max_replicas=4, max_particles=1 << 14, pb=128, tp=2)
    e.set_variant(capi.VARIANT_PERSISTENT, 3)
    a = e.add(c["pos4"], c["box"], p, 2, vel4=c["vel4"], max_nbrs=40)
    b = e.add(d["pos4"], d["box"], p, 2, vel4=d["vel4"])
    e.queue(a, 600)
    e.queue(b, 600)
    left = 1
    while left > 0:
        t1 = e.run_queued_async(150)
        t2 = e.run_queued_async(150)
        e.wait(t1)
        _, snap = e.wait(t2)
        left = max(snap[a, 2], snap[b, 2])
    cnt = e.counters()
    assert cnt["list_repairs"] >= 1 and cnt["graphs_dropped_by_list_repair"] == 0
    sa = e.stats(a)
    pa = e.get(a, "pos", 3000)
    e.close()
    ref = capi.Engine(device=0, pb=128, tp=2)
    r = ref.add(c["pos4"], c["box"], p, 2, vel4=c["vel4"], max_nbrs=40)
    ref.queue(r, 600)
    ref.run_queued(0)
    assert sa["steps"] == ref.stats(r)["steps"] == 600
    assert sa["pe"] == ref.stats(r)["pe"] and sa["xi"] == ref.stats(r)["xi"]
    assert np.array_equal(pa, ref.get(r, "pos", 3000))
    ref.close()
