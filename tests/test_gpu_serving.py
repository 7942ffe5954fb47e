"""Serving on the GPU: jobs that arrive while others run are admitted into the
same launches (continuous batching), and every job's result is the same alone
and in the mix.  Stated tolerance: identical bits (the engine's per-replica
arithmetic and FP64 reduction trees do not depend on the other replicas)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_equal_results_alone():
    from rumd_b200 import capi, serving
    jobs = serving.poisson_stream(14, rate=400.0, seed=7, n_range=(256, 4096), steps_range=(200, 3000))
    eng = capi.Engine(device=0, max_replicas=16, pb=64, tp=4)
    srv = serving.MDServer(eng, hbm_budget=2e9, chunk_steps=128)
    mix = srv.serve(jobs)
    assert max(srv.queue_depth) >= 0
    overlap = sum(1 for a in mix for b in mix if a.id < b.id and a.admitted < b.done and b.admitted < a.done)
    assert overlap > 0, "jobs should share the GPU"
    eng.close()
    alone = serving.serve_one_at_a_time(lambda: capi.Engine(device=0, pb=64, tp=4),
                                        serving.poisson_stream(14, rate=400.0, seed=7, n_range=(256, 4096),
                                                               steps_range=(200, 3000)))
    by_id = {j.id: j for j in alone}
    for j in mix:
        a = by_id[j.id]
        assert j.result["steps"] == j.steps == a.result["steps"]
        assert j.result["pe"] == a.result["pe"]
        assert j.result["ke"] == a.result["ke"]
        assert j.result["xi"] == a.result["xi"]
    s = serving.latency_summary(mix)
    assert np.isfinite(s["p99_s"]) and s["throughput"] > 0
