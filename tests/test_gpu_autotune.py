"""Autotuner on the device: every candidate gives the same forces (pe
invariance, Autotune.py:929-937) and the chosen shape runs."""
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_small_grid(tmp_path):
    from rumd_b200 import autotune, capi, initconf
    c = initconf.ka_config(4000, T=1.0, seed=2)
    reps = [dict(pos4=c["pos4"], vel4=c["vel4"], box=c["box"], params=initconf.lj_params(2, initconf.KA),
                 ntypes=2, T=1.0, n=4000, density=1.2)]
    at = autotune.Autotune(cache_path=str(tmp_path / "at.json"), pbs=(32, 64), tps=(2, 4), skins=(0.3, 0.4))
    best = at.tune(reps, autotune.device_measure(capi, reps, steps=200, warmup=50), variants=True)
    assert all(r["ok"] for r in best["table"])
    assert all(r["ok"] for r in best["variant_table"])  # every variant: same pe
    assert best["rate"] >= max(r["rate"] for r in best["table"])
    e = capi.Engine()
    autotune.apply(e, best)
    assert e.get_variant(capi.VARIANT_BUILD_LANES) == best["build_lanes"]
    rid = e.add(c["pos4"], c["box"], reps[0]["params"], 2, skin=best["skin"], vel4=c["vel4"])
    e.run(100)
    assert e.stats(rid)["steps"] == 100
    e.close()
