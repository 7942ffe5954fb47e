"""Autotuner search logic on the CPU (fake timings)."""
import json


def test_candidates_respect_block_limit():
    from rumd_b200 import autotune
    c = autotune.candidates()
    assert all(pb * tp <= 512 for pb, tp, _ in c)
    assert (128, 8, 0.3) not in c and (64, 8, 0.3) in c


def test_search_picks_fastest_valid_candidate():
    from rumd_b200 import autotune

    def measure(pb, tp, skin):
        rate = pb * tp / (1 + abs(skin - 0.3) * 10)
        pe = -5.0 if (pb, tp) != (64, 8) else -4.9  # (64, 8) breaks the pe invariance
        return rate, pe

    best, table = autotune.search(autotune.candidates(), measure)
    assert (best["pb"], best["tp"], best["skin"]) == (128, 4, 0.3)
    assert any(not r["ok"] for r in table)


def test_cache_round_trip(tmp_path):
    from rumd_b200 import autotune
    calls = []

    def measure(pb, tp, skin):
        calls.append((pb, tp, skin))
        return float(tp), -5.0

    reps = [{"n": 1000, "density": 1.2, "ntypes": 2}]
    at = autotune.Autotune(cache_path=str(tmp_path / "a.json"), pbs=(32, 64), tps=(1, 2), skins=(0.3,))
    r1 = at.tune(reps, measure)
    n = len(calls)
    r2 = at.tune(reps, measure)
    assert len(calls) == n and r1["tp"] == r2["tp"] == 2
    assert json.load(open(tmp_path / "a.json"))


def test_variant_stage_picks_fastest_and_is_cached(tmp_path):
    from rumd_b200 import autotune

    def measure(pb, tp, skin, force_mode=None, build_lanes=None, sm_tiles=None, persistent=None):
        if force_mode is None:
            return float(pb * tp), -5.0
        # streamed index loads, the persistent kernel and two build lanes
        # fastest; staged with one lane breaks pe
        rate = 1000.0 + (200.0 if force_mode == 0 else 0.0) - 10.0 * abs(build_lanes - 2) + 5.0 * (persistent or 0)
        pe = -5.0 if (force_mode, build_lanes) != (1, 1) else -4.0
        return rate, pe

    reps = [{"n": 2000, "density": 1.2, "ntypes": 2}]
    at = autotune.Autotune(cache_path=str(tmp_path / "v.json"), pbs=(32, 64), tps=(1, 2), skins=(0.3,))
    r = at.tune(reps, measure, variants=True)
    assert (r["force_mode"], r["build_lanes"], r["persistent"]) == (0, 2, 1)
    assert len(r["variant_table"]) == len(autotune.VARIANTS)
    assert any(not v["ok"] for v in r["variant_table"])
    assert json.load(open(tmp_path / "v.json"))[autotune.signature(reps)]["build_lanes"] == 2
