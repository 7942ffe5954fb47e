"""The persistent step kernels against one kernel launch per step:
  * k_steps (persistent = 1 when every tile has a resident block): fused
    steps back to back in one cooperative launch, a grid barrier between
    them, leaving the launch for each list rebuild;
  * k_batch (persistent = 2): whole steps, the list rebuilds included
    (sorts and builds claimed as work items), one grid barrier per step.
  * k_flow (persistent = 3, or 1 when the tiles outnumber the resident
    blocks): the same items, each replica stepping on its own through a
    queue of items whose inputs are complete (no step barrier).
They run the same per-replica arithmetic (sort, list, per-tile sums and
reduction tree), so every result must agree bit for bit."""
import numpy as np
import pytest

from test_gpu_parity import melted_ka

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from rumd_b200 import build, capi
    build.build_lib()
    return capi


@pytest.fixture(scope="module")
def ka_params(oracle):
    return oracle.lj_params(2, oracle.ka_table())


def engine(capi, persistent, pb=64, tp=2):
    e = capi.Engine(device=0, pb=pb, tp=tp)
    e.set_variant(capi.VARIANT_PERSISTENT, persistent)
    assert e.get_variant(capi.VARIANT_PERSISTENT) == persistent
    return e


def state(e, rid, n):
    return (e.get(rid, "pos", n), e.get(rid, "vel", n), e.get(rid, "images", n), e.get(rid, "force", n))


@pytest.mark.parametrize("pb,tp", [(64, 2), (32, 1), (64, 4), (128, 1)])
def test_trajectory_with_rebuilds_bit_identical(capi, ka_params, pb, tp):
    n = 5000
    m = melted_ka(capi, ka_params, n, steps=100, seed=3)
    res = []
    for persistent in (0, 1, 2):
        e = engine(capi, persistent, pb, tp)
        rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", dt=0.005, T=0.9, vel4=m["vel4"],
                    energy_interval=7, energy_capacity=200)
        e.run(333)
        e.run(41)  # a second run: new budget, momentum-reset schedule restarts
        res.append((state(e, rid, n), e.stats(rid), e.energy_log(rid)))
        e.close()
    s0, st0, log0 = res[0]
    for s1, st1, log1 in res[1:]:
        for a, b in zip(s0, s1):
            assert np.array_equal(a, b)
        assert st0["rebuilds"] == st1["rebuilds"] > 5
        for k in ("xi", "pe", "virial", "ke", "steps"):
            assert st0[k] == st1[k], k
        assert np.array_equal(log0, log1)


def test_batch_uneven_queues_bit_identical(capi, ka_params):
    """Replicas that finish at different steps leave the loop one by one."""
    from rumd_b200 import initconf as I
    sizes, temps, steps = [600, 2048, 777, 3000], [0.5, 1.0, 1.5, 2.0], [50, 131, 7, 90]
    confs = [I.ka_config(s, T=t, seed=s) for s, t in zip(sizes, temps)]
    res = []
    for persistent in (0, 1, 2):
        e = engine(capi, persistent)
        ids = [e.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", dt=0.005, T=t, vel4=c["vel4"])
               for c, t in zip(confs, temps)]
        for rid, k in zip(ids, steps):
            e.queue(rid, k)
        assert e.run_queued() == max(steps)
        res.append([(state(e, rid, s), e.stats(rid)) for rid, s in zip(ids, sizes)])
        e.close()
    for other in res[1:]:
        for (sa, ta), (sb, tb), k in zip(res[0], other, steps):
            assert ta["steps"] == tb["steps"] == k
            assert ta["xi"] == tb["xi"]
            for a, b in zip(sa, sb):
                assert np.array_equal(a, b)


def test_more_tiles_than_resident_blocks(capi, ka_params):
    """A batch larger than the GPU holds at once: persistent = 1 then runs
    k_flow (many tiles per block, rebuilds inside the launch, each replica
    stepping on its own), with the results of one launch per step."""
    from rumd_b200 import initconf as I
    c = I.ka_config(4000, T=1.0, seed=9)
    res = []
    for persistent in (0, 1):
        e = engine(capi, persistent, pb=32, tp=1)
        ids = [e.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", dt=0.005, T=1.0 + 0.01 * k, vel4=c["vel4"])
               for k in range(48)]  # 48 x 125 tiles of 32
        e.run(60)
        assert e.get_variant(capi.VARIANT_PERSISTENT_ACTIVE) == (3 if persistent else 0)
        res.append([e.get(rid, "pos", 4000) for rid in ids[::7]] + [e.stats(ids[-1])["xi"]] +
                   [e.stats(rid)["rebuilds"] for rid in ids])
        e.close()
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(a, b)


def test_batch_kernel_mixed_sizes_types_and_methods(capi, ka_params, oracle):
    """k_batch on a mix it must handle: replicas of one and two types, a
    small box on the all-pairs list (no sort), sizes from 2 to 6000, uneven
    step queues, and an energy log; against one launch per step (itself
    checked against the oracle elsewhere), bit for bit.  k_batch runs with
    every cell-method replica sorted in phases over many blocks (split
    threshold 1 tile), with the default threshold (16 tiles: the 6000, 3000
    and 1500-particle replicas) and with none split."""
    from rumd_b200 import initconf as I
    lj = oracle.lj_params(1, oracle.lj_table())
    specs = [("ka", 6000, 0.7, 90), ("lj", 3000, 1.2, 120), ("ka", 300, 2.0, 45), ("lj", 64, 1.0, 120),
             ("ka", 2, 1.0, 33), ("ka", 1500, 0.45, 120)]
    res = []
    for persistent, split in ((0, 16), (2, 1), (2, 16), (2, 1 << 20), (3, 1), (3, 16)):
        e = engine(capi, persistent)
        e.set_variant(capi.VARIANT_SPLIT_SORT_TILES, split)
        ids = []
        for kind, n, T, k in specs:
            c = (I.ka_config if kind == "ka" else I.lj_config)(n, T=T, seed=n)
            box = c["box"]
            if n == 2:
                box = np.array([4.0, 4.0, 4.0], np.float32)
                c["pos4"][:, :3] = [[0.0, 0.0, 0.0], [1.1, 0.2, -0.1]]
            rid = e.add(c["pos4"], box, ka_params if kind == "ka" else lj, 2 if kind == "ka" else 1, cutoff="SF",
                        dt=0.004, T=T, vel4=c["vel4"], energy_interval=5, energy_capacity=64)
            e.queue(rid, k)
            ids.append((rid, n, kind, box))
        assert e.run_queued() == 120
        if persistent:
            assert e.get_variant(capi.VARIANT_PERSISTENT_ACTIVE) == persistent
        res.append([(state(e, rid, n), e.stats(rid), e.energy_log(rid)) for rid, n, _, _ in ids])
        e.close()
    for other in res[1:]:
        for (sa, ta, la), (sb, tb, lb), spec in zip(res[0], other, specs):
            assert ta["steps"] == tb["steps"] == spec[3]
            assert ta["rebuilds"] == tb["rebuilds"]
            assert ta["xi"] == tb["xi"]
            assert np.array_equal(la, lb)
            for a, b in zip(sa, sb):
                assert np.array_equal(a, b)


def test_overflow_repair_under_persistent_runs(capi, ka_params):
    n = 4000
    m = melted_ka(capi, ka_params, n, steps=50, seed=13)
    res = []
    for persistent, cap in ((0, 0), (1, 40), (2, 40), (3, 40)):
        e = engine(capi, persistent)
        rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", vel4=m["vel4"], max_nbrs=cap)
        e.run(120)
        st = e.stats(rid)
        assert st["overflow"] == 0 and st["steps"] == 120
        res.append(e.get(rid, "pos", n))
        e.close()
    for other in res[1:]:
        assert np.array_equal(res[0], other)
