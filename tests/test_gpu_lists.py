"""Neighbour lists and the sort permutation against the oracle, bit for bit,
beyond a single build from the identity order:

  * across in-run rebuilds: RUMD re-sorts already-sorted particles at every
    rebuild (a stable sort by cell key, ties broken by the current slot,
    Sample.h:174-188), so the permutation is a chain of stable sorts.  The
    run goes step by step (Sample::CalcF + Integrate); before each force
    evaluation the test records the particles' positions in slot order, and
    whenever the engine rebuilds it replays the oracle's stable sort of those
    positions and compares the cumulative permutation (d_unsorted_index) and
    the list, entries and order;
  * on the configurations the benchmark names: Kob-Andersen N=1000 at
    density 1.2 (L = 9.41, 6 cells a side), RUMD's own N256L6.0 file with the
    cell method (5 cells a side, the stencil's minimum, every row wraps), and
    single-component LJ at density 0.8442 (N = 32000 and N = 1,048,576);
  * the Kob-Andersen N=1000 run itself (T = 0.73, seeds 1, 2, 3, 1000 steps):
    per-step energies against the FP32 oracle over the first 100 steps, mean
    energies over the run, and forces and lists at its final state.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from rumd_b200 import build, capi
    build.build_lib()
    return capi


@pytest.fixture(scope="module")
def ka_params(oracle):
    return oracle.lj_params(2, oracle.ka_table())


@pytest.fixture(scope="module")
def lj_params(oracle):
    return oracle.lj_params(1, oracle.lj_table())


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def compare_lists(gc, gl, uidx, counts, nbl):
    """GPU list (original ids, row i = particle i) against the oracle's list
    in sorted space (row s = slot s, entries are slots); uidx[s] = original id
    of slot s.  Entries and order, all particles, vectorised."""
    n = len(uidx)
    g_counts = gc[uidx]
    assert np.array_equal(g_counts, counts), int((g_counts != counts).sum())
    width = int(counts.max()) if n else 0
    mask = np.arange(width)[None, :] < counts[:, None].astype(np.int64)
    g_rows = gl[uidx][:, :width]
    o_rows = uidx[nbl[:, :width]]
    assert np.array_equal(g_rows[mask], o_rows[mask])


def identity_build(capi, oracle, pos4, box, params, ntypes, skin=0.3, max_nbrs=400, method=None):
    """A fresh replica (identity order) built once, against the oracle."""
    n = len(pos4)
    e = capi.Engine(device=0, pb=64, tp=4, max_particles=n)
    rid = e.add(pos4, box, params, ntypes, cutoff="SF", skin=skin)
    if method:
        e.set_nb_method(rid, method)
    e.calc_f()
    L = np.asarray(box, np.float32)
    nc = oracle.cell_grid(L, oracle.max_cutoff(params, ntypes), skin)
    if method == "sort":
        nc = np.maximum(nc, 5)
    keys = oracle.cell_keys(pos4, L, nc)
    old = oracle.stable_sort_perm(keys, int(np.prod(nc)))
    counts, nbl, ov = oracle.nbl_cells(pos4[old], L, nc, ntypes, params, skin, max_nbrs)
    assert not ov
    assert np.array_equal(e.cell_grid(rid), nc)
    uidx = e.sort_index(rid, n)
    assert np.array_equal(uidx, old)
    gc, gl = e.nbl(rid, n, max_nbrs)
    compare_lists(gc, gl, uidx, counts, nbl)
    st = e.stats(rid)
    e.close()
    return st


@pytest.mark.parametrize("build_lanes", [0, 32])
def test_permutation_and_lists_across_in_run_rebuilds(capi, oracle, ka_params, build_lanes):
    from rumd_b200 import initconf as I
    n, skin = 4096, 0.3
    c = I.ka_config(n, T=1.0, seed=17)
    e = capi.Engine(device=0, pb=64, tp=4)
    e.set_variant(capi.VARIANT_BUILD_LANES, build_lanes)
    rid = e.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", skin=skin, dt=0.005, T=1.0, vel4=c["vel4"])
    L = np.asarray(c["box"], np.float32)
    nc = oracle.cell_grid(L, oracle.max_cutoff(ka_params, 2), skin)
    seen = 0
    for step in range(120):
        u_prev = e.sort_index(rid, n)
        pos_slot = e.get(rid, "pos", n)[u_prev]        # positions in the current slot order
        r0 = e.stats(rid)["rebuilds"]
        e.calc_f()
        if e.stats(rid)["rebuilds"] > r0:
            keys = oracle.cell_keys(pos_slot, L, nc)
            perm = oracle.stable_sort_perm(keys, int(np.prod(nc)))  # new slot -> old slot
            u_new = e.sort_index(rid, n)
            assert np.array_equal(u_new, u_prev[perm]), step
            counts, nbl, ov = oracle.nbl_cells(pos_slot[perm], L, nc, 2, ka_params, skin, 400)
            assert not ov
            gc, gl = e.nbl(rid, n, 400)
            compare_lists(gc, gl, u_new, counts, nbl)
            seen += 1
        e.integrate()
    # the first build is from the identity order; the rest re-sort sorted data
    assert seen >= 4, seen
    assert not np.array_equal(e.sort_index(rid, n), np.arange(n))
    e.close()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_lists_kob_andersen_n1000(capi, oracle, ka_params, seed):
    """The small plain configuration: N = 1000 at density 1.2, L = 9.41 (six
    cells a side, so many rows wrap), melted from the FCC start at T = 0.73."""
    from rumd_b200 import initconf as I
    n = 1000
    c = I.ka_config(n, T=0.73, seed=seed)
    e = capi.Engine(device=0, pb=64, tp=4)
    rid = e.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", dt=0.005, T=0.73, vel4=c["vel4"])
    e.run(300)
    pos4 = e.get(rid, "pos", n)
    e.close()
    assert abs(float(c["box"][0]) - 9.41) < 0.01
    identity_build(capi, oracle, pos4, c["box"], ka_params, 2)


def test_lists_five_cell_reference_configuration(capi, oracle, ka_params):
    """RUMD's Conf/KobAndersen/N256L6.0: L = 6 gives floor(2L/(rc+skin)) = 4
    cells, raised to the stencil's minimum of 5, so the 5x5x5 stencil covers
    the whole box and every row wraps; the cell method is forced."""
    g = load_golden(os.path.join(GOLDEN, "ka_N256L6.0.npz"))
    pos4 = np.zeros((len(g["pos"]), 4), np.float32)
    pos4[:, :3] = g["pos"]
    pos4[:, 3] = g["type"].astype(np.int32).view(np.float32)
    st = identity_build(capi, oracle, pos4, g["L"], ka_params, 2, method="sort")
    assert st["mean_nbrs"] > 0


@pytest.mark.parametrize("n", [32000, 1048576])
def test_lists_single_component_lj(capi, oracle, lj_params, n):
    """Single-component LJ at density 0.8442 (SF rc = 2.5): N = 32000 and the
    HBM-scale N = 1,048,576 (76 cells a side)."""
    from rumd_b200 import initconf as I
    c = I.lj_config(n, density=0.8442, T=1.5, seed=8)
    e = capi.Engine(device=0, pb=64, tp=4, max_particles=n)
    rid = e.add(c["pos4"], c["box"], lj_params, 1, cutoff="SF", dt=0.004, T=1.5, vel4=c["vel4"])
    e.run(200)
    pos4 = e.get(rid, "pos", n)
    e.close()
    identity_build(capi, oracle, pos4, c["box"], lj_params, 1, max_nbrs=256)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_kob_andersen_n1000_run(capi, oracle, ka_params, seed):
    """The small plain configuration run as specified: KA N = 1000, FCC start
    with seeded types and Maxwell-Boltzmann velocities at T = 0.73, NVT
    tau = 0.2, dt = 0.005, skin 0.3, 1000 steps, on the GPU and with the FP32
    oracle from the same state.  Per-step energies agree over the first 100
    steps (RUMD_Test tolerances, 1e-4 relative); after that FP32 round-off
    makes the trajectories decorrelate, so the run-averaged potential and
    kinetic energies per particle are compared (0.05), and at the GPU's final
    state the forces meet 1e-5 against the FP64 oracle and the list is the
    oracle's bit for bit."""
    from rumd_b200 import initconf as I
    n, steps = 1000, 1000
    c = I.ka_config(n, T=0.73, seed=seed)
    e = capi.Engine(device=0, pb=64, tp=4)
    rid = e.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", dt=0.005, T=0.73, tau=0.2, vel4=c["vel4"],
                energy_interval=1, energy_capacity=steps)
    e.run(steps)
    log = e.energy_log(rid)
    pos4 = e.get(rid, "pos", n)
    f = e.get(rid, "force", n)
    st = e.stats(rid)
    e.close()
    ref = oracle.md_run(c["pos4"], c["vel4"], c["im3"], c["box"], 2, ka_params, oracle.SF, 0.3, 0.005, 0.73, 0.2,
                        steps)
    assert len(log) == steps
    # the lattice melts in these steps and pe passes through zero, so the
    # 1e-4 is relative to the run's energy scale
    for col, rcol in ((1, 0), (3, 2)):
        scale = np.abs(ref["energies"][:100, rcol]).max()
        assert np.abs(log[:100, col] - ref["energies"][:100, rcol]).max() <= 1e-4 * scale, col
    half = slice(steps // 2, steps)
    # two independent stretches of 500 correlated steps of N = 1000
    assert abs(log[half, 1].mean() - ref["energies"][half, 0].mean()) / n < 0.05
    assert abs(log[half, 3].mean() - ref["energies"][half, 2].mean()) / n < 0.05
    assert st["rebuilds"] >= 10
    types = pos4[:, 3].view(np.int32)
    fref, u, w = oracle.forces_f64(pos4[:, :3].astype(np.float64), types, c["box"], 2, ka_params, oracle.SF)
    assert rms_rel(f[:, :3].astype(np.float64), fref) <= 1e-5
    identity_build(capi, oracle, pos4, c["box"], ka_params, 2)


def test_lists_asymmetric_cutoff_table(capi, oracle, ka_params):
    """A pair table whose (A, B) and (B, A) cut-offs differ (RUMD stores the
    table per ordered type pair): each particle's list uses its own row of the
    table, as the oracle's does."""
    from rumd_b200 import initconf as I
    n = 4096
    params = ka_params.copy().reshape(4, -1)
    params[2, 0] = params[1, 0] * 0.9  # rc of (1, 0) below that of (0, 1)
    params = params.reshape(-1)
    c = I.ka_config(n, T=1.0, seed=21)
    identity_build(capi, oracle, c["pos4"], c["box"], params, 2)


def test_lists_over_full_cell(capi, oracle, lj_params):
    """LJ at density 0.8442 with 70 particles moved into a cube of side 1.2 --
    one cell holds them all and the rows through it have over a hundred
    candidates; then the particles are spread again and the same engine
    rebuilds.  Both lists are the oracle's."""
    from rumd_b200 import initconf as I
    n, k = 32000, 70
    c = I.lj_config(n, density=0.8442, T=1.0, seed=5)
    pos_blob = c["pos4"].copy()
    rng = np.random.default_rng(5)
    centre = np.asarray(c["box"], np.float32) * 0.3
    pos_blob[:k, :3] = centre + rng.uniform(-0.6, 0.6, (k, 3)).astype(np.float32)
    box = c["box"]
    identity_build(capi, oracle, pos_blob, box, lj_params, 1, max_nbrs=400)
    spread = I.lj_config(n, density=0.8442, T=1.0, seed=6)["pos4"]
    e = capi.Engine(device=0, pb=64, tp=4, max_particles=n)
    rid = e.add(pos_blob, box, lj_params, 1, cutoff="SF", skin=0.3, max_nbrs=400)
    e.calc_f()
    assert e.stats(rid)["rebuilds"] == 1
    e.set(rid, "pos", spread)
    e.calc_f()
    assert e.stats(rid)["rebuilds"] == 2
    L = np.asarray(box, np.float32)
    nc = oracle.cell_grid(L, oracle.max_cutoff(lj_params, 1), 0.3)
    uidx = e.sort_index(rid, n)
    pos_slot = e.get(rid, "pos", n)[uidx]
    counts, nbl, ov = oracle.nbl_cells(pos_slot, L, nc, 1, lj_params, 0.3, 400)
    assert not ov
    gc, gl = e.nbl(rid, n, 400)
    compare_lists(gc, gl, uidx, counts, nbl)
    e.close()
