"""GPU parity: the CUDA path (called through the C ABI) against the CPU oracle.

Tolerances
  * neighbour lists and the sort permutation: bit-exact (sets in original ids,
    and the list order in sorted space);
  * forces: rms relative error <= 1e-5 against the FP64 oracle pair sum;
  * energies: relative 1e-5 against the FP64 oracle for the same positions;
  * short trajectories (<= 100 steps) against the FP32 oracle: positions and
    velocities within 1e-3 (RUMD_Test.py:49-55 trajectory tolerances),
    energies within 1e-4 relative (RUMD_Test.py:57-65).
"""
import numpy as np
import pytest

from conftest import golden_files, load_golden

pytestmark = pytest.mark.gpu

FILES = golden_files()


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def golden_pos4(g):
    pos4 = np.zeros((len(g["pos"]), 4), np.float32)
    pos4[:, :3] = g["pos"]
    pos4[:, 3] = g["type"].astype(np.int32).view(np.float32)
    return pos4


def golden_vel4(g):
    v = np.zeros((len(g["pos"]), 4), np.float32)
    v[:, :3] = g["vel"]
    v[:, 3] = 1.0
    return v


@pytest.fixture(scope="module")
def capi():
    from rumd_b200 import build, capi
    build.build_lib()
    return capi


@pytest.fixture(scope="module")
def ka_params(oracle):
    return oracle.lj_params(2, oracle.ka_table())


def new_engine(capi, pb=64, tp=4):
    return capi.Engine(device=0, pb=pb, tp=tp)


def melted_ka(capi, ka_params, n, T=2.0, steps=400, seed=0, cutoff="SF"):
    """A disordered KA configuration: the FCC start melted on the GPU."""
    from rumd_b200 import initconf as I
    c = I.ka_config(n, T=T, seed=seed)
    e = new_engine(capi)
    rid = e.add(c["pos4"], c["box"], ka_params, 2, cutoff=cutoff, dt=0.004, T=T, vel4=c["vel4"])
    e.run(steps)
    out = dict(pos4=e.get(rid, "pos", n), vel4=e.get(rid, "vel", n), im3=e.get(rid, "images", n), box=c["box"])
    e.close()
    return out


# ---------------------------------------------------------------------------
# arithmetic of the neighbour-list decisions
# ---------------------------------------------------------------------------

def test_dist2_explicit_form_equals_nvcc_contraction_of_reference_expression(capi):
    rng = np.random.default_rng(1)
    L = np.array([37.94, 37.94, 37.94], np.float32)
    n = 1 << 20
    a = np.zeros((n, 4), np.float32)
    b = np.zeros((n, 4), np.float32)
    a[:, :3] = rng.uniform(-L / 2, L / 2, (n, 3))
    # partners near the list cut-off (2.8) and across the periodic boundary
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    b[:, :3] = a[:, :3] + d * rng.uniform(2.7, 2.9, (n, 1))
    b[:, :3] -= L * np.rint(b[:, :3] / L)
    out = capi.probe_dist2(a, b, L)
    assert np.array_equal(out[:, 0].view(np.uint32), out[:, 1].view(np.uint32))


def test_cell_coordinate_explicit_form_equals_reference_expression(capi):
    rng = np.random.default_rng(2)
    L, nc = np.float32(37.94), 27
    x = rng.uniform(-L / 2, L / 2, 1 << 20).astype(np.float32)
    # include coordinates next to every cell boundary
    edges = (np.arange(nc + 1, dtype=np.float64) / nc - 0.5) * float(L)
    near = np.concatenate([np.nextafter(edges.astype(np.float32), s) for s in (-np.inf, np.inf)] +
                          [edges.astype(np.float32)])
    x = np.concatenate([x, near.astype(np.float32)])
    out = capi.probe_cell(x, L, nc)
    assert np.array_equal(out[:, 0], out[:, 1])


@pytest.mark.parametrize("dt", [0.005, 0.004, 0.0025])
def test_nvt_update_explicit_form_equals_nvcc_contraction_of_reference_expression(capi, dt):
    """integrateNVTAlgorithm's velocity and position update and the periodic
    wrap (IntegratorNVT.cu:385-399, SimulationBox.h:140-155), compiled as
    written with default nvcc flags, against the engine's explicit forms
    (nvt_coef / nvt_velocity / nvt_position / wrap_*), bit for bit, on 2^20
    random states: thermostat states across and beyond the range runs reach
    (xi = 0 included), forces up to the r^-13 wall, particles that leave the
    box on any face."""
    rng = np.random.default_rng(5)
    n = 1 << 20
    L = np.array([37.94, 9.41, 107.49], np.float32)
    r = np.zeros((n, 4), np.float32)
    v = np.zeros((n, 4), np.float32)
    f = np.zeros((n, 4), np.float32)
    r[:, :3] = rng.uniform(-L / 2, L / 2, (n, 3))
    r[: n // 8, :3] = (L / 2) * np.sign(rng.normal(size=(n // 8, 3))) * rng.uniform(0.999, 1.0, (n // 8, 3))
    v[:, :3] = rng.normal(size=(n, 3)) * rng.uniform(0.3, 3.0, (n, 1))
    v[:, 3] = rng.choice(np.array([1.0, 0.5, 1.0 / 3.0], np.float32), n)
    f[:, :3] = rng.normal(size=(n, 3)) * np.exp(rng.uniform(0, 8, (n, 1)))
    xi = rng.normal(size=n).astype(np.float32) * 2.0
    xi[::16] = 0.0
    ref, eng = capi.probe_nvt(r, v, f, xi, dt, L)
    bad = (ref.view(np.uint32) != eng.view(np.uint32)).sum(axis=0)
    assert bad.sum() == 0, dict(zip(["vx", "vy", "vz", "x", "y", "z", "kx", "ky", "kz"], bad.tolist()))


def test_explicit_dist2_matches_oracle_restatement(capi, oracle):
    """The oracle (fmaf on the CPU) and the GPU agree bit for bit."""
    rng = np.random.default_rng(3)
    L = np.array([9.41, 10.0, 107.49], np.float32)
    n = 1 << 18
    a = np.zeros((n, 4), np.float32)
    b = np.zeros((n, 4), np.float32)
    a[:, :3] = rng.uniform(-L / 2, L / 2, (n, 3))
    b[:, :3] = rng.uniform(-L / 2, L / 2, (n, 3))
    out = capi.probe_dist2(a, b, L)
    ref = oracle.dist2(a, b, L)
    assert np.array_equal(out[:, 1].view(np.uint32), ref.view(np.uint32))


# ---------------------------------------------------------------------------
# forces, energies, virial
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("path", FILES, ids=[p.split("/")[-1][3:-4] for p in FILES])
def test_forces_on_reference_configurations(capi, oracle, ka_params, path):
    """GPU forces on RUMD's own configurations: vs the FP64 oracle (1e-5) and
    vs the forces RUMD stored in the files (SP cut-off, print precision)."""
    g = load_golden(path)
    pos4 = golden_pos4(g)
    n = len(pos4)
    for cutoff in ("SP", "SF", "NS"):
        e = new_engine(capi)
        rid = e.add(pos4, g["L"], ka_params, 2, cutoff=cutoff, vel4=golden_vel4(g))
        e.calc_f()
        f = e.get(rid, "force", n)
        w = e.get(rid, "virial", n)
        st = e.stats(rid)
        ref, u, w64 = oracle.forces_f64(pos4[:, :3].astype(np.float64), g["type"], g["L"], 2, ka_params,
                                        capi.CUTOFF[cutoff])
        assert rms_rel(f[:, :3].astype(np.float64), ref) <= 1e-5, cutoff
        assert abs(st["pe"] - u.sum()) <= 1e-5 * abs(u.sum())
        assert abs(st["virial"] - w64.sum() / 6) <= 1e-5 * abs(w64.sum() / 6) + 1e-3
        assert np.abs(f[:, 3] - u).max() < 1e-4
        assert np.abs(w[:, 3] - w64).max() < 1e-3 * max(1.0, np.abs(w64).max() / 100)
        if cutoff == "SP":
            assert rms_rel(f[:, :3].astype(np.float64), g["force"]) < 2e-5
            assert np.abs(f[:, 3] - g["pe"]).max() < 2e-4
            if "vir" in g:
                assert np.abs(w[:, 3] / 2 - g["vir"]).max() < 2e-3
        e.close()


@pytest.mark.parametrize("n", [4000, 65536])
@pytest.mark.parametrize("tp", [1, 2, 4, 8])
def test_forces_large_melt_all_tp(capi, oracle, ka_params, n, tp):
    m = melted_ka(capi, ka_params, n, steps=200)
    e = capi.Engine(device=0, pb=64 if tp <= 4 else 32, tp=tp)
    rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", vel4=m["vel4"])
    e.calc_f()
    f = e.get(rid, "force", n)
    types = m["pos4"][:, 3].view(np.int32)
    ref, u, w = oracle.forces_f64(m["pos4"][:, :3].astype(np.float64), types, m["box"], 2, ka_params, 2)
    assert rms_rel(f[:, :3].astype(np.float64), ref) <= 1e-5
    assert abs(e.stats(rid)["pe"] - u.sum()) <= 1e-5 * abs(u.sum())
    e.close()


def test_single_component_lj_forces(capi, oracle):
    from rumd_b200 import initconf as I
    params = oracle.lj_params(1, oracle.lj_table())
    c = I.lj_config(32000, T=3.0, seed=5)
    e = new_engine(capi)
    rid = e.add(c["pos4"], c["box"], params, 1, cutoff="SF", dt=0.004, T=3.0, vel4=c["vel4"])
    e.run(300)
    pos = e.get(rid, "pos", 32000)
    f = e.get(rid, "force", 32000)
    ref, u, w = oracle.forces_f64(pos[:, :3].astype(np.float64), np.zeros(32000, np.int32), c["box"], 1, params, 2)
    assert rms_rel(f[:, :3].astype(np.float64), ref) <= 1e-5
    e.close()


# ---------------------------------------------------------------------------
# neighbour list and sort permutation (bit-exact)
# ---------------------------------------------------------------------------

def oracle_sorted_list(oracle, pos4, L, params, ntypes, skin, max_nbrs):
    L = np.asarray(L, np.float32)
    nc = oracle.cell_grid(L, oracle.max_cutoff(params, ntypes), skin)
    keys = oracle.cell_keys(pos4, L, nc)
    old = oracle.stable_sort_perm(keys, int(np.prod(nc)))
    counts, nbl, ov = oracle.nbl_cells(pos4[old], L, nc, ntypes, params, skin, max_nbrs)
    return nc, old, counts, nbl, ov


@pytest.mark.parametrize("n", [4096, 20000, 65536])
def test_neighbour_list_and_permutation_bit_exact(capi, oracle, ka_params, n):
    m = melted_ka(capi, ka_params, n, steps=150, seed=n)
    e = new_engine(capi)
    rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", vel4=m["vel4"])
    e.calc_f()  # fresh replica: identity order, so the sort permutation is one stable sort
    nc, old, counts, nbl, ov = oracle_sorted_list(oracle, m["pos4"], m["box"], ka_params, 2, 0.3, 400)
    assert not ov
    assert np.array_equal(e.cell_grid(rid), nc)
    assert np.array_equal(e.sort_index(rid, n), old)
    gc, gl = e.nbl(rid, n, 400)
    # same entries in the same order, in original particle ids
    for s in range(n):
        i = old[s]
        assert gc[i] == counts[s]
        assert np.array_equal(gl[i, : gc[i]], old[nbl[s, : counts[s]]])
    e.close()


@pytest.mark.parametrize("lanes", [0, 2, 32])
def test_n2_and_sort_methods_give_same_sets(capi, oracle, ka_params, lanes):
    n = 5000
    m = melted_ka(capi, ka_params, n, steps=100, seed=7)
    sets = []
    for method in ("sort", "n2"):
        e = new_engine(capi)
        e.set_variant(capi.VARIANT_BUILD_LANES, lanes)
        rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", vel4=m["vel4"])
        e.set_nb_method(rid, method)
        e.calc_f()
        c, l = e.nbl(rid, n, 400)
        sets.append([frozenset(l[i, : c[i]].tolist()) for i in range(n)])
        e.close()
    assert sets[0] == sets[1]
    c2, n2, _ = oracle.nbl_n2(m["pos4"], m["box"], 2, ka_params, 0.3, 400)
    assert sets[1] == [frozenset(n2[i, : c2[i]].tolist()) for i in range(n)]


# ---------------------------------------------------------------------------
# trajectories
# ---------------------------------------------------------------------------

def min_image(d, L):
    return d - L * np.round(d / L)


@pytest.mark.parametrize("path", [p for p in FILES if "KA_N1000_T1.0" in p or "N2000" in p])
def test_short_trajectory_matches_fp32_oracle(capi, oracle, ka_params, path):
    g = load_golden(path)
    pos4, vel4 = golden_pos4(g), golden_vel4(g)
    n = len(pos4)
    im3 = np.zeros((n, 3), np.int32)
    steps = 100
    ref = oracle.md_run(pos4, vel4, im3, g["L"], 2, ka_params, oracle.SF, 0.3, 0.005, 0.8, 0.2, steps)
    e = new_engine(capi)
    rid = e.add(pos4, g["L"], ka_params, 2, cutoff="SF", dt=0.005, T=0.8, tau=0.2, vel4=vel4,
                energy_interval=1, energy_capacity=steps)
    e.run(steps)
    p = e.get(rid, "pos", n)
    v = e.get(rid, "vel", n)
    im = e.get(rid, "images", n)
    L = g["L"].astype(np.float64)
    unwrap_g = p[:, :3].astype(np.float64) + im * L
    unwrap_o = ref["pos4"][:, :3].astype(np.float64) + ref["im3"] * L
    assert np.abs(unwrap_g - unwrap_o).max() < 1e-3
    assert np.abs(v[:, :3] - ref["vel4"][:, :3]).max() < 1e-3
    log = e.energy_log(rid)
    assert len(log) == steps
    # pe(t), W(t), KE(t), xi per step
    assert np.allclose(log[:, 1], ref["energies"][:, 0], rtol=1e-4)
    assert np.allclose(log[:, 3], ref["energies"][:, 2], rtol=1e-4)
    assert np.allclose(log[:, 4], ref["energies"][:, 3], rtol=1e-3, atol=1e-4)
    assert e.stats(rid)["rebuilds"] >= 2
    e.close()


def test_fused_run_equals_separate_calcf_integrate(capi, ka_params):
    """Simulation.Run through the fused graph path == the step-by-step API."""
    n = 3000
    m = melted_ka(capi, ka_params, n, steps=100, seed=11)
    out = []
    for fused in (True, False):
        e = new_engine(capi)
        rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", dt=0.005, T=0.9, vel4=m["vel4"])
        steps = 250
        if fused:
            e.run(steps)
        else:
            for i in range(steps):
                if i % 100 == 0:
                    e.zero_momentum()
                e.calc_f()
                e.integrate()
            e.calc_f()
        out.append((e.get(rid, "pos", n), e.get(rid, "vel", n), e.get(rid, "force", n), e.stats(rid)))
        e.close()
    (p1, v1, f1, s1), (p2, v2, f2, s2) = out
    assert np.array_equal(p1, p2)
    assert np.array_equal(v1, v2)
    assert np.array_equal(f1, f2)
    assert s1["xi"] == s2["xi"]


VARIANTS = [  # (force_mode, build_lanes, build_smem, sm_tiles)
    (1, 8, 1, 0), (0, 8, 1, 0), (1, 1, 0, 0), (0, 1, 0, 0), (0, 2, 0, 0), (0, 4, 0, 0), (0, 8, 0, 0),
    (0, 1, 1, 0), (2, 2, 0, 0), (2, 8, 1, 0), (2, 1, 0, 0), (2, 4, 0, 0), (0, 32, 0, 0), (1, 32, 0, 0),
    (2, 32, 0, 0), (0, 32, 0, 1), (0, 2, 0, 1), (2, 32, 0, 1), (0, 0, 0, 0), (1, 0, 0, 0), (0, 0, 0, 1), (2, 0, 0, 0)]


@pytest.mark.parametrize("tp", [1, 4])
def test_kernel_variants_give_identical_lists_and_trajectories(capi, oracle, ka_params, tp):
    """Every (force index staging, list-build lanes, list-build staging) choice
    gives the oracle's list and the same trajectory bit for bit."""
    n = 6000
    m = melted_ka(capi, ka_params, n, steps=100, seed=21)
    nc, old, counts, nbl, ov = oracle_sorted_list(oracle, m["pos4"], m["box"], ka_params, 2, 0.3, 400)
    assert not ov
    res = []
    for fs, lanes, bs, smt in VARIANTS:
        e = new_engine(capi, pb=64, tp=tp)
        e.set_variant(capi.VARIANT_FORCE_MODE, fs)
        e.set_variant(capi.VARIANT_BUILD_LANES, lanes)
        e.set_variant(capi.VARIANT_BUILD_SMEM, bs)
        e.set_variant(capi.VARIANT_SM_TILES, smt)
        assert e.get_variant(capi.VARIANT_BUILD_LANES) == lanes
        rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", dt=0.005, T=0.9, vel4=m["vel4"])
        e.calc_f()
        gc, gl = e.nbl(rid, n, 400)
        for s in range(0, n, 7):
            i = old[s]
            assert gc[i] == counts[s]
            assert np.array_equal(gl[i, : gc[i]], old[nbl[s, : counts[s]]])
        f0 = e.get(rid, "force", n)
        if fs == 2:  # the window path is taken, not the streamed fallback
            st0 = e.stats(rid)
            assert st0["window_tiles"] == st0["tiles"] > 0
        e.run(200)
        res.append((f0, e.get(rid, "pos", n), e.get(rid, "vel", n), e.stats(rid)))
        e.close()
    for f0, p, v, st in res[1:]:
        assert np.array_equal(f0, res[0][0])
        assert np.array_equal(p, res[0][1])
        assert np.array_equal(v, res[0][2])
        assert st["xi"] == res[0][3]["xi"] and st["rebuilds"] == res[0][3]["rebuilds"]


def test_conditional_and_plain_graphs_agree(capi, ka_params):
    n = 3000
    m = melted_ka(capi, ka_params, n, steps=50, seed=12)
    res = []
    for cond in (1, 0):
        e = new_engine(capi)
        e.set_graph_mode(cond)
        rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", vel4=m["vel4"])
        e.run(300)
        res.append((e.get(rid, "pos", n), e.stats(rid)))
        e.close()
    assert np.array_equal(res[0][0], res[1][0])
    assert res[0][1]["rebuilds"] == res[1][1]["rebuilds"]


@pytest.mark.parametrize("persistent", [1, 2, 3])
def test_replica_in_batch_equals_alone(capi, ka_params, oracle, persistent):
    """A replica advanced in a batch -- by the step graphs with k_steps
    (persistent = 1), by the batched kernel k_batch with its in-launch
    rebuilds (persistent = 2) or by k_flow, each replica stepping on its own
    (persistent = 3) -- ends bit for bit where it ends alone."""
    from rumd_b200 import initconf as I
    sizes = [600, 2048, 777, 5000]
    temps = [0.5, 1.0, 1.5, 2.0]
    confs = [I.ka_config(s, T=t, seed=s) for s, t in zip(sizes, temps)]
    steps = 300
    batch = new_engine(capi)
    batch.set_variant(capi.VARIANT_PERSISTENT, persistent)
    ids = [batch.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", dt=0.005, T=t, vel4=c["vel4"])
           for c, t in zip(confs, temps)]
    batch.run(steps)
    for c, t, rid, s in zip(confs, temps, ids, sizes):
        alone = new_engine(capi)
        a = alone.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", dt=0.005, T=t, vel4=c["vel4"])
        alone.run(steps)
        assert np.array_equal(alone.get(a, "pos", s), batch.get(rid, "pos", s))
        assert alone.stats(a)["xi"] == batch.stats(rid)["xi"]
        assert alone.stats(a)["rebuilds"] == batch.stats(rid)["rebuilds"]
        alone.close()
    batch.close()


def test_queued_uneven_steps(capi, ka_params):
    from rumd_b200 import initconf as I
    e = new_engine(capi)
    c1, c2 = I.ka_config(1000, seed=1), I.ka_config(1500, seed=2)
    r1 = e.add(c1["pos4"], c1["box"], ka_params, 2, vel4=c1["vel4"])
    r2 = e.add(c2["pos4"], c2["box"], ka_params, 2, vel4=c2["vel4"])
    e.queue(r1, 70)
    e.queue(r2, 130)
    done = e.run_queued()
    assert done == 130
    assert e.stats(r1)["steps"] == 70 and e.stats(r2)["steps"] == 130
    e.close()


def test_list_overflow_is_repaired(capi, ka_params):
    n = 4000
    m = melted_ka(capi, ka_params, n, steps=50, seed=13)
    res = []
    for cap in (0, 40):
        e = new_engine(capi)
        rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", vel4=m["vel4"], max_nbrs=cap)
        e.run(120)
        st = e.stats(rid)
        assert st["overflow"] == 0
        res.append(e.get(rid, "pos", n))
        if cap:
            assert st["max_nbrs"] > 40
        e.close()
    assert np.array_equal(res[0], res[1])


def test_nve_energy_drift(capi, ka_params):
    """NVE (thermostat off), KA N=1000 at T~0.73, dt=0.005, 1e4 steps."""
    m = melted_ka(capi, ka_params, 1000, T=0.73, steps=2000, seed=21)
    e = new_engine(capi)
    steps = 10000
    rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", dt=0.005, thermostat=False, vel4=m["vel4"],
                energy_interval=10, energy_capacity=steps // 10, reset_interval=0)
    e.run(steps)
    log = e.energy_log(rid)
    etot = (log[:, 1] + log[:, 3]) / 1000.0
    slope = np.polyfit(log[:, 0], etot, 1)[0]
    # drift (the linear trend) over 1e4 steps, per particle
    assert abs(slope * steps) < 1e-4
    # leap-frog fluctuations at dt=0.005 stay bounded (no secular growth)
    assert np.abs(etot - etot[0]).max() < 5e-3
    e.close()


def test_thermostat_reaches_target(capi, ka_params):
    from rumd_b200 import initconf as I
    c = I.ka_config(8000, T=2.0, seed=3)
    e = new_engine(capi)
    rid = e.add(c["pos4"], c["box"], ka_params, 2, cutoff="SF", dt=0.005, T=0.8, tau=0.2, vel4=c["vel4"],
                energy_interval=10, energy_capacity=400)
    e.run(4000)
    log = e.energy_log(rid)
    T = 2 * log[-200:, 3] / (3 * 8000 - 3)
    assert abs(T.mean() - 0.8) < 0.02
    e.close()


def test_stress_tensor_trace_equals_virial(capi, ka_params):
    n = 4000
    m = melted_ka(capi, ka_params, n, steps=50, seed=31)
    e = new_engine(capi)
    rid = e.add(m["pos4"], m["box"], ka_params, 2, cutoff="SF", vel4=m["vel4"])
    e.calc_f(stress=True)
    s = e.stress(rid)
    V = float(np.prod(m["box"].astype(np.float64)))
    W = e.stats(rid)["virial"]
    # configurational stress: -tr(sigma)/3 * V == W  (Sample.cu:393-444 sign convention)
    assert abs(-(s[0] + s[1] + s[2]) / 3 * V - W) < 1e-4 * abs(W) + 1e-3
    e.close()


@pytest.mark.parametrize("cutoff,tp", [("SF", 4), ("SP", 1), ("NS", 2)])
def test_stress_tensor_against_fp64_oracle(capi, oracle, ka_params, cutoff, tp):
    """All six components of the pair stress (fij's STR branch,
    PairPotential.h:1232-1241) per particle against the FP64 oracle (rms
    relative 1e-5 over the components), and Sample::GetStress
    (Sample.cu:393-444) with and without the kinetic part: the diagonal to
    1e-5 relative, the off-diagonal (which fluctuate around zero) to 1e-5 of
    the diagonal's size.  Non-cubic box, every cut-off method.  The oracle
    sums the pairs the reference's FP32 cut-off test admits (with NS and SP
    the pair force does not vanish at rc, so one pair within a rounding
    error of rc would otherwise differ between FP32 and FP64)."""
    n = 4000
    m = melted_ka(capi, ka_params, n, steps=80, seed=33, cutoff=cutoff)
    stretch = np.array([1.2, 0.9, 1.0 / 1.08], np.float32)
    box = (m["box"] * stretch).astype(np.float32)
    pos4 = m["pos4"].copy()
    pos4[:, :3] *= stretch
    e = new_engine(capi, tp=tp)
    rid = e.add(pos4, box, ka_params, 2, cutoff=cutoff, vel4=m["vel4"])
    e.calc_f(stress=True)
    sts = e.get(rid, "stress", n).astype(np.float64)
    w = e.get(rid, "virial", n).astype(np.float64)
    g6 = np.stack([sts[:, 0], sts[:, 1], sts[:, 2], sts[:, 3], w[:, 1], w[:, 2]], 1)
    types = pos4[:, 3].view(np.int32)
    o6 = oracle.stress_f64(pos4[:, :3].astype(np.float64), types, box, 2, ka_params, capi.CUTOFF[cutoff])
    assert rms_rel(g6, o6) <= 1e-5
    vel = e.get(rid, "vel", n)
    for kin in (False, True):
        s = e.stress(rid, include_kinetic=kin)
        ref = oracle.sample_stress(o6, vel, box, include_kinetic=kin)
        scale = abs(ref[:3]).mean()
        assert np.all(np.abs(s[:3] - ref[:3]) <= 1e-5 * np.abs(ref[:3])), (kin, s, ref)
        assert np.all(np.abs(s[3:] - ref[3:]) <= 1e-5 * scale), (kin, s, ref)
    e.close()
