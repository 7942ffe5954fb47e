"""Edge cases on the device: the smallest systems, pairs across the periodic
boundary, tiles that are mostly empty, and rejected inputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from rumd_b200 import build, capi
    build.build_lib()
    return capi


def pos4_of(xyz, types):
    p = np.zeros((len(xyz), 4), np.float32)
    p[:, :3] = xyz
    p[:, 3] = np.asarray(types, np.int32).view(np.float32)
    return p


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("cutoff", ["SF", "SP", "NS"])
@pytest.mark.parametrize("xyz", [
    [[0.0, 0.0, 0.0], [1.2, 0.0, 0.0]],          # plain pair
    [[-4.5, 0.3, -0.2], [4.7, 0.1, 0.4]],        # pair across the x face (0.8 apart)
    [[4.9, -4.8, 4.7], [-4.6, 4.9, -4.9]],       # across three faces
])
def test_two_particles_against_fp64(capi, oracle, cutoff, xyz):
    params = oracle.lj_params(1, oracle.lj_table())
    box = np.array([10.0, 10.0, 10.0], np.float32)
    pos = pos4_of(xyz, [0, 0])
    e = capi.Engine(device=0, pb=32, tp=1)
    rid = e.add(pos, box, params, 1, cutoff=cutoff)
    e.calc_f()
    f = e.get(rid, "force", 2)
    ref, u, w = oracle.forces_f64(pos[:, :3].astype(np.float64), np.zeros(2, np.int32), box, 1, params,
                                  capi.CUTOFF[cutoff])
    assert np.abs(ref).max() > 0  # the pair interacts
    # the force tolerance (1e-5): a pair 0.7 apart across three faces loses
    # ~1e-6 of its separation to the FP32 subtraction of coordinates near
    # +-L/2, which the r^-13 wall amplifies about 13-fold
    assert rms_rel(f[:, :3].astype(np.float64), ref) < 1e-5
    assert np.allclose(f[0, :3], -f[1, :3], rtol=1e-6, atol=1e-7)  # Newton's third law
    assert abs(e.stats(rid)["pe"] - u.sum()) <= 1e-5 * max(1.0, abs(u.sum()))
    e.close()


@pytest.mark.parametrize("n,tp", [(3, 8), (5, 8), (33, 4), (65, 2)])
def test_tiny_and_ragged_systems(capi, oracle, n, tp):
    """Systems smaller than a tile or a warp, in a small box (fewer than 7
    cells a side: every axis needs the minimum image)."""
    rng = np.random.default_rng(n)
    params = oracle.lj_params(2, oracle.ka_table())
    L = float((n / 0.6) ** (1.0 / 3.0)) + 5.0
    box = np.array([L, L, L], np.float32)
    # random positions at least 0.9 apart
    xyz = []
    while len(xyz) < n:
        c = rng.uniform(-L / 2, L / 2, 3)
        if all(np.linalg.norm((c - q) - L * np.rint((c - q) / L)) > 0.9 for q in xyz):
            xyz.append(c)
    types = rng.integers(0, 2, n)
    pos = pos4_of(np.array(xyz), types)
    e = capi.Engine(device=0, pb=32, tp=tp)
    rid = e.add(pos, box, params, 2, cutoff="SF")
    e.calc_f()
    f = e.get(rid, "force", n)
    ref, u, w = oracle.forces_f64(pos[:, :3].astype(np.float64), types.astype(np.int32), box, 2, params, 2)
    if np.abs(ref).sum() > 0:
        assert rms_rel(f[:, :3].astype(np.float64), ref) < 1e-5
    e.run(50)  # the step loop runs on such systems too
    assert e.stats(rid)["steps"] == 50
    assert np.isfinite(e.get(rid, "pos", n)).all()
    e.close()


def test_rejected_inputs(capi, oracle):
    params = oracle.lj_params(1, oracle.lj_table())
    e = capi.Engine(device=0)
    with pytest.raises(ValueError):
        e.add(pos4_of([[0.0, 0.0, 0.0]], [0]), [10.0, 10.0, 10.0], params, 1)  # one particle
    with pytest.raises(ValueError):
        e.add(pos4_of([[0, 0, 0], [1, 0, 0]], [0, 0]), [10.0, -1.0, 10.0], params, 1)  # bad box
    rid = e.add(pos4_of([[0, 0, 0], [1.1, 0, 0]], [0, 0]), [10.0, 10.0, 10.0], params, 1)
    e.remove(rid)
    with pytest.raises(Exception):
        e.stats(rid)  # removed replica
    e.close()


@pytest.mark.parametrize("req,eff", [((16, 4), (32, 4)), ((48, 1), (64, 1)), ((96, 3), (96, 2)),
                                     ((192, 8), (192, 2)), ((64, 64), (64, 8)), ((128, 16), (128, 4))])
def test_rumd_launch_shapes_are_mapped(capi, oracle, req, eff):
    """RUMD's autotuner shapes (pb 16..192, tp up to 64; Autotune.py:156-158)
    run: pb becomes whole warps and tp one of 1, 2, 4, 8 with pb*tp <= 512,
    and the forces meet the FP64 tolerance."""
    from rumd_b200 import initconf as I
    c = I.ka_config(2000, T=1.0, seed=9)
    params = oracle.lj_params(2, oracle.ka_table())
    e = capi.Engine(device=0, pb=req[0], tp=req[1])
    assert e.launch() == eff
    rid = e.add(c["pos4"], c["box"], params, 2, cutoff="SF")
    e.calc_f()
    f = e.get(rid, "force", 2000)
    e.set_launch(64, 4)
    e.set_launch(*req)
    assert e.launch() == eff
    e.close()
    ref, _, _ = oracle.forces_f64(c["pos4"][:, :3].astype(np.float64), c["types"], c["box"], 2, params, 2)
    assert rms_rel(f[:, :3].astype(np.float64), ref) < 1e-5
