"""The CPU oracle against RUMD's own golden vectors and internal invariants.

The golden vectors are the forces, per-particle energies and virials stored
by RUMD in Conf/KobAndersen/*.xyz.gz (SP cut-off at 2.5 sigma_ij, KA
parameters); see tests/golden/make_golden.py.  They are printed with 6 to 9
significant digits, which sets the tolerances below.
"""
import numpy as np
import pytest

from conftest import golden_files, load_golden

FILES = golden_files()


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("path", FILES, ids=[p.split("/")[-1] for p in FILES])
def test_oracle_reproduces_reference_forces(oracle, path):
    g = load_golden(path)
    params = oracle.lj_params(2, oracle.ka_table())
    pos = g["pos"].astype(np.float32).astype(np.float64)
    f, u, w = oracle.forces_f64(pos, g["type"], g["L"], 2, params, oracle.SP)
    # stored with 6 decimals (older files) or 9 (newer): rms-rel at the print limit
    assert rms_rel(f, g["force"]) < 2e-5
    assert np.abs(u - g["pe"]).max() < 2e-4
    if "vir" in g:
        # vir column = w.w / 2 (ConfigurationWriterReader.cu:173)
        assert np.abs(w / 2 - g["vir"]).max() < 2e-3
        assert rms_rel(w / 2, g["vir"]) < 1e-5


def test_param_table_matches_reference_mapping(oracle):
    p = oracle.lj_params(2, oracle.ka_table()).reshape(2, 2, 12)
    # Pot_LJ_12_6::SetParams: A12 = 4 eps sigma^12, A6 = -4 eps sigma^6, Rcut*sigma
    assert p[0, 1, 0] == np.float32(2.5) * np.float32(0.8)
    assert p[0, 1, 1] == np.float32(4 * np.float64(np.float32(1.5)) * np.float64(np.float32(0.8)) ** 12)
    assert np.array_equal(p[0, 1], p[1, 0])
    # shift constants: u(rc) and s(rc)*rc with the FP32 ComputeInteraction
    rc = np.float32(2.5)
    inv2 = np.float32(1) / (rc * rc)
    inv6 = inv2 * inv2 * inv2
    assert p[0, 0, 11] == inv6 * (np.float32(4) * inv6 + np.float32(-4))


def test_numpy_param_tables_equal_oracle(oracle):
    from rumd_b200 import initconf as I
    a = oracle.lj_params(2, oracle.ka_table())
    b = I.lj_params(2, I.KA)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("path", FILES[:6], ids=[p.split("/")[-1] for p in FILES[:6]])
@pytest.mark.parametrize("cutoff", [0, 1, 2])
def test_fp32_restatement_within_1e5_of_fp64(oracle, path, cutoff):
    g = load_golden(path)
    params = oracle.lj_params(2, oracle.ka_table())
    pos4 = np.zeros((len(g["pos"]), 4), np.float32)
    pos4[:, :3] = g["pos"]
    pos4[:, 3] = g["type"].view(np.float32)
    counts, nbl, ov = oracle.nbl_n2(pos4, g["L"], 2, params, 0.3, 400)
    assert not ov
    f4, w = oracle.forces_f32(pos4, g["L"], 2, params, cutoff, counts, nbl)
    f, u, w64 = oracle.forces_f64(pos4[:, :3].astype(np.float64), g["type"], g["L"], 2, params, cutoff)
    assert rms_rel(f4[:, :3].astype(np.float64), f) < 1e-5
    assert abs(f4[:, 3].astype(np.float64).sum() - u.sum()) / abs(u.sum()) < 1e-5


def _pos4(g):
    pos4 = np.zeros((len(g["pos"]), 4), np.float32)
    pos4[:, :3] = g["pos"]
    pos4[:, 3] = g["type"].view(np.float32)
    return pos4


@pytest.mark.parametrize("path", [p for p in FILES if "N2000" in p or "N4096" in p or "N1372" in p])
def test_cell_list_sets_equal_all_pairs(oracle, path):
    g = load_golden(path)
    params = oracle.lj_params(2, oracle.ka_table())
    pos4 = _pos4(g)
    L = g["L"].astype(np.float32)
    nc = oracle.cell_grid(L, oracle.max_cutoff(params, 2), 0.3)
    keys = oracle.cell_keys(pos4, L, nc)
    old = oracle.stable_sort_perm(keys, int(np.prod(nc)))
    # stable sort permutation == numpy stable argsort
    assert np.array_equal(old, np.argsort(keys, kind="stable").astype(np.uint32))
    counts, nbl, ov = oracle.nbl_cells(pos4[old], L, nc, 2, params, 0.3, 300)
    c2, n2, ov2 = oracle.nbl_n2(pos4, L, 2, params, 0.3, 300)
    assert not ov and not ov2
    for s in range(len(pos4)):
        i = old[s]
        a = set(old[nbl[s, : counts[s]]].tolist())
        b = set(n2[i, : c2[i]].tolist())
        assert a == b


def test_sorted_scan_order(oracle):
    """Entries of the sorted cell scan appear in (dz, dy, dx, ascending j) order."""
    from rumd_b200 import initconf as I
    g = load_golden(FILES[-1])
    params = oracle.lj_params(2, oracle.ka_table())
    pos4 = _pos4(g)
    L = g["L"].astype(np.float32)
    nc = oracle.cell_grid(L, oracle.max_cutoff(params, 2), 0.3)
    keys = oracle.cell_keys(pos4, L, nc)
    old = oracle.stable_sort_perm(keys, int(np.prod(nc)))
    ps = pos4[old]
    ks = keys[old]
    counts, nbl, _ = oracle.nbl_cells(ps, L, nc, 2, params, 0.3, 300)
    for s in range(0, len(ps), 97):
        cx, cy, cz = ks[s] % nc[0], (ks[s] // nc[0]) % nc[1], ks[s] // (nc[0] * nc[1])
        order = []
        for j in nbl[s, : counts[s]]:
            k = ks[j]
            jx, jy, jz = k % nc[0], (k // nc[0]) % nc[1], k // (nc[0] * nc[1])
            d = [((jz - cz + 2) % nc[2]), ((jy - cy + 2) % nc[1]), ((jx - cx + 2) % nc[0]), j]
            order.append(tuple(int(x) for x in d))
        assert order == sorted(order)


def test_max_nbrs_estimate_rule(oracle):
    assert oracle.max_nbrs_estimate(1000, 2.5, 0.3, 9.41 ** 3) == 1000
    est = oracle.max_nbrs_estimate(65536, 2.5, 0.3, 65536 / 1.2)
    assert est == int(1.5 * 4 / 3 * np.pi * np.float32(2.8) ** 3 * 65536 / (65536 / 1.2))


def test_md_run_fp32_vs_fp64_short_horizon(oracle):
    from rumd_b200 import initconf as I
    g = load_golden([p for p in FILES if "KA_N1000_T1.0" in p][0])
    params = oracle.lj_params(2, oracle.ka_table())
    pos4 = _pos4(g)
    vel4 = np.zeros_like(pos4)
    vel4[:, :3] = g["vel"]
    vel4[:, 3] = 1.0
    im3 = np.zeros((len(pos4), 3), np.int32)
    kw = dict(L=g["L"], ntypes=2, params=params, cutoff=oracle.SF, skin=0.3, dt=0.005, T=1.0, tau=0.2, nsteps=50)
    a = oracle.md_run(pos4, vel4, im3, precision="f32", **kw)
    b = oracle.md_run(pos4, vel4, im3, precision="f64", **kw)
    L = g["L"]
    d = a["pos4"][:, :3].astype(np.float64) - b["pos4"][:, :3]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-3
    assert np.allclose(a["energies"][:, 0], b["energies"][:, 0], rtol=1e-4)
    assert a["rebuilds"] >= 1
