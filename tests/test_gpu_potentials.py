"""The other pair functions on the device: Pot_LJ_12_6_smooth_2_4 and
Pot_IPL_n (PairPotential.h:210-256, 603-637) through the C ABI and through the
RUMD classes.

Tolerances are those of the LJ parity tests: forces rms relative 1e-5 against
the FP64 oracle pair sum of the same pair function, energies 1e-5 relative,
NVE drift (the linear trend of E/N over 1e4 steps) below 1e-4."""
import numpy as np
import pytest

from test_gpu_parity import melted_ka, rms_rel
from test_gpu_rumd_api import golden_sample

pytestmark = pytest.mark.gpu

KA = {(0, 0): (1.0, 1.0, 2.5), (0, 1): (0.8, 1.5, 2.5), (1, 1): (0.88, 0.5, 2.5)}
CASES = [("LJ_12_6_smooth_2_4", None), ("IPL_n", 12.0), ("IPL_n", 18.0), ("IPL_n", 9.5)]


@pytest.fixture(scope="module")
def capi():
    from rumd_b200 import build, capi
    build.build_lib()
    return capi


@pytest.fixture(scope="module")
def rumd():
    from rumd_b200 import build
    build.build()
    from rumd_b200 import rumd
    return rumd


@pytest.fixture(scope="module")
def melt(capi, oracle):
    return melted_ka(capi, oracle.lj_params(2, oracle.ka_table()), 4000, steps=200, seed=5)


def table(oracle, potential, n):
    return oracle.smooth_params(2, KA) if potential == "LJ_12_6_smooth_2_4" else oracle.ipl_n_params(2, n, KA)


@pytest.mark.parametrize("tp", [1, 4])
@pytest.mark.parametrize("cutoff", ["SF", "SP", "NS"])
@pytest.mark.parametrize("potential,n", CASES, ids=[f"{p}-{n}" for p, n in CASES])
def test_forces_energy_virial_against_fp64(capi, oracle, melt, potential, n, cutoff, tp):
    params = table(oracle, potential, n)
    N = len(melt["pos4"])
    e = capi.Engine(device=0, pb=64, tp=tp)
    rid = e.add(melt["pos4"], melt["box"], params, 2, cutoff=cutoff, potential=potential)
    e.calc_f()
    f = e.get(rid, "force", N)
    st = e.stats(rid)
    types = melt["pos4"][:, 3].view(np.int32)
    ref, u, w = oracle.forces_f64(melt["pos4"][:, :3].astype(np.float64), types, melt["box"], 2, params,
                                  capi.CUTOFF[cutoff], potential)
    assert rms_rel(f[:, :3].astype(np.float64), ref) <= 1e-5
    assert abs(st["pe"] - u.sum()) <= 1e-5 * abs(u.sum())
    assert abs(st["virial"] - w.sum() / 6) <= 1e-5 * abs(w.sum() / 6) + 1e-3
    e.close()


@pytest.mark.parametrize("potential,n", CASES[:2], ids=[f"{p}-{n}" for p, n in CASES[:2]])
def test_force_modes_bit_identical(capi, oracle, melt, potential, n):
    """The streamed, staged and window force paths give the same bits for
    every pair function, over a short trajectory with list rebuilds."""
    params = table(oracle, potential, n)
    N = len(melt["pos4"])
    res = []
    for mode in (0, 1, 2):
        e = capi.Engine(device=0, pb=64, tp=2)
        e.set_variant(capi.VARIANT_FORCE_MODE, mode)
        rid = e.add(melt["pos4"], melt["box"], params, 2, cutoff="SF", dt=0.004, T=1.0, vel4=melt["vel4"],
                    potential=potential)
        e.run(150)
        res.append((e.get(rid, "pos", N), e.get(rid, "force", N), e.stats(rid)))
        e.close()
    for p, f, st in res[1:]:
        assert np.array_equal(p, res[0][0])
        assert np.array_equal(f, res[0][1])
        assert st["rebuilds"] == res[0][2]["rebuilds"] > 1


def test_smooth_nve_energy_drift(capi, oracle):
    """NVE with the smoothed LJ potential (ShiftedPotential: energy and force
    both continuous at rc), KA N=1000, dt=0.005, 1e4 steps."""
    from rumd_b200 import initconf as I
    params = oracle.smooth_params(2, KA)
    c = I.ka_config(1000, T=0.73, seed=21)
    e = capi.Engine(device=0, pb=64, tp=4)
    rid = e.add(c["pos4"], c["box"], params, 2, cutoff="SP", dt=0.004, T=2.0, vel4=c["vel4"],
                potential="LJ_12_6_smooth_2_4")
    e.run(1000)  # melt
    e.set_integrator(rid, 0.005, 0.73, 0.2)
    e.run(1000)  # equilibrate at T = 0.73
    pos4, vel4 = e.get(rid, "pos", 1000), e.get(rid, "vel", 1000)
    e.close()
    steps = 10000
    e = capi.Engine(device=0, pb=64, tp=4)
    rid = e.add(pos4, c["box"], params, 2, cutoff="SP", dt=0.005, thermostat=False, vel4=vel4,
                energy_interval=10, energy_capacity=steps // 10, reset_interval=0, potential="LJ_12_6_smooth_2_4")
    e.run(steps)
    log = e.energy_log(rid)
    etot = (log[:, 1] + log[:, 3]) / 1000.0
    slope = np.polyfit(log[:, 0], etot, 1)[0]
    assert abs(slope * steps) < 1e-4
    assert np.abs(etot - etot[0]).max() < 5e-3
    e.close()


def test_set_potential_switches_pair_function(capi, oracle, melt):
    """One replica changes pair function in place (Sample::SetPotential with
    another class): the forces follow, and unknown kinds are refused."""
    N = len(melt["pos4"])
    types = melt["pos4"][:, 3].view(np.int32)
    lj = oracle.lj_params(2, oracle.ka_table())
    e = capi.Engine(device=0, pb=64, tp=2)
    rid = e.add(melt["pos4"], melt["box"], lj, 2, cutoff="SF")
    for potential, n in CASES + [("LJ_12_6", None)]:
        params = lj if potential == "LJ_12_6" else table(oracle, potential, n)
        e.set_potential(rid, 2, params, "SF", 0.3, potential)
        e.calc_f()
        ref, u, w = oracle.forces_f64(melt["pos4"][:, :3].astype(np.float64), types, melt["box"], 2, params, 2,
                                      potential)
        assert rms_rel(e.get(rid, "force", N)[:, :3].astype(np.float64), ref) <= 1e-5, potential
    with pytest.raises(ValueError):
        e.set_potential(rid, 2, lj, "SF", 0.3, 3)
    bad = oracle.ipl_n_params(2, 12.0, KA)
    bad[1] = 0.0  # 1/sigma^2 of (0, 0)
    with pytest.raises(ValueError):
        e.set_potential(rid, 2, bad, "SF", 0.3, "IPL_n")
    with pytest.raises(ValueError):
        e.add(melt["pos4"], melt["box"], lj, 2, potential=7)
    e.close()


@pytest.mark.parametrize("cls", ["smooth", "ipl"])
def test_rumd_classes_on_reference_configuration(rumd, oracle, tmp_path, cls):
    s, g = golden_sample(rumd, tmp_path)
    if cls == "smooth":
        pot = rumd.Pot_LJ_12_6_smooth_2_4(cutoff_method=rumd.ShiftedPotential)
        potential, params = "LJ_12_6_smooth_2_4", oracle.smooth_params(2, KA)
    else:
        pot = rumd.Pot_IPL_n(n=12.0, cutoff_method=rumd.ShiftedForce)
        potential, params = "IPL_n", oracle.ipl_n_params(2, 12.0, KA)
    for (i, j), (sig, eps, rc) in KA.items():
        pot.SetParams(i, j, sig, eps, rc)
    s.SetPotential(pot)
    s.CalcF()
    f = np.asarray(s.GetForces(), np.float64)
    pos = np.asarray(s.GetPositions(), np.float64)
    ref, u, w = oracle.forces_f64(pos, np.asarray(s.GetTypes(), np.int32), np.asarray(s.GetBoxLengths()), 2, params,
                                  pot.GetCutoffMethod(), potential)
    assert rms_rel(f, ref) <= 1e-5
    assert abs(s.GetPotentialEnergy() - u.sum()) <= 1e-5 * abs(u.sum())


# A second potential with its own, shorter cut-off (2.0 sigma): the list is
# built with the larger one, and each pair function applies its own.
SMOOTH2 = {(0, 0): (1.0, 0.3, 2.0), (0, 1): (0.8, 0.45, 2.0), (1, 1): (0.88, 0.15, 2.0)}


@pytest.mark.parametrize("tp", [1, 4])
@pytest.mark.parametrize("force_mode", [0, 1, 2])
def test_second_potential_adds_to_the_first(capi, oracle, melt, force_mode, tp):
    """Sample::CalcF's potential loop (Sample.cu:335-336): LJ 12-6 (SF,
    rc 2.5 sigma) plus a smoothed LJ (SP, rc 2.0 sigma) on one sample against
    the sum of the FP64 oracle's two pair sums, in every force mode: forces
    rms relative 1e-5, energy and virial 1e-5 relative, the six pair-stress
    components rms relative 1e-5."""
    N = len(melt["pos4"])
    lj = oracle.lj_params(2, oracle.ka_table())
    sm = oracle.smooth_params(2, SMOOTH2)
    e = capi.Engine(device=0, pb=64, tp=tp)
    e.set_variant(capi.VARIANT_FORCE_MODE, force_mode)
    rid = e.add(melt["pos4"], melt["box"], lj, 2, cutoff="SF")
    e.add_potential(rid, 2, sm, "SP", "LJ_12_6_smooth_2_4")
    with pytest.raises(ValueError):
        e.add_potential(rid, 2, sm, "SP", "LJ_12_6_smooth_2_4")  # two at most
    e.calc_f(stress=True)
    f = e.get(rid, "force", N).astype(np.float64)
    st = e.stats(rid)
    sts = e.get(rid, "stress", N).astype(np.float64)
    w = e.get(rid, "virial", N).astype(np.float64)
    g6 = np.stack([sts[:, 0], sts[:, 1], sts[:, 2], sts[:, 3], w[:, 1], w[:, 2]], 1)
    e.close()
    pos = melt["pos4"][:, :3].astype(np.float64)
    types = melt["pos4"][:, 3].view(np.int32)
    f1, u1, w1 = oracle.forces_f64(pos, types, melt["box"], 2, lj, capi.CUTOFF["SF"], "LJ_12_6")
    f2, u2, w2 = oracle.forces_f64(pos, types, melt["box"], 2, sm, capi.CUTOFF["SP"], "LJ_12_6_smooth_2_4")
    assert rms_rel(f2, f1) > 0.01  # the second potential matters
    assert rms_rel(f[:, :3], f1 + f2) <= 1e-5
    assert np.abs(f[:, 3] - (u1 + u2)).max() < 1e-4
    u = u1.sum() + u2.sum()
    assert abs(st["pe"] - u) <= 1e-5 * abs(u)
    assert abs(st["virial"] - (w1 + w2).sum() / 6) <= 1e-5 * abs((w1 + w2).sum() / 6) + 1e-3
    o6 = (oracle.stress_f64(pos, types, melt["box"], 2, lj, capi.CUTOFF["SF"], "LJ_12_6")
          + oracle.stress_f64(pos, types, melt["box"], 2, sm, capi.CUTOFF["SP"], "LJ_12_6_smooth_2_4"))
    assert rms_rel(g6, o6) <= 1e-5


def test_two_half_potentials_run_as_one(capi, oracle, melt):
    """LJ 12-6 with epsilon/2, added twice, is LJ 12-6 with epsilon bit for
    bit: halving epsilon halves every coefficient and every pair term exactly
    (a power of two), both passes sum the same list in the same order, and the
    second's sums are added to the first's.  So a 300-step NVT run with the
    two potentials (per-step graphs) must give the one-potential run's
    positions, energies and thermostat state exactly."""
    N = len(melt["pos4"])
    full = oracle.lj_params(2, oracle.ka_table())
    half = oracle.lj_params(2, {k: (s, eps / 2, rc) for k, (s, eps, rc) in KA.items()})
    assert np.array_equal(half[1::12] * 2, full[1::12])  # A12
    out = []
    for two in (False, True):
        e = capi.Engine(device=0, pb=64, tp=4)
        rid = e.add(melt["pos4"], melt["box"], half if two else full, 2, cutoff="SF", T=0.8, vel4=melt["vel4"])
        if two:
            e.add_potential(rid, 2, half, "SF")
        e.run(300)
        st = e.stats(rid)
        kind = e.get_variant(capi.VARIANT_PERSISTENT_ACTIVE)
        out.append((e.get(rid, "pos", N), st, kind))
        e.close()
    (p1, s1, k1), (p2, s2, k2) = out
    assert k2 == 0  # the replica with two potentials ran on the per-step graphs
    assert s1["rebuilds"] == s2["rebuilds"] > 1
    assert s1["pe"] == s2["pe"] and s1["ke"] == s2["ke"] and s1["xi"] == s2["xi"]
    assert np.array_equal(p1, p2)


def test_rumd_classes_add_potential(rumd, oracle, tmp_path):
    """Sample::AddPotential through the RUMD classes: both potentials act, a
    third is refused, SetPotential goes back to one."""
    s, g = golden_sample(rumd, tmp_path)
    lj = rumd.Pot_LJ_12_6(cutoff_method=rumd.ShiftedForce)
    sm = rumd.Pot_LJ_12_6_smooth_2_4(cutoff_method=rumd.ShiftedPotential)
    for (i, j), (sig, eps, rc) in KA.items():
        lj.SetParams(i, j, sig, eps, rc)
    for (i, j), (sig, eps, rc) in SMOOTH2.items():
        sm.SetParams(i, j, sig, eps, rc)
    s.SetPotential(lj)
    s.AddPotential(sm)
    assert len(s.GetPotentials()) == 2
    s.CalcF()
    pos = np.asarray(s.GetPositions(), np.float64)
    types = np.asarray(s.GetTypes(), np.int32)
    box = np.asarray(s.GetBoxLengths())
    f1, u1, _ = oracle.forces_f64(pos, types, box, 2, oracle.lj_params(2, KA), 2, "LJ_12_6")
    f2, u2, _ = oracle.forces_f64(pos, types, box, 2, oracle.smooth_params(2, SMOOTH2), 1, "LJ_12_6_smooth_2_4")
    assert rms_rel(np.asarray(s.GetForces(), np.float64), f1 + f2) <= 1e-5
    assert abs(s.GetPotentialEnergy() - (u1.sum() + u2.sum())) <= 1e-5 * abs(u1.sum() + u2.sum())
    third = rumd.Pot_LJ_12_6(cutoff_method=rumd.ShiftedForce)
    with pytest.raises(Exception):
        s.AddPotential(third)
    s.SetPotential(lj)
    assert len(s.GetPotentials()) == 1
    s.CalcF()
    assert rms_rel(np.asarray(s.GetForces(), np.float64), f1) <= 1e-5
