"""The other pair functions on the host: Pot_LJ_12_6_smooth_2_4 and Pot_IPL_n.

The reference ships no fixtures for these classes, so the oracle's
restatement is pinned by the mathematics instead: the FP64 force is minus the
gradient of the FP64 energy (central differences), the IPL force has its
closed form, the smoothed LJ force and its slope vanish at the cut-off, and
the parameter rows (with the shift constants p10, p11 of CopyParamsToGPU)
agree bit for bit between the oracle, the Python table builders and the C++
classes."""
import numpy as np
import pytest

from test_rumd_api_cpu import rumd  # noqa: F401  (module fixture)

KA = {(0, 0): (1.0, 1.0, 2.5), (0, 1): (0.8, 1.5, 2.5), (1, 1): (0.88, 0.5, 2.5)}
EXPONENTS = [6.0, 9.5, 12.0, 18.0, 36.0]


def pair_energy_force(oracle, params, r, potential, cutoff, t=(0, 0), ntypes=2):
    pos = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0]])
    f, u, w = oracle.forces_f64(pos, np.array(t, np.int32), [50.0, 50.0, 50.0], ntypes, params, cutoff,
                                potential)
    return u.sum(), f[1, 0]


def test_smooth_table_builders_agree(oracle):
    from rumd_b200 import initconf
    a = initconf.smooth_params(2, KA)
    b = oracle.smooth_params(2, KA)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    row = b.reshape(4, 12)[0]
    assert row[0] == np.float32(2.5) and row[1] == 1.0 and row[2] == 4.0
    # the force at rc is zero up to float rounding of c2, c4
    assert abs(row[10]) < 1e-7


@pytest.mark.parametrize("n", EXPONENTS)
def test_ipl_n_table_builders_agree(oracle, n):
    from rumd_b200 import initconf
    a = initconf.ipl_n_params(2, n, KA)
    b = oracle.ipl_n_params(2, n, KA)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    row = b.reshape(4, 12)[1]  # (0, 1): sigma 0.8, eps 1.5
    rc = np.float32(2.5) * np.float32(0.8)
    assert row[0] == rc and row[3] == np.float32(n)
    assert np.isclose(row[11], 1.5 * 2.5 ** -n, rtol=1e-5)          # u(rc)
    assert np.isclose(row[10], n * 1.5 * 2.5 ** -n / rc, rtol=1e-5)  # s(rc) rc


def test_cpp_classes_store_the_same_rows(rumd, oracle):  # noqa: F811
    pot = rumd.Pot_LJ_12_6_smooth_2_4(cutoff_method=rumd.ShiftedPotential)
    for (i, j), (s, e, rc) in KA.items():
        pot.SetParams(i, j, s, e, rc)
    assert np.array_equal(np.array(pot.ParamTable(2), np.float32).view(np.uint32),
                          oracle.smooth_params(2, KA).view(np.uint32))
    assert pot.GetID_String() == "potLJ_12_6_smooth_2_4"
    ipl = rumd.Pot_IPL_n(n=18.0, cutoff_method=rumd.ShiftedForce)
    for (i, j), (s, e, rc) in KA.items():
        ipl.SetParams(i, j, s, e, rc)
    assert np.array_equal(np.array(ipl.ParamTable(2), np.float32).view(np.uint32),
                          oracle.ipl_n_params(2, 18.0, KA).view(np.uint32))
    assert ipl.GetExponent() == 18.0
    assert ipl.GetID_String() == "potIPL_18"
    assert ipl.GetMaxCutoff() == np.float32(2.5)


@pytest.mark.parametrize("potential", ["LJ_12_6_smooth_2_4", "IPL_n"])
@pytest.mark.parametrize("cutoff", [0, 1, 2])
def test_fp64_force_is_minus_energy_gradient(oracle, potential, cutoff):
    params = oracle.smooth_params(2, KA) if potential != "IPL_n" else oracle.ipl_n_params(2, 12.0, KA)
    h = 1e-5
    for t in [(0, 0), (0, 1), (1, 1)]:
        for r in [0.85, 1.0, 1.3, 1.9]:
            up, _ = pair_energy_force(oracle, params, r + h, potential, cutoff, t)
            um, _ = pair_energy_force(oracle, params, r - h, potential, cutoff, t)
            _, f = pair_energy_force(oracle, params, r, potential, cutoff, t)
            # f is the force on the particle at +r along x: F = -dU/dr
            assert f == pytest.approx(-(up - um) / (2 * h), rel=1e-6, abs=1e-9)


@pytest.mark.parametrize("n", EXPONENTS)
def test_ipl_n_closed_form(oracle, n):
    params = oracle.ipl_n_params(2, n, KA)
    # the row holds 1/sigma^2 in float: sigma is what that value says
    sig = 1.0 / np.sqrt(np.float64(np.float32(1.0) / (np.float32(0.8) * np.float32(0.8))))
    eps = np.float64(np.float32(1.5))
    for r in [0.7, 1.0, 1.5]:
        u, f = pair_energy_force(oracle, params, r, "IPL_n", 0, (0, 1))
        assert u == pytest.approx(eps * (sig / r) ** n, rel=1e-12)
        assert f == pytest.approx(n * eps * (sig / r) ** n / r, rel=1e-12)


def test_smooth_force_and_slope_vanish_at_cutoff(oracle):
    params = oracle.smooth_params(2, KA)
    for t, (sig, eps, rc) in zip([(0, 0), (0, 1), (1, 1)], KA.values()):
        rcut = float(np.float32(rc) * np.float32(sig))
        _, f0 = pair_energy_force(oracle, params, rcut * (1 - 1e-7), "LJ_12_6_smooth_2_4", 0, t)
        _, f1 = pair_energy_force(oracle, params, rcut * (1 - 1e-3), "LJ_12_6_smooth_2_4", 0, t)
        _, fcore = pair_energy_force(oracle, params, sig * 1.0, "LJ_12_6_smooth_2_4", 0, t)
        assert abs(f0) < 1e-6 * abs(fcore)
        # zero slope too: the force grows quadratically away from rc
        assert abs(f1) < 1e-4 * abs(fcore)
        # with ShiftedPotential the energy is continuous at rc
        u_sp, _ = pair_energy_force(oracle, params, rcut * (1 - 1e-7), "LJ_12_6_smooth_2_4", 1, t)
        assert abs(u_sp) < 1e-9
