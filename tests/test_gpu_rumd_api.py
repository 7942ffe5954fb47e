"""The RUMD class surface on the GPU: Sample / Pot_LJ_12_6 / IntegratorNVT /
Simulation used the way RUMD scripts use them."""
import numpy as np
import pytest

from conftest import golden_files, load_golden
from test_rumd_api_cpu import ka_potential, write_xyz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rumd():
    from rumd_b200 import build
    build.build()
    from rumd_b200 import rumd
    return rumd


def golden_sample(rumd, tmp_path, name="N1000_T0.5"):
    g = load_golden([p for p in golden_files() if name in p][0])
    path = tmp_path / "start.xyz.gz"
    write_xyz(path, g)
    s = rumd.Sample(0, 0)
    s.ReadConf(str(path))
    return s, g


def test_calcf_reproduces_reference_golden_forces(rumd, tmp_path):
    s, g = golden_sample(rumd, tmp_path)
    pot = ka_potential(rumd, rumd.ShiftedPotential)
    s.SetPotential(pot)
    s.CalcF()
    f = s.GetForces().astype(np.float64)
    err = np.sqrt(((f - g["force"]) ** 2).sum() / (g["force"] ** 2).sum())
    assert err < 2e-5
    assert abs(s.GetPotentialEnergy() - g["pe"].sum()) < 1e-3
    assert abs(pot.GetPotentialEnergy() - g["pe"].sum()) < 1e-3
    assert np.abs(np.array(s.GetPotentialEnergies()) - g["pe"]).max() < 2e-4
    assert pot.GetActualMaxNumNbrs() > 50


def test_simulation_run_matches_stepwise_and_records_energies(rumd, tmp_path):
    results = []
    for mode in ("run", "stepwise"):
        s, g = golden_sample(rumd, tmp_path, "KA_N1000_T1.0")
        sim = rumd.Simulation(sample=s)
        pot = ka_potential(rumd, rumd.ShiftedForce)
        pot.SetNbListSkin(0.3)
        sim.SetPotential(pot)
        itg = rumd.IntegratorNVT(timeStep=0.005, targetTemperature=1.0, thermostatRelaxationTime=0.2)
        sim.SetIntegrator(itg)
        if mode == "run":
            sim.Run(600)
            E = sim.GetEnergies()
            assert E.shape == (3, 8)
            assert np.array_equal(E[:, 0], [0, 256, 512])
            assert np.all(np.abs(E[:, 4] - 1.0) < 0.3)
            assert sim.timing and sim.timing[-1][0] == 600
        else:
            sim.RunStepwise(600)
        results.append((s.GetPositions(), s.GetVelocities(), itg.GetThermostatState(), s.GetPotentialEnergy()))
    (p1, v1, x1, e1), (p2, v2, x2, e2) = results
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    assert x1 == x2 and e1 == e2


def test_kinetic_energy_and_thermostat_api(rumd, tmp_path):
    s, g = golden_sample(rumd, tmp_path, "KA_N1000_T1.0")
    pot = ka_potential(rumd, rumd.ShiftedForce)
    s.SetPotential(pot)
    itg = rumd.IntegratorNVT(timeStep=0.005, targetTemperature=1.0, thermostatRelaxationTime=0.2)
    s.SetIntegrator(itg)
    itg.SetThermostatState(0.25)
    assert itg.GetThermostatState() == 0.25
    s.CalcF()
    ke = itg.GetKineticEnergy()
    v = g["vel"]
    assert abs(ke - 0.5 * (v ** 2).sum()) / ke < 0.05
    s.Run(100)
    assert itg.GetThermostatState() != 0.25
    itg.SetTargetTemperature(2.0, True)
    assert itg.GetThermostatState() == 0.0
    assert itg.GetTargetTemperature() == 2.0


def test_write_read_round_trip(rumd, tmp_path):
    s, g = golden_sample(rumd, tmp_path)
    s.SetPotential(ka_potential(rumd, rumd.ShiftedForce))
    s.SetIntegrator(rumd.IntegratorNVT(0.005, 0.5, 0.2))
    s.Run(50)
    out = tmp_path / "end.xyz.gz"
    s.WriteConf(str(out))
    t = rumd.Sample(0, 0)
    t2 = rumd.IntegratorNVT(0.001, 1.0, 1.0)
    t.SetIntegrator(t2)
    t.ReadConf(str(out), True)
    assert np.allclose(t.GetPositions(), s.GetPositions(), atol=1e-8)
    assert np.array_equal(t.GetImages(), s.GetImages())
    assert np.allclose(t.GetVelocities(), s.GetVelocities(), atol=1e-8)
    # RUMD's ioformat=2 header (ConfigurationWriterReader.cu:90-141): the box
    # and integrator as info strings, no ioformat=1 keys
    import gzip
    with gzip.open(out, "rt") as fh:
        fh.readline()
        meta = dict(tok.split("=", 1) for tok in fh.readline().split())
    assert meta["ioformat"] == "2" and "boxLengths" not in meta and "dt" not in meta
    assert meta["sim_box"].startswith("RectangularSimulationBox,")
    assert [np.float32(x) for x in meta["sim_box"].split(",")[1:]] == [np.float32(x) for x in g["L"]]
    assert meta["integrator"].split(",")[0] == "IntegratorNVT"
    assert t2.GetTimeStep() == np.float32(0.005) and t2.GetTargetTemperature() == 0.5
    # info-string parameters are read as float (ParseInfoString.cc:22)
    xi = s.GetIntegrator().GetThermostatState()
    assert abs(t2.GetThermostatState() - xi) <= 1e-6 * max(1.0, abs(xi))


def test_pb_tp_do_not_change_physics(rumd, tmp_path):
    """Autotune.py:929-937 invariance: pe after a run does not depend on pb/tp."""
    pes = []
    for pb, tp in ((32, 1), (64, 4), (32, 8), (128, 2)):
        s, g = golden_sample(rumd, tmp_path)
        s.SetPB_TP(pb, tp)
        s.SetPotential(ka_potential(rumd, rumd.ShiftedForce))
        s.CalcF()
        pes.append(s.GetPotentialEnergy())
    assert max(pes) - min(pes) < 0.005
