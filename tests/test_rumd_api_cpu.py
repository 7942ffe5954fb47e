"""Host-side logic of the RUMD class surface (no GPU calls).

Parameter mapping, configuration files and error behaviour run entirely on
the host until the first force evaluation creates the device replica."""
import gzip
import os

import numpy as np
import pytest

from conftest import golden_files, load_golden


@pytest.fixture(scope="module")
def rumd():
    from rumd_b200 import build
    build.build()
    from rumd_b200 import rumd
    return rumd


def write_xyz(path, g):
    n = len(g["type"])
    L = g["L"]
    with gzip.open(path, "wt") as fh:
        fh.write(f"{n}\n")
        fh.write(f"ioformat=1 dt=0.005 boxLengths={L[0]:.9f},{L[1]:.9f},{L[2]:.9f} numTypes=2 "
                 f"Nose-Hoover-Ps={g['xi']:.9f} Barostat-Pv=0.0 mass=1.0,1.0 columns=type,x,y,z,vx,vy,vz,fx,fy,fz,pe\n")
        for i in range(n):
            p, v, f = g["pos"][i], g["vel"][i], g["force"][i]
            fh.write(f"{g['type'][i]} {p[0]:.6f} {p[1]:.6f} {p[2]:.6f} {v[0]:.6f} {v[1]:.6f} {v[2]:.6f} "
                     f"{f[0]:.6f} {f[1]:.6f} {f[2]:.6f} {g['pe'][i]:.6f}\n")


def ka_potential(rumd, method):
    pot = rumd.Pot_LJ_12_6(cutoff_method=method)
    pot.SetParams(0, 0, 1.0, 1.0, 2.5)
    pot.SetParams(0, 1, 0.8, 1.5, 2.5)
    pot.SetParams(1, 1, 0.88, 0.5, 2.5)
    return pot


def test_lj_parameter_table_equals_oracle(rumd, oracle):
    pot = ka_potential(rumd, rumd.ShiftedForce)
    table = np.array(pot.ParamTable(2), np.float32)
    ref = oracle.lj_params(2, oracle.ka_table())
    assert np.array_equal(table.view(np.uint32), ref.view(np.uint32))
    # GetPotentialParameter(i, j, 0) is the absolute cut-off Rcut*sigma
    assert pot.GetPotentialParameter(1, 0, 0) == np.float32(2.5) * np.float32(0.8)
    assert pot.GetMaxCutoff() == np.float32(2.5)
    assert len(pot.GetPotentialParameters(2)) == 4 * 10


def test_ipl_and_lj_agree(rumd):
    lj = rumd.Pot_LJ_12_6(rumd.ShiftedPotential)
    lj.SetParams(0, 0, 1.0, 1.0, 2.5)
    ipl = rumd.Pot_IPL_12_6(rumd.ShiftedPotential)
    ipl.SetParams(0, 0, 4.0, -4.0, 2.5)
    assert lj.ParamTable(1) == ipl.ParamTable(1)


def test_readconf_host_side(rumd, tmp_path):
    g = load_golden([p for p in golden_files() if "N1000_T0.5" in p][0])
    path = tmp_path / "conf.xyz.gz"
    write_xyz(path, g)
    s = rumd.Sample(0, 0)
    s.ReadConf(str(path))
    assert s.GetNumberOfParticles() == 1000
    assert s.GetNumberOfTypes() == 2
    assert s.GetNumberThisType(1) == int((g["type"] == 1).sum())
    assert np.allclose(s.GetPositions(), g["pos"], atol=1e-6)
    assert np.allclose(s.GetVelocities(), g["vel"], atol=1e-6)
    assert s.GetNumberOfDOFs() == 3 * 1000 - 3
    assert abs(s.GetVolume() - float(np.prod(g["L"]))) < 1e-3


CONF = os.path.join(os.path.dirname(__file__), "golden", "conf")


def test_read_rumd_ioformat1_file(rumd):
    """RUMD's own Conf/KobAndersen/KA_N256_L6.0_T0.50.xyz.gz (ioformat=1:
    dt, boxLengths, Nose-Hoover-Ps).  Without init_itg the integrator keeps
    its state; with it the thermostat state comes from the file
    (Sample.cu:584-600)."""
    g = load_golden([p for p in golden_files() if "KA_N256_L6.0_T0.50" in p][0])
    path = os.path.join(CONF, "KA_N256_L6.0_T0.50.xyz.gz")
    s = rumd.Sample(0, 0)
    itg = rumd.IntegratorNVT(timeStep=0.005, targetTemperature=0.5, thermostatRelaxationTime=0.2)
    s.SetIntegrator(itg)
    s.ReadConf(path)
    assert itg.GetThermostatState() == 0.0
    s.ReadConf(path, True)
    assert abs(itg.GetThermostatState() - 0.568610489) < 1e-6
    assert s.GetNumberOfParticles() == 256 and s.GetNumberOfTypes() == 2
    assert abs(s.GetVolume() - 216.0) < 1e-3
    assert np.allclose(s.GetPositions(), g["pos"], atol=1e-6)
    assert np.allclose(s.GetVelocities(), g["vel"], atol=1e-6)
    assert np.array_equal(np.asarray(s.GetImages()).reshape(-1, 3), g["im"])


def test_read_rumd_ioformat2_file(rumd):
    """RUMD's own Conf/SingleComponentLiquid/MgCu_equil_0.051_0.055.xyz.gz
    (ioformat=2: integrator=IntegratorNVT,dt,T,tau,xi and
    sim_box=RectangularSimulationBox,Lx,Ly,Lz; masses 24.305 and 63.54).
    With init_itg the integrator takes the file's info string
    (IntegratorNVT::InitializeFromInfoString, IntegratorNVT.cu:265-290)."""
    path = os.path.join(CONF, "MgCu_equil_0.051_0.055.xyz.gz")
    with gzip.open(path, "rt") as fh:
        n = int(fh.readline())
        header = fh.readline().split()
        rows = np.array([fh.readline().split() for _ in range(n)], np.float64)
    meta = dict(t.split("=", 1) for t in header)
    assert meta["ioformat"] == "2"
    s = rumd.Sample(0, 0)
    itg = rumd.IntegratorNVT(timeStep=0.001, targetTemperature=1.0, thermostatRelaxationTime=0.2)
    s.SetIntegrator(itg)
    s.ReadConf(path, True)
    assert s.GetNumberOfParticles() == 1000 and s.GetNumberOfTypes() == 2
    L = np.float32(26.9322929)
    assert abs(s.GetVolume() - float(L) ** 3) < 1e-2
    assert np.allclose(s.GetPositions(), rows[:, 1:4], atol=1e-6)
    assert np.allclose(s.GetVelocities(), rows[:, 7:10], atol=1e-6)
    assert itg.GetTimeStep() == np.float32(0.5)
    assert abs(itg.GetTargetTemperature() - 0.0551250086) < 1e-7
    assert itg.GetRelaxationTime() == np.float32(5.0)
    assert abs(itg.GetThermostatState() - 0.0240456783) < 1e-8
    assert abs(s.GetMass(0) - 24.305) < 1e-4 and abs(s.GetMass(1) - 63.54) < 1e-4
    info = itg.GetInfoString(11)
    assert info.startswith("IntegratorNVT,0.5,")


def test_readconf_rejects_files_without_rumd_metadata(rumd, tmp_path):
    """ConfigurationMetaData::ReadMetaData's checks: ioformat is required,
    ioformat=2 takes the box from sim_box= (boxLengths= is an ioformat=1 key),
    and only the rectangular box is supported here."""
    cases = {
        "noioformat": "boxLengths=5,5,5 columns=type,x,y,z",
        "format2_boxlengths": "ioformat=2 boxLengths=5,5,5 columns=type,x,y,z",
        "lees_edwards": "ioformat=2 sim_box=LeesEdwardsSimulationBox,5,5,5,0.1 columns=type,x,y,z",
    }
    for name, header in cases.items():
        path = tmp_path / f"{name}.xyz.gz"
        with gzip.open(path, "wt") as fh:
            fh.write(f"2\n{header}\n0 0.0 0.0 0.0\n0 1.0 0.0 0.0\n")
        with pytest.raises(RuntimeError):
            rumd.Sample(0, 0).ReadConf(str(path))


def test_errors_map_to_python_exceptions(rumd, tmp_path):
    s = rumd.Sample(0, 0)
    with pytest.raises(RuntimeError):
        s.CalcF()  # no configuration
    with pytest.raises(ValueError):
        s.SetPB_TP(2048, 4)  # beyond any launch shape (RUMD's 16..192 are mapped)
    pot = rumd.Pot_LJ_12_6(rumd.ShiftedForce)
    with pytest.raises(RuntimeError):
        pot.SetNB_Method("cells")
    with pytest.raises(RuntimeError):
        s.ReadConf(str(tmp_path / "missing.xyz.gz"))
    sim = rumd.Simulation(sample=rumd.Sample())
    with pytest.raises(ValueError):
        sim.Run(10)  # no integrator


def test_integrator_settings_before_sample(rumd):
    itg = rumd.IntegratorNVT(timeStep=0.005, targetTemperature=0.8, thermostatRelaxationTime=0.2)
    assert itg.GetTimeStep() == np.float32(0.005)
    assert itg.GetTargetTemperature() == 0.8
    assert itg.GetThermostatOn()
    itg.SetThermostatOn(False)
    assert itg.GetThermostatState() == 0.0
    nve = rumd.IntegratorNVE(timeStep=0.004)
    assert not nve.GetThermostatOn()
    with pytest.raises(RuntimeError):
        itg.SetThermostatOnParticleType(40, True)
