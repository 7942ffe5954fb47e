"""The FP64 engine (b2md_f64_*, RUMD's step in double precision throughout, as
built by changeToDouble.sh) against the FP64 oracle, and the FP32 engine
against it: the accuracy statements for the single-component LJ system of
N = 1,048,576 at density 0.8442 (the HBM-scale plain configuration)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from rumd_b200 import build, capi
    build.build_lib()
    return capi


def melted(capi, cfg, params, ntypes, T, steps, dt=0.004):
    e = capi.Engine(device=0, pb=64, tp=2)
    rid = e.add(cfg["pos4"], cfg["box"], params, ntypes, cutoff="SF", dt=dt, T=T, vel4=cfg["vel4"])
    e.run(steps)
    n = len(cfg["pos4"])
    out = dict(pos4=e.get(rid, "pos", n), vel4=e.get(rid, "vel", n), box=cfg["box"])
    e.close()
    return out


def test_f64_forces_match_fp64_oracle(capi, oracle):
    from rumd_b200 import initconf as I
    params = oracle.lj_params(2, oracle.ka_table())
    m = melted(capi, I.ka_config(6000, T=1.0, seed=4), params, 2, T=1.0, steps=200, dt=0.005)
    types = np.ascontiguousarray(m["pos4"][:, 3]).view(np.int32)
    f_ref, u_ref, w_ref = oracle.forces_f64(m["pos4"][:, :3].astype(np.float64), types, m["box"], 2, params, 2)
    e = capi.F64Engine(m["pos4"], m["box"], params, 2, cutoff="SF", vel4=m["vel4"].astype(np.float64))
    e.calc_f()
    f = e.get("force")
    st = e.stats()
    e.close()
    err = np.sqrt(np.sum((f[:, :3] - f_ref) ** 2) / np.sum(f_ref ** 2))
    assert err < 1e-12
    assert abs(st["pe"] - u_ref.sum()) <= 1e-11 * abs(u_ref.sum())
    assert abs(st["virial"] - w_ref.sum() / 6.0) <= 1e-11 * abs(w_ref.sum())
    assert np.allclose(f[:, 3], u_ref, rtol=0, atol=1e-12)


@pytest.mark.parametrize("thermostat", [True, False])
def test_f64_trajectory_matches_fp64_oracle(capi, oracle, thermostat):
    """100 NVT (or NVE) steps from the same start: per-step pe, W, KE(t), xi."""
    from rumd_b200 import initconf as I
    params = oracle.lj_params(2, oracle.ka_table())
    m = melted(capi, I.ka_config(2000, T=0.9, seed=6), params, 2, T=0.9, steps=300, dt=0.005)
    n = 2000
    im3 = np.zeros((n, 3), np.int32)
    dt, T, tau, steps = np.float32(0.005), 0.9, 0.2, 100
    ref = oracle.md_run(m["pos4"], m["vel4"], im3, m["box"], 2, params, 2, 0.3, dt, T, tau, steps,
                        thermostat=thermostat, reset_interval=100, precision="f64")
    e = capi.F64Engine(m["pos4"], m["box"], params, 2, cutoff="SF", skin=0.3, dt=float(dt), T=T, tau=tau,
                       thermostat=thermostat, reset_interval=100, vel4=m["vel4"].astype(np.float64))
    en = e.run(steps, energies=True)
    pos = e.get("pos")
    im = e.get("images")
    e.close()
    rel = np.abs(en - ref["energies"]) / np.maximum(np.abs(ref["energies"]), 1e-3)
    assert rel[:, :3].max() < 1e-9
    if thermostat:
        assert np.abs(en[:, 3] - ref["energies"][:, 3]).max() < 1e-9
    # the oracle hands positions back rounded to float32
    assert np.abs(pos[:, :3] - ref["pos4"][:, :3].astype(np.float64)).max() < 1e-5
    assert np.array_equal(im, ref["im3"])


def test_f64_rejects_bad_input(capi, oracle):
    params = oracle.lj_params(1, oracle.lj_table())
    pos4 = np.zeros((10, 4))
    pos4[:, 3] = 3.0  # type 3 of a 1-type system
    with pytest.raises(ValueError):
        capi.F64Engine(pos4, [5.0, 5.0, 5.0], params, 1)


def lj_state(capi, oracle, n, T, steps):
    from rumd_b200 import initconf as I
    params = oracle.lj_params(1, oracle.lj_table())
    return params, melted(capi, I.lj_config(n, T=2.0, seed=8), params, 1, T=T, steps=steps)


def test_fp32_engine_against_f64_engine_same_configuration(capi, oracle):
    """At one configuration: FP32 forces rms rel <= 1e-5 against FP64, and the
    energy and pressure differences per particle."""
    params, m = lj_state(capi, oracle, 32000, T=0.722, steps=400)
    n = 32000
    e32 = capi.Engine(device=0, pb=64, tp=2)
    rid = e32.add(m["pos4"], m["box"], params, 1, cutoff="SF", dt=0.004, T=0.722, vel4=m["vel4"])
    e32.calc_f()
    f32 = e32.get(rid, "force", n)
    s32 = e32.stats(rid)
    e32.close()
    e64 = capi.F64Engine(m["pos4"], m["box"], params, 1, cutoff="SF", vel4=m["vel4"].astype(np.float64))
    e64.calc_f()
    f64 = e64.get("force")
    s64 = e64.stats()
    e64.close()
    err = np.sqrt(np.sum((f32[:, :3] - f64[:, :3]) ** 2) / np.sum(f64[:, :3] ** 2))
    assert err <= 1e-5
    vol = float(np.prod(m["box"]))
    assert abs(s32["pe"] - s64["pe"]) / n < 2e-6
    assert abs(s32["virial"] - s64["virial"]) / vol < 2e-6


def nve_drift(log_t, etot):
    return np.polyfit(log_t, etot, 1)[0]


def test_hbm_scale_lj_fp32_and_fp64_nve_drift(capi, oracle):
    """Single-component LJ, N = 1,048,576, density 0.8442, SF rc = 2.5,
    dt = 0.004, skin 0.3: 1e4 NVE steps in FP32 and in FP64 from the same
    equilibrated state; drift of (pe + KE)/N, the linear trend over the run,
    below 1e-4 in both."""
    n, steps = 1048576, 10000
    params, m = lj_state(capi, oracle, n, T=0.722, steps=600)
    # FP32 engine, NVE
    e32 = capi.Engine(device=0, pb=64, tp=2)
    rid = e32.add(m["pos4"], m["box"], params, 1, cutoff="SF", dt=0.004, thermostat=False, vel4=m["vel4"],
                  reset_interval=0, energy_interval=50, energy_capacity=steps // 50)
    e32.run(steps)
    log = e32.energy_log(rid)
    e32.close()
    et32 = (log[:, 1] + log[:, 3]) / n
    d32 = nve_drift(log[:, 0], et32) * steps
    # FP64 engine, NVE
    e64 = capi.F64Engine(m["pos4"], m["box"], params, 1, cutoff="SF", dt=0.004, thermostat=False,
                         reset_interval=0, vel4=m["vel4"].astype(np.float64))
    en = e64.run(steps, energies=True)
    e64.close()
    et64 = (en[:, 0] + en[:, 2]) / n
    d64 = nve_drift(np.arange(steps), et64) * steps
    print(f"NVE drift per particle over 1e4 steps: FP32 {d32:.3e}, FP64 {d64:.3e}; "
          f"E/N start FP32 {et32[0]:.7f} FP64 {et64[0]:.7f}")
    assert abs(d32) < 1e-4
    assert abs(d64) < 1e-4
    # the two runs start from the same state: the first energies agree to FP32 accuracy
    assert abs(et32[0] - et64[0]) < 1e-5
