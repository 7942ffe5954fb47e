"""ctypes wrapper of the CPU oracle (oracle/md_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and
by the cpu_baseline / ``--impl reference`` legs of ``bench.py``.  The product
package ``rumd_b200`` never imports this module.

Every function restates a piece of the RUMD reference; the citations are in
``md_oracle.cpp``.  Positions are passed as ``float32[n,4]`` with the particle
type bit-cast into the fourth component (``ParticleData.h:41``), velocities as
``float32[n,4]`` with 1/m in the fourth component.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

NS, SP, SF = 0, 1, 2
NUM_PARAM = 12


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        i, f, d, u = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_uint
        L.orc_lj_set_params.argtypes = [i, P, i, i, f, f, f]
        L.orc_cell_grid.argtypes = [P, f, f, P]
        L.orc_dist2.argtypes = [i, P, P, P, P]
        L.orc_cell_keys.argtypes = [i, P, P, P, P]
        L.orc_stable_sort_perm.argtypes = [i, P, i, P]
        L.orc_nbl_build_cells.argtypes = [i, P, P, P, i, P, f, i, P, P]
        L.orc_nbl_build_cells.restype = i
        L.orc_nbl_build_n2.argtypes = [i, P, P, i, P, f, i, P, P]
        L.orc_nbl_build_n2.restype = i
        L.orc_max_nbrs_estimate.argtypes = [u, f, f, d]
        L.orc_max_nbrs_estimate.restype = u
        L.orc_forces_f64.argtypes = [i, P, P, P, i, P, i, P, P, P]
        L.orc_forces_f64_pot.argtypes = [i, P, P, P, i, P, i, i, P, P, P]
        L.orc_forces_stress_f64_pot.argtypes = [i, P, P, P, i, P, i, i, P, P, P, P, i]
        L.orc_smooth_set_params.argtypes = [i, P, i, i, f, f, f]
        L.orc_ipl_n_set_params.argtypes = [i, P, i, i, f, f, f, f]
        L.orc_forces_f32.argtypes = [i, P, P, i, P, i, P, P, i, P, P]
        run_args = [i, P, P, P, P, i, P, i, f, f, d, d, P, i, i, i, i, P, P]
        L.orc_md_run_f32.argtypes = run_args
        L.orc_md_run_f32.restype = i
        L.orc_md_run_f64.argtypes = run_args
        L.orc_md_run_f64.restype = i
        L.orc_num_threads.restype = i
        L.orc_set_num_threads.argtypes = [i]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def lj_params(ntypes, table):
    """Parameter table from {(i, j): (sigma, epsilon, rcut_in_sigma)}.

    Pot_LJ_12_6::SetParams (PairPotential.h:202-207) + CopyParamsToGPU
    (PairPotential.cu:82-125); (j, i) mirrored.
    """
    params = np.zeros(ntypes * ntypes * NUM_PARAM, np.float32)
    for (i, j), (sig, eps, rc) in table.items():
        lib().orc_lj_set_params(ntypes, _p(params), i, j, sig, eps, rc)
    return params


def smooth_params(ntypes, table):
    """Pot_LJ_12_6_smooth_2_4 table from {(i, j): (sigma, epsilon, rcut_in_sigma)}
    (PairPotential.h:232-246 + CopyParamsToGPU)."""
    params = np.zeros(ntypes * ntypes * NUM_PARAM, np.float32)
    for (i, j), (sig, eps, rc) in table.items():
        lib().orc_smooth_set_params(ntypes, _p(params), i, j, sig, eps, rc)
    return params


def ipl_n_params(ntypes, n, table):
    """Pot_IPL_n table with exponent n from {(i, j): (sigma, epsilon, rcut_in_sigma)}
    (PairPotential.h:616-628 + CopyParamsToGPU)."""
    params = np.zeros(ntypes * ntypes * NUM_PARAM, np.float32)
    for (i, j), (sig, eps, rc) in table.items():
        lib().orc_ipl_n_set_params(ntypes, _p(params), i, j, n, sig, eps, rc)
    return params


def ka_table():
    """Kob-Andersen 80:20 parameters with cut-off 2.5 sigma_ij."""
    return {(0, 0): (1.0, 1.0, 2.5), (0, 1): (0.8, 1.5, 2.5), (1, 1): (0.88, 0.5, 2.5)}


def lj_table():
    return {(0, 0): (1.0, 1.0, 2.5)}


def max_cutoff(params, ntypes):
    return float(params.reshape(ntypes * ntypes, NUM_PARAM)[:, 0].max())


def dist2(a4, b4, L):
    a4 = np.ascontiguousarray(a4, np.float32)
    b4 = np.ascontiguousarray(b4, np.float32)
    out = np.zeros(len(a4), np.float32)
    lib().orc_dist2(len(a4), _p(a4), _p(b4), _p(np.asarray(L, np.float32)), _p(out))
    return out


def cell_grid(L, max_cut, skin):
    nc = np.zeros(3, np.int32)
    Lf = np.asarray(L, np.float32)
    lib().orc_cell_grid(_p(Lf), max_cut, skin, _p(nc))
    return nc


def cell_keys(pos4, L, nc):
    pos4 = np.ascontiguousarray(pos4, np.float32)
    keys = np.zeros(len(pos4), np.int32)
    lib().orc_cell_keys(len(pos4), _p(pos4), _p(np.asarray(L, np.float32)), _p(np.asarray(nc, np.int32)), _p(keys))
    return keys


def stable_sort_perm(keys, ncells):
    keys = np.ascontiguousarray(keys, np.int32)
    old = np.zeros(len(keys), np.uint32)
    lib().orc_stable_sort_perm(len(keys), _p(keys), int(ncells), _p(old))
    return old


def nbl_cells(pos4_sorted, L, nc, ntypes, params, skin, max_nbrs):
    """Sorted cell scan; returns (counts, row-major nbl, overflow)."""
    n = len(pos4_sorted)
    pos4_sorted = np.ascontiguousarray(pos4_sorted, np.float32)
    counts = np.zeros(n, np.uint32)
    nbl = np.zeros((n, max_nbrs), np.uint32)
    ov = lib().orc_nbl_build_cells(n, _p(pos4_sorted), _p(np.asarray(L, np.float32)),
                                   _p(np.asarray(nc, np.int32)), ntypes, _p(params), skin,
                                   max_nbrs, _p(counts), _p(nbl))
    return counts, nbl, ov


def nbl_n2(pos4, L, ntypes, params, skin, max_nbrs):
    n = len(pos4)
    pos4 = np.ascontiguousarray(pos4, np.float32)
    counts = np.zeros(n, np.uint32)
    nbl = np.zeros((n, max_nbrs), np.uint32)
    ov = lib().orc_nbl_build_n2(n, _p(pos4), _p(np.asarray(L, np.float32)), ntypes, _p(params),
                                skin, max_nbrs, _p(counts), _p(nbl))
    return counts, nbl, ov


def max_nbrs_estimate(n, max_cut, skin, volume):
    return int(lib().orc_max_nbrs_estimate(n, max_cut, skin, volume))


POTENTIAL = {"LJ_12_6": 0, "LJ_12_6_smooth_2_4": 1, "IPL_n": 2}


def forces_f64(pos3, types, L, ntypes, params, cutoff, potential="LJ_12_6"):
    """FP64 pair sum; returns (f[n,3], u[n], w[n]) with u halved, w = sum d^2 s."""
    pos3 = np.ascontiguousarray(pos3, np.float64)
    types = np.ascontiguousarray(types, np.int32)
    n = len(pos3)
    f = np.zeros((n, 3)); u = np.zeros(n); w = np.zeros(n)
    lib().orc_forces_f64_pot(n, _p(pos3), _p(types), _p(np.asarray(L, np.float64)), ntypes,
                             _p(params), cutoff, POTENTIAL[potential], _p(f), _p(u), _p(w))
    return f, u, w


def stress_f64(pos3, types, L, ntypes, params, cutoff, potential="LJ_12_6", fp32_cut=True):
    """FP64 per-particle pair stress of fij's STR branch (PairPotential.h:1232-1241):
    [n, 6] = (xx, yy, zz, yz, xz, xy), each -sum_j d_a d_b s.  fp32_cut: the
    pairs summed are those the reference's FP32 cut-off test admits."""
    pos3 = np.ascontiguousarray(pos3, np.float64)
    types = np.ascontiguousarray(types, np.int32)
    n = len(pos3)
    f = np.zeros((n, 3)); u = np.zeros(n); w = np.zeros(n); sts = np.zeros((n, 6))
    lib().orc_forces_stress_f64_pot(n, _p(pos3), _p(types), _p(np.asarray(L, np.float64)), ntypes,
                                    _p(params), cutoff, POTENTIAL[potential], _p(f), _p(u), _p(w), _p(sts),
                                    int(bool(fp32_cut)))
    return sts


def sample_stress(sts6, vel4, L, include_kinetic=True):
    """Sample::GetStress (Sample.cu:393-444): 0.5 * (sum of the particles'
    pair stresses, minus 2 m v_a v_b per particle when the kinetic part is
    included) / V, in FP64, order (xx, yy, zz, yz, xz, xy)."""
    st = np.asarray(sts6, np.float64).sum(axis=0)
    if include_kinetic:
        v = np.asarray(vel4, np.float64)
        m2 = 2.0 / v[:, 3]
        vx, vy, vz = v[:, 0], v[:, 1], v[:, 2]
        st = st - np.array([(m2 * vx * vx).sum(), (m2 * vy * vy).sum(), (m2 * vz * vz).sum(),
                            (m2 * vy * vz).sum(), (m2 * vx * vz).sum(), (m2 * vx * vy).sum()])
    V = float(np.prod(np.asarray(L, np.float64)))
    return 0.5 * st / V


def forces_f32(pos4, L, ntypes, params, cutoff, counts, nbl):
    pos4 = np.ascontiguousarray(pos4, np.float32)
    nbl = np.ascontiguousarray(nbl, np.uint32)
    n = len(pos4)
    f4 = np.zeros((n, 4), np.float32); w = np.zeros(n, np.float32)
    lib().orc_forces_f32(n, _p(pos4), _p(np.asarray(L, np.float32)), ntypes, _p(params), cutoff,
                         _p(np.ascontiguousarray(counts, np.uint32)), _p(nbl), nbl.shape[1],
                         _p(f4), _p(w))
    return f4, w


def md_run(pos4, vel4, im3, L, ntypes, params, cutoff, skin, dt, T, tau, nsteps,
           xi=0.0, thermostat=True, reset_interval=100, max_nbrs=None, precision="f32",
           want_forces=False):
    """Runs Simulation.Run(nsteps) on the CPU.

    Returns dict with updated pos4/vel4/im3 (original order), xi, per-step
    energies [nsteps, 4] = (pe, W, KE(t), xi) and the number of list rebuilds.
    """
    pos4 = np.array(pos4, np.float32, copy=True)
    vel4 = np.array(vel4, np.float32, copy=True)
    im3 = np.array(im3, np.int32, copy=True)
    n = len(pos4)
    if max_nbrs is None:
        vol = float(np.prod(np.asarray(L, np.float64)))
        max_nbrs = max(64, int(2.0 * (4.0 / 3.0) * np.pi * (max_cutoff(params, ntypes) + skin) ** 3 * n / vol))
    en = np.zeros((nsteps, 4))
    xi_c = ctypes.c_double(xi)
    f_out = np.zeros((n, 3)) if want_forces else None
    fn = lib().orc_md_run_f32 if precision == "f32" else lib().orc_md_run_f64
    rb = fn(n, _p(pos4), _p(vel4), _p(im3), _p(np.asarray(L, np.float32)), ntypes, _p(params),
            cutoff, skin, dt, T, tau, ctypes.byref(xi_c), int(bool(thermostat)), nsteps,
            reset_interval, max_nbrs, _p(en), _p(f_out) if f_out is not None else None)
    if rb < 0:
        raise RuntimeError("oracle neighbour list overflow")
    out = dict(pos4=pos4, vel4=vel4, im3=im3, xi=xi_c.value, energies=en, rebuilds=rb)
    if want_forces:
        out["forces"] = f_out
    return out


def num_threads():
    return int(lib().orc_num_threads())


def set_num_threads(n):
    lib().orc_set_num_threads(int(n))
