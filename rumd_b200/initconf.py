"""Seeded initial configurations and LJ parameter tables.

Configurations follow the recipe of RUMD's ``rumd_init_conf`` tool
(Tools/rumd_init_conf.h:16-52): an FCC lattice scaled to the requested number
density, a seeded random assignment of particle types, and Maxwell-Boltzmann
velocities at temperature T with the centre-of-mass momentum removed.  When
4*n^3 != N the first N sites of the smallest FCC lattice with >= N sites are
used.

Parameter tables reproduce Pot_LJ_12_6::SetParams (PairPotential.h:202-207)
followed by PairPotential::CopyParamsToGPU (PairPotential.cu:82-125): A12 and
A6 are evaluated in double and stored as float, the cut-off is Rcut*sigma in
float, and the shift constants p10 = s(rc)*rc and p11 = u(rc) are computed
with the FP32 Pot_IPL_12_6::ComputeInteraction arithmetic.  The tables of
Pot_LJ_12_6_smooth_2_4 and Pot_IPL_n follow their SetParams the same way.
"""
import math

import numpy as np

NUM_PARAM = 12
KA = {(0, 0): (1.0, 1.0, 2.5), (0, 1): (0.8, 1.5, 2.5), (1, 1): (0.88, 0.5, 2.5)}
LJ = {(0, 0): (1.0, 1.0, 2.5)}


def _ipl_12_6_f32(dist2, a12, a6):
    f = np.float32
    inv2 = f(1.0) / f(dist2)
    inv6 = inv2 * inv2 * inv2
    temp = f(a12) * inv6
    s = inv6 * inv2 * (f(12.0) * temp + f(6.0) * f(a6))
    u = f(0.0) + inv6 * (temp + f(a6))
    return f(s), f(u)


def lj_row(sigma, epsilon, rcut):
    f = np.float32
    row = np.zeros(NUM_PARAM, np.float32)
    sigma, epsilon, rcut = f(sigma), f(epsilon), f(rcut)
    row[0] = rcut * sigma
    row[1] = f(4.0 * float(epsilon) * float(sigma) ** 12)
    row[2] = f(-4.0 * float(epsilon) * float(sigma) ** 6)
    rc = row[0]
    if rc > 0:
        s, u = _ipl_12_6_f32(rc * rc, row[1], row[2])
        row[NUM_PARAM - 1] = u
        row[NUM_PARAM - 2] = s * rc
    return row


def _shifts(row, pair):
    """p11 = u(rc), p10 = s(rc)*rc from the float pair function (PairPotential.cu:82-125)."""
    rc = row[0]
    if rc > 0:
        s, u = pair(rc * rc, row)
        row[NUM_PARAM - 1] = u
        row[NUM_PARAM - 2] = s * rc
    return row


def _smooth_2_4_f32(dist2, p):
    # Pot_LJ_12_6_smooth_2_4::ComputeInteraction (PairPotential.h:248-255)
    f = np.float32
    d2 = f(dist2) * p[1]
    i2 = f(1.0) / d2
    i6 = i2 * i2 * i2
    s = p[2] * p[1] * (i2 * i6 * (f(12.0) * i6 - f(6.0)) - f(2.0) * p[3] - f(4.0) * p[4] * d2)
    u = f(0.0) + p[2] * (i6 * (i6 - f(1.0)) + p[3] * d2 + p[4] * d2 * d2)
    return f(s), f(u)


def _ipl_n_f32(dist2, p):
    # Pot_IPL_n::ComputeInteraction (PairPotential.h:630-636); logf, expf as
    # correctly rounded float functions
    f = np.float32
    i2 = f(1.0) / (f(dist2) * p[1])
    tn = f(math.exp(float(f(math.log(float(i2))) * p[3] * f(0.5))))
    s = p[1] * p[2] * p[3] * tn * i2
    u = f(0.0) + p[2] * tn
    return f(s), f(u)


def smooth_row(sigma, epsilon, rcut):
    """Pot_LJ_12_6_smooth_2_4::SetParams (PairPotential.h:232-246): c2, c4 in
    double from rcut in units of sigma, stored as float."""
    f = np.float32
    row = np.zeros(NUM_PARAM, np.float32)
    sigma, epsilon, rcut = f(sigma), f(epsilon), f(rcut)
    row[0] = rcut * sigma
    row[1] = f(1.0) / (sigma * sigma)
    row[2] = f(4.0) * epsilon
    x = float(rcut)
    row[3] = f(48.0 * x ** -14.0 - 15.0 * x ** -8.0)
    row[4] = f(6.0 * x ** -10.0 - 21.0 * x ** -16.0)
    return _shifts(row, _smooth_2_4_f32)


def ipl_n_row(n, sigma, epsilon, rcut):
    """Pot_IPL_n::SetParams (PairPotential.h:616-628)."""
    f = np.float32
    row = np.zeros(NUM_PARAM, np.float32)
    sigma, epsilon, rcut = f(sigma), f(epsilon), f(rcut)
    row[0] = rcut * sigma
    row[1] = f(1.0) / (sigma * sigma)
    row[2] = epsilon
    row[3] = f(n)
    return _shifts(row, _ipl_n_f32)


def _table(ntypes, table, row_of):
    p = np.zeros((ntypes, ntypes, NUM_PARAM), np.float32)
    for (i, j), args in table.items():
        row = row_of(*args)
        p[i, j] = row
        p[j, i] = row
    return p.reshape(-1)


def lj_params(ntypes, table):
    """RUMD parameter table float32[ntypes*ntypes*12] from {(i,j): (sigma, eps, rcut/sigma)}."""
    return _table(ntypes, table, lj_row)


def smooth_params(ntypes, table):
    """Pot_LJ_12_6_smooth_2_4 table from {(i,j): (sigma, eps, rcut/sigma)}."""
    return _table(ntypes, table, smooth_row)


def ipl_n_params(ntypes, n, table):
    """Pot_IPL_n table with exponent n from {(i,j): (sigma, eps, rcut/sigma)}."""
    return _table(ntypes, table, lambda sig, eps, rc: ipl_n_row(n, sig, eps, rc))


def fcc_positions(n, density):
    """The first n sites of the smallest FCC lattice with >= n sites, box
    scaled to density, as RUMD's rumd_init_conf drops the trailing sites
    (Tools/rumd_init_conf.cc:460-467).  When n is not 4 m^3 the particles fill
    part of the box at up to twice the density at the start; neighbour lists
    sized for the mean density may overflow in the first steps, and the
    engine enlarges them (NeighborList.cu:657-676)."""
    m = 1
    while 4 * m ** 3 < n:
        m += 1
    L = (n / density) ** (1.0 / 3.0)
    a = L / m
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    sites = (g[:, None, :] + basis[None, :, :]).reshape(-1, 3)[:n]
    pos = (sites + 0.25) * a - L / 2.0
    return pos, np.array([L, L, L])


def make_config(n, density, T, fractions=(1.0,), masses=(1.0,), seed=0):
    """Returns dict(pos4, vel4, im3, box, types): float32 arrays ready for the engine."""
    rng = np.random.default_rng(seed)
    pos, box = fcc_positions(n, density)
    counts = [int(round(fr * n)) for fr in fractions]
    counts[-1] = n - sum(counts[:-1])
    types = np.concatenate([np.full(c, t, np.int32) for t, c in enumerate(counts)])
    rng.shuffle(types)
    m = np.asarray(masses, np.float64)[types]
    vel = rng.normal(size=(n, 3)) * np.sqrt(T / m)[:, None]
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    pos32 = pos.astype(np.float32)
    # wrap into [-L/2, L/2) exactly as the integrator would
    Lf = box.astype(np.float32)
    pos32 = pos32 - Lf * np.rint(pos32 * (np.float32(1) / Lf))
    pos4 = np.zeros((n, 4), np.float32)
    pos4[:, :3] = pos32
    pos4[:, 3] = types.view(np.float32)
    vel4 = np.zeros((n, 4), np.float32)
    vel4[:, :3] = vel
    vel4[:, 3] = (1.0 / m).astype(np.float32)
    return dict(pos4=pos4, vel4=vel4, im3=np.zeros((n, 3), np.int32), box=Lf, types=types)


def ka_config(n, density=1.2, T=0.73, seed=0):
    """Kob-Andersen 80:20 binary mixture."""
    return make_config(n, density, T, fractions=(0.8, 0.2), masses=(1.0, 1.0), seed=seed)


def lj_config(n, density=0.8442, T=0.722, seed=0):
    return make_config(n, density, T, seed=seed)


def ka_batch_workload(seed=0, replicas=256, n_min=512, n_max=8192, T_min=0.45, T_max=2.0):
    """The batching configuration: Kob-Andersen replicas at density 1.2 with
    N = floor(exp(U(ln n_min, ln n_max))) (seeded PCG64) and temperatures
    log-spaced from T_min to T_max.  Returns (sizes, temperatures, configs)."""
    rng = np.random.default_rng(seed)
    ns = np.floor(np.exp(rng.uniform(np.log(n_min), np.log(n_max), replicas))).astype(int)
    Ts = np.exp(np.linspace(np.log(T_min), np.log(T_max), replicas))
    confs = [ka_config(int(n), T=float(T), seed=seed + k) for k, (n, T) in enumerate(zip(ns, Ts))]
    return ns, Ts, confs
