// Kernels of the B200 RUMD engine (sm_100a).  See engine_dev.cuh for layout.
//
// Arithmetic contract
//   * Neighbour-list decisions (cell keys, d^2 < (rc+skin)^2, displacement
//     trigger) use the exact FP32 operation sequence of the reference source
//     (SimulationBox.h:111-125, NeighborList.cu:1106-1140, 1282-1285) with the
//     multiply-add contractions that nvcc applies to it written out as
//     __fmaf_rn, so list sets and the sort permutation are bit-exact.
//   * Pair forces are FP32 (PairPotential.h:161-168, 1198-1244); 1/r is the
//     hardware reciprocal square root refined by one Newton-Raphson step and
//     1/r^2 its square.
//   * Reductions (pe, virial, kinetic energy, momentum) are FP64 with a fixed
//     summation tree, so results do not depend on scheduling or on which other
//     replicas share the launch; the thermostat state is FP64.
#pragma once
#include "engine_dev.cuh"
#include "pbc_math.cuh"
#include "tma.cuh"

namespace b2md {

__device__ __forceinline__ double warp_sum_d(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Block sum of kNPart doubles per thread -> s_out[kNPart] (valid after return,
// fixed tree: warp butterfly then warps in index order).
__device__ __forceinline__ void block_sum8(double (&v)[kNPart], double* s_warp, double* s_out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < kNPart; ++k) {
    double x = warp_sum_d(v[k]);
    if (lane == 0) s_warp[wid * kNPart + k] = x;
  }
  __syncthreads();
  if (threadIdx.x < kNPart) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += s_warp[w * kNPart + threadIdx.x];
    s_out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Ordered strided sum of count rows of kNPart doubles (deterministic).
__device__ __forceinline__ void block_rows_sum(const double* base, int count, double* s_scr, double* s_out) {
  const int nslot = blockDim.x / kNPart;
  const int k = threadIdx.x % kNPart, slot = threadIdx.x / kNPart;
  double acc = 0.0;
  if (slot < nslot) {
    // two rows' loads in flight at a time (the sum stays in row order)
    int t = slot;
    for (; t + nslot < count; t += 2 * nslot) {
      const double x0 = __ldcg(base + (size_t)t * kNPart + k);
      const double x1 = __ldcg(base + (size_t)(t + nslot) * kNPart + k);
      acc += x0;
      acc += x1;
    }
    if (t < count) acc += __ldcg(base + (size_t)t * kNPart + k);
  }
  s_scr[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < kNPart) {
    double s = 0.0;
    for (int q = 0; q < nslot; ++q) s += s_scr[q * kNPart + threadIdx.x];
    s_out[threadIdx.x] = s;
  }
  __syncthreads();
}

// atomicAdd with release (the block's earlier writes, ordered before by a
// block barrier, are visible first) and acquire (the caller then sees the
// writes the other blocks released) at GPU scope: one round trip where a
// fence followed by an atomic took two.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Two-level deterministic replica reduction.  Every block of the replica
// calls it with its block totals in s_blk; returns true in exactly one block
// (the last to finish) with the replica totals in s_tot.
__device__ bool replica_reduce(const EngArgs& a, int rep, const RepDev& R, int lt,
                               const double* s_blk, double* s_scr, double* s_tot) {
  __shared__ int s_last;
  const int g = lt / kGroup;
  const int gfirst = g * kGroup;
  const int gsize = min(kGroup, R.ntiles - gfirst);
  if (threadIdx.x < kNPart) a.tpart[(size_t)(R.tile0 + lt) * kNPart + threadIdx.x] = s_blk[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned c = atom_add_acq_rel(&a.gctr[R.group0 + g], 1u);
    s_last = (c == (unsigned)(gsize - 1));
  }
  __syncthreads();
  if (!s_last) return false;
  block_rows_sum(a.tpart + (size_t)(R.tile0 + gfirst) * kNPart, gsize, s_scr, s_tot);
  if (threadIdx.x < kNPart) a.gpart[(size_t)(R.group0 + g) * kNPart + threadIdx.x] = s_tot[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    a.gctr[R.group0 + g] = 0u;
    unsigned c = atom_add_acq_rel(&a.rctr[rep], 1u);
    s_last = (c == (unsigned)(R.ngroups - 1));
  }
  __syncthreads();
  if (!s_last) return false;
  block_rows_sum(a.gpart + (size_t)R.group0 * kNPart, R.ngroups, s_scr, s_tot);
  if (threadIdx.x == 0) a.rctr[rep] = 0u;
  return true;
}

// The replica reduction of k_steps, run by every block after its step-barrier
// arrival, on the step's half (par) of the partial-sum and counter buffers:
// the tile's group counter, then (last block of the group) the group total
// and the replica counter.  Returns true in the replica's last block, which
// then sums the group totals and finishes the step; the other blocks have
// gone on to the next step and wait for that only before they integrate.
__device__ bool post_reduce(const EngArgs& a, int tile, int rep, const RepDev& R, int par, double* s_scr,
                            double* s_tot) {
  __shared__ int s_last;
  const int lt = tile - R.tile0;
  const int g = lt / kGroup;
  const int gfirst = g * kGroup;
  const int gsize = min(kGroup, R.ntiles - gfirst);
  unsigned* gctr = a.gctr + (size_t)par * a.gctr_half;
  unsigned* rctr = a.rctr + (size_t)par * a.rctr_half;
  double* gpart = a.gpart + (size_t)par * a.gpart_half;
  const double* tpart = a.tpart + (size_t)par * a.tpart_half;
  if (threadIdx.x == 0) {
    unsigned c = atom_add_acq_rel(&gctr[R.group0 + g], 1u);
    s_last = (c == (unsigned)(gsize - 1));
  }
  __syncthreads();
  if (!s_last) return false;
  block_rows_sum(tpart + (size_t)(R.tile0 + gfirst) * kNPart, gsize, s_scr, s_tot);
  if (threadIdx.x < kNPart) gpart[(size_t)(R.group0 + g) * kNPart + threadIdx.x] = s_tot[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    gctr[R.group0 + g] = 0u;
    unsigned c = atom_add_acq_rel(&rctr[rep], 1u);
    s_last = (c == (unsigned)(R.ngroups - 1));
    if (s_last) rctr[rep] = 0u;
  }
  __syncthreads();
  if (!s_last) return false;
  block_rows_sum(gpart + (size_t)R.group0 * kNPart, R.ngroups, s_scr, s_tot);
  return true;
}

// Last block of the whole grid: publishes "any replica needs a rebuild" to
// the next conditional graph node (or nothing when launched eagerly), and
// clears the SM-region tile counters (every block has made its last claim).
__device__ __forceinline__ void grid_final(const EngArgs& a, int has_cond, cudaGraphConditionalHandle h) {
  if (threadIdx.x == 0) {
    unsigned c = atom_add_acq_rel(a.fctr, 1u);
    if (c == gridDim.x - 1) {
      int any = atomicExch(a.any_rebuild, 0);
      *a.fctr = 0u;
      for (int k = 0; k <= a.nreg && a.nreg > 0; ++k) a.smctr[k] = 0u;
      if (has_cond) cudaGraphSetConditional(h, any ? 1u : 0u);
    }
  }
}

// First tile of SM region r (regions split [0, ntiles) evenly).
__device__ __forceinline__ int region_first(const EngArgs& a, int r) {
  return (int)(((long long)r * a.ntiles) / a.nreg);
}

// Called by warp 0; returns (in every lane) a tile no other block has
// claimed, or -1 when every tile is claimed.  A block first claims from its
// own SM's region (smctr[r] counts claim attempts there; the first
// region-size ones succeed); when that is used up and smctr[nreg] (tiles
// claimed so far) shows tiles left, the warp scans the other regions, 32 at
// a time, and claims from one with tiles left.  Every claim is a single
// atomic; nothing waits on another block.
__device__ int claim_tile(const EngArgs& a) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nreg = a.nreg;
  unsigned* ctr = a.smctr;
  unsigned smid;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
  const int r0 = (int)(smid % (unsigned)nreg);
  int tile = -1;
  if (lane == 0) {
    const int lo = region_first(a, r0), size = region_first(a, r0 + 1) - lo;
    if (size > 0) {
      const unsigned t = atomicAdd(&ctr[r0], 1u);
      if (t < (unsigned)size) tile = lo + (int)t;
    }
  }
  tile = __shfl_sync(FULL, tile, 0);
  if (tile < 0) {
    const unsigned done = __shfl_sync(FULL, lane == 0 ? *(volatile unsigned*)&ctr[nreg] : 0u, 0);
    if (done < (unsigned)a.ntiles) {
      for (int base = 1; base < nreg && tile < 0; base += 32) {
        const int q = base + lane;
        int r = -1, lo = 0, size = 0;
        if (q < nreg) {
          r = (r0 + q) % nreg;
          lo = region_first(a, r);
          size = region_first(a, r + 1) - lo;
          if (*(volatile unsigned*)&ctr[r] >= (unsigned)size) r = -1;
        }
        unsigned m = __ballot_sync(FULL, r >= 0);
        while (m && tile < 0) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          const int rr = __shfl_sync(FULL, r, src), rlo = __shfl_sync(FULL, lo, src);
          const int rsize = __shfl_sync(FULL, size, src);
          int got = -1;
          if (lane == 0) {
            const unsigned t = atomicAdd(&ctr[rr], 1u);
            if (t < (unsigned)rsize) got = rlo + (int)t;
          }
          tile = __shfl_sync(FULL, got, 0);
        }
      }
    }
  }
  if (tile >= 0 && lane == 0) atomicAdd(&ctr[nreg], 1u);
  return tile;
}

// Nose-Hoover leap-frog for one particle (integrateNVTAlgorithm,
// IntegratorNVT.cu:364-418); accumulates FP64 kinetic sums.
__device__ __forceinline__ void integrate_one(const RepDev& R, float xi_f, float3 vshift, bool do_reset,
                                              float4 r, float4 f, float4& v, int4& im, float4& rn,
                                              double (&acc)[kNPart], bool& exceed, float4 lr) {
  const int ti = __float_as_int(r.w);
  const bool thermo = (R.thermo_mask >> ti) & 1u;
  if (do_reset) { v.x -= vshift.x; v.y -= vshift.y; v.z -= vshift.z; }
  const float xs = thermo ? xi_f : 0.f;
  const float dt = R.dt;
  const NvtCoef c = nvt_coef(xs, dt);
  const double vb = (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z;
  float vx = nvt_velocity(c, v.x, v.w, f.x, dt);
  float vy = nvt_velocity(c, v.y, v.w, f.y, dt);
  float vz = nvt_velocity(c, v.z, v.w, f.z, dt);
  float x = nvt_position(r.x, vx, dt), y = nvt_position(r.y, vy, dt), z = nvt_position(r.z, vz, dt);
  float kx = wrap_image(x, R.invL[0]), ky = wrap_image(y, R.invL[1]), kz = wrap_image(z, R.invL[2]);
  x = wrap_apply(x, R.L[0], kx); y = wrap_apply(y, R.L[1], ky); z = wrap_apply(z, R.L[2], kz);
  im.x += (int)kx; im.y += (int)ky; im.z += (int)kz;
  v.x = vx; v.y = vy; v.z = vz;
  rn = make_float4(x, y, z, r.w);
  const double m = 1.0 / (double)v.w;
  const double vf = (double)vx * vx + (double)vy * vy + (double)vz * vz;
  acc[P_KET] += 0.25 * m * (vb + vf);
  if (thermo) acc[P_KE2] += m * vf;
  acc[P_PX] += m * vx; acc[P_PY] += m * vy; acc[P_PZ] += m * vz;
  acc[P_M] += m;
  // displacement since the last build (displacement_since_nb_build, NeighborList.cu:970-997)
  float d2 = dist2_ref(mi_comp(x - lr.x, R.L[0], R.invL[0]), mi_comp(y - lr.y, R.L[1], R.invL[1]),
                       mi_comp(z - lr.z, R.L[2], R.invL[2]));
  exceed = d2 > R.skin2_4;
}

// k_steps: what this block adds to its step-barrier arrival (its replica
// still has steps, its tile asks for a rebuild); thread 0 only.
__shared__ unsigned long long s_step_tally;
// k_flow: the finalizing block's decision for its replica's next step
// (-1: this block did not finalize; 0 stop, 1 force items, 2 rebuild items)
__shared__ int s_fin;
constexpr int kFlowPar = -2;  // finish_step's bpar in k_flow
constexpr int kTallyMoreShift = 24, kTallyRebuildShift = 44;
constexpr unsigned long long kTallyArriveMask = (1ull << kTallyMoreShift) - 1ull;
constexpr unsigned long long kTallyField = (1ull << 20) - 1ull;

// Replica bookkeeping after an integration step (last block only).
// bpar >= 0 (k_batch): the replica tallies "steps left" with the block's
// barrier arrival and, when its list is due and it has steps left, joins the
// rebuild list of the next step (parity bpar).
__device__ void finish_step(const EngArgs& a, int rep, const RepDev& R, RepState* S, const double* tot,
                            bool with_forces, int bpar = -1) {
  if (threadIdx.x != 0) return;
  // the state is read past L1 (in k_steps the previous step's finalizer may
  // have run on another SM), all loads at once: this runs on the step's
  // critical path
  const double T0 = __ldcg(&S->T), dT = __ldcg(&S->dT), xi0 = __ldcg(&S->xi);
  const double pe0 = __ldcg(&S->pe), vir0 = __ldcg(&S->vir);
  const long long run_idx = __ldcg(&S->run_step);  // step index inside the current run, before this step
  const long long steps = __ldcg(&S->steps), left = __ldcg(&S->steps_left);
  const int rbuf = __ldcg(&S->rbuf), nlog = __ldcg(&S->nlog);
  double xi = xi0, T = T0;
  if (R.thermo_mask) {
    double dev = tot[P_KE2] / (R.dof * T0) - 1.0;
    if (dev > 10.0) dev = 10.0;  // updateNVTThermostatState (IntegratorNVT.cu:426-437)
    xi = xi0 + (double)R.dt * (double)R.omega2 * dev;
    T = T0 + dT;
  }
  S->xi = xi;
  S->T = T;
  S->ke2 = tot[P_KE2];
  S->ke_t = tot[P_KET];
  const double pe = with_forces ? tot[P_PE] : pe0, vir = with_forces ? tot[P_W] / 6.0 : vir0;
  S->pe = pe;
  S->vir = vir;
  S->P[0] = tot[P_PX]; S->P[1] = tot[P_PY]; S->P[2] = tot[P_PZ]; S->M = tot[P_M];
  S->rbuf = rbuf ^ 1;
  S->steps = steps + 1;
  S->run_step = run_idx + 1;
  if (left > 0) S->steps_left = left - 1;
  int ex = atomicExch(&S->exceed, 0);
  S->rebuild = ex > 0;
  if (ex > 0) atomicAdd(a.any_rebuild, 1);
  if (bpar == kFlowPar) {
    // k_flow: the replica's steps in this launch, and what comes next
    const int ls = __ldcg(&S->launch_steps) + 1;
    S->launch_steps = ls;
    atomicMax(&a.pctl->ran, ls);
    s_fin = (left > 1 && ls < __ldcg(&a.pctl->budget)) ? (ex > 0 ? 2 : 1) : 0;
  }
  if (bpar >= 0 && left > 1) {
    s_step_tally += 1ull << kTallyMoreShift;
    if (ex > 0) {
      PersistCtl* c = a.pctl;
      const int pos = atomicAdd(&c->fcnt[bpar], 1);
      a.flist[(size_t)bpar * a.rctr_half + pos] = rep;
      atomicAdd(&c->ftiles[bpar], R.ntiles);
    }
  }
  // energies at run steps i with i % interval == 0, as Simulation.Run's
  // energies output schedule (Simulation.py:44, 587-589)
  if (R.energy_interval > 0 && (run_idx % R.energy_interval) == 0 && R.energy_cap > 0) {
    int k = nlog % R.energy_cap;
    double* e = a.elog + (size_t)(R.elog0 + k) * 5;
    e[0] = (double)run_idx; e[1] = pe; e[2] = vir; e[3] = tot[P_KET]; e[4] = xi;
    S->nlog = nlog + 1;
  }
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// finish_step for k_steps, run by the replica's finalizer after its
// step-barrier arrival: the same updates, except that the rebuild flag is
// raised by the blocks themselves (and cleared by the list build) and the
// loop tallies go with the arrivals.  The step count is stored last, with
// release: the next step's blocks wait for it before they integrate.
__device__ void finish_step_persist(const EngArgs& a, const RepDev& R, RepState* S, const double* tot) {
  if (threadIdx.x != 0) return;
  const double T0 = __ldcg(&S->T), dT = __ldcg(&S->dT), xi0 = __ldcg(&S->xi);
  const long long run_idx = __ldcg(&S->run_step);
  const long long steps = __ldcg(&S->steps), left = __ldcg(&S->steps_left);
  const int rbuf = __ldcg(&S->rbuf), nlog = __ldcg(&S->nlog);
  double xi = xi0, T = T0;
  if (R.thermo_mask) {
    double dev = tot[P_KE2] / (R.dof * T0) - 1.0;
    if (dev > 10.0) dev = 10.0;  // updateNVTThermostatState (IntegratorNVT.cu:426-437)
    xi = xi0 + (double)R.dt * (double)R.omega2 * dev;
    T = T0 + dT;
  }
  S->xi = xi;
  S->T = T;
  S->ke2 = tot[P_KE2];
  S->ke_t = tot[P_KET];
  const double pe = tot[P_PE], vir = tot[P_W] / 6.0;
  S->pe = pe;
  S->vir = vir;
  S->P[0] = tot[P_PX]; S->P[1] = tot[P_PY]; S->P[2] = tot[P_PZ]; S->M = tot[P_M];
  S->rbuf = rbuf ^ 1;
  S->run_step = run_idx + 1;
  if (left > 0) S->steps_left = left - 1;
  if (R.energy_interval > 0 && (run_idx % R.energy_interval) == 0 && R.energy_cap > 0) {
    int k = nlog % R.energy_cap;
    double* e = a.elog + (size_t)(R.elog0 + k) * 5;
    e[0] = (double)run_idx; e[1] = pe; e[2] = vir; e[3] = tot[P_KET]; e[4] = xi;
    S->nlog = nlog + 1;
  }
  st_release_u64(reinterpret_cast<unsigned long long*>(&S->steps), (unsigned long long)(steps + 1));
}

// ---------------------------------------------------------------------------
// Pair force (+ fused integration).  FUSED = one MD step: forces from r[rbuf],
// integrate, write r[rbuf^1].  Otherwise Sample::CalcF only.
// ---------------------------------------------------------------------------
// Per-thread force accumulators of one particle.  The stress terms are
// fij's FP32 products (PairPotential.h:1232-1241) summed in FP64: a
// particle's six components cancel strongly over its neighbours, and FP32
// sums of them lose about 1e-5 (stresses are computed only on request,
// never in the fused step).
struct PairAcc {
  float fx = 0.f, fy = 0.f, fz = 0.f, uu = 0.f, ww = 0.f;
  double sxx = 0.0, syy = 0.0, szz = 0.0, syz = 0.0, sxz = 0.0, sxy = 0.0;
};

// The pair rows of particle i's type, looked up by the neighbour's type.
//   RowsShared  the packed rows in shared memory: any pair function, any
//               number of types;
//   RowsLJ<NT>  the LJ 12-6 rows (rc^2, A12, A6, c_s, c_u0) of a replica with
//               NT = 1 or 2 types, held in registers: no lookup (NT = 1) or a
//               select (NT = 2), which keeps the table reads off the L1 data
//               pipe that the neighbour gathers use.
struct RowsShared {
  const float* prow;
  __device__ __forceinline__ const float* row(int tj) const { return prow + tj * kParStride; }
  __device__ __forceinline__ void lj(int tj, float4& q, float& cu0) const {
    const float* pp = row(tj);
    q = *reinterpret_cast<const float4*>(pp);
    cu0 = pp[4];
  }
};

template <int NT>
struct RowsLJ {
  float4 q0, q1;
  float c0, c1;
  __device__ __forceinline__ explicit RowsLJ(const float* prow) {
    q0 = *reinterpret_cast<const float4*>(prow);
    c0 = prow[4];
    if (NT == 2) {
      q1 = *reinterpret_cast<const float4*>(prow + kParStride);
      c1 = prow[kParStride + 4];
    } else {
      q1 = q0;
      c1 = c0;
    }
  }
  __device__ __forceinline__ const float* row(int) const { return nullptr; }
  __device__ __forceinline__ void lj(int tj, float4& q, float& cu0) const {
    if (NT == 1) {
      q = q0;
      cu0 = c0;
    } else {
      const bool b = tj != 0;
      q = make_float4(b ? q1.x : q0.x, b ? q1.y : q0.y, b ? q1.z : q0.z, b ? q1.w : q0.w);
      cu0 = b ? c1 : c0;
    }
  }
};

// fij (PairPotential.h:1198-1244) for one neighbour, without branches so
// that consecutive pairs interleave, for the pair function POT:
//   POT_LJ_12_6            Pot_IPL_12_6 / Pot_LJ_12_6::ComputeInteraction
//                          (PairPotential.h:161-168)
//   POT_LJ_12_6_SMOOTH_2_4 Pot_LJ_12_6_smooth_2_4::ComputeInteraction
//                          (PairPotential.h:248-255)
//   POT_IPL_N              Pot_IPL_n::ComputeInteraction (PairPotential.h:630-636)
// 1/r comes from one MUFU rsqrt refined by one Newton-Raphson step
// (y <- y (3/2 - x y^2 / 2)); 1/r^2 = y^2.  The cut-off method is folded into
// the packed pair row: s -= c_s / r and u += c_s r + c_u0, which is
// s(rc) rc / r and s(rc) rc (r - rc) - u(rc) for SF, -u(rc) for SP, 0 for NS.
// WRAP = false skips the minimum-image step; the caller uses it only when it
// is exactly the identity (see k_force).
template <bool STRESS, bool WRAP, int POT, class Rows>
__device__ __forceinline__ void lj_pair(PairAcc& A, const float4& ri, const float4& rj, const Rows& rows, float Lx,
                                        float Ly, float Lz, float iLx, float iLy, float iLz) {
  float dx = ri.x - rj.x, dy = ri.y - rj.y, dz = ri.z - rj.z;
  if (WRAP) {
    dx = mi_comp(dx, Lx, iLx);
    dy = mi_comp(dy, Ly, iLy);
    dz = mi_comp(dz, Lz, iLz);
  }
  const float d2 = dist2_ref(dx, dy, dz);
  const int tj = __float_as_int(rj.w);
  float y = rsqrt_approx(d2);
  y = y * __fmaf_rn(-0.5f * d2 * y, y, 1.5f);
  const float i2 = y * y;
  float s, u;
  bool in;
  if constexpr (POT == POT_LJ_12_6) {
    float4 q;  // rc^2, A12, A6, c_s (= c_ur)
    float cu0;
    rows.lj(tj, q, cu0);
    const float i6 = i2 * i2 * i2;
    const float t = q.y * i6;
    s = __fmaf_rn(-q.w, y, i6 * i2 * __fmaf_rn(12.f, t, 6.f * q.z));
    u = __fmaf_rn(i6, t + q.z, __fmaf_rn(q.w, d2 * y, cu0));
    in = d2 < q.x;
  } else if constexpr (POT == POT_LJ_12_6_SMOOTH_2_4) {
    const float* pp = rows.row(tj);
    const float4 q = *reinterpret_cast<const float4*>(pp);       // rc^2, sigma^2, 4 eps, b
    const float4 q1 = *reinterpret_cast<const float4*>(pp + 4);  // c, e, -, g
    const float2 q2 = *reinterpret_cast<const float2*>(pp + 8);  // c_s, c_u0
    const float t2 = q.y * i2;  // (sigma / r)^2
    const float t6 = t2 * t2 * t2;
    s = __fmaf_rn(-q2.x, y, __fmaf_rn(q1.x, d2, __fmaf_rn(q.z * i2 * t6, __fmaf_rn(12.f, t6, -6.f), q.w)));
    u = __fmaf_rn(q.z * t6, t6 - 1.f, __fmaf_rn(d2, __fmaf_rn(q1.w, d2, q1.y), __fmaf_rn(q2.x, d2 * y, q2.y)));
    in = d2 < q.x;
  } else {
    const float* pp = rows.row(tj);
    const float4 q = *reinterpret_cast<const float4*>(pp);       // rc^2, sigma^2, eps, n/2
    const float ne = pp[4];                                       // n eps
    const float2 q2 = *reinterpret_cast<const float2*>(pp + 8);  // c_s, c_u0
    const float tn = expf(logf(q.y * i2) * q.w);                 // (sigma / r)^n
    s = __fmaf_rn(-q2.x, y, ne * tn * i2);
    u = __fmaf_rn(q.z, tn, __fmaf_rn(q2.x, d2 * y, q2.y));
    in = d2 < q.x;
  }
  s = in ? s : 0.f;
  u = in ? u : 0.f;
  A.fx = __fmaf_rn(dx, s, A.fx);
  A.fy = __fmaf_rn(dy, s, A.fy);
  A.fz = __fmaf_rn(dz, s, A.fz);
  A.ww = __fmaf_rn(d2, s, A.ww);
  A.uu += u;
  if (STRESS) {
    A.sxx -= (double)(dx * dx * s); A.syy -= (double)(dy * dy * s); A.szz -= (double)(dz * dz * s);
    A.syz -= (double)(dy * dz * s); A.sxz -= (double)(dx * dz * s); A.sxy -= (double)(dx * dy * s);
  }
}

// One list entry, read once: streamed past L1 so that L1 keeps the gathered
// neighbour positions (which neighbouring particles share).
__device__ __forceinline__ unsigned ld_stream(const unsigned* p) {
  unsigned v;
  asm volatile("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ unsigned ld_stream_u16(const unsigned short* p) {
  unsigned short v;
  asm volatile("ld.global.nc.L1::no_allocate.u16 %0, [%1];" : "=h"(v) : "l"(p));
  return v;
}

__device__ __forceinline__ uint4 ld_stream_v4(const unsigned* p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}

__device__ __forceinline__ uint2 ld_stream_v2(const unsigned* p) {
  uint2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
  return v;
}

// The list entries one of a particle's TP lanes handles: with E = 8/TP, lane
// t takes entries 8m + E t + (0 .. E-1) of every block m of 8, so its q-th
// entry is lane_entry(q).  Four consecutive q (q a multiple of 4) are one
// 16-byte run of a block when E >= 4, two 8-byte runs when E = 2, and four
// single entries when E = 1.
template <int TP>
__device__ __forceinline__ unsigned lane_entry(unsigned q, unsigned t) {
  constexpr unsigned E = 8 / TP;
  return 8u * (q / E) + E * t + q % E;
}

// The number of this lane's entries below nn.
template <int TP>
__device__ __forceinline__ unsigned lane_count(unsigned nn, unsigned t) {
  constexpr int E = 8 / TP;
  const int rem = (int)(nn & 7u) - E * (int)t;
  return (nn >> 3) * (unsigned)E + (unsigned)min(E, max(0, rem));
}

// List-entry readers for force_loop: one(k) is entry k of the particle;
// group<TP>(q, t) is lane t's entries q .. q+3 (q a multiple of 4).
// Streamed: read from the global list inside the loop, past L1.
struct IdxStreamed {
  const unsigned* base;  // the replica's list
  unsigned i;            // the particle's slot
  size_t stride;
  __device__ __forceinline__ unsigned one(unsigned k) const { return ld_stream(base + lpos(k, i, stride)); }
  template <int TP>
  __device__ __forceinline__ uint4 group(unsigned q, unsigned t) const {
    constexpr unsigned E = 8 / TP;
    if (E >= 4) return ld_stream_v4(base + lpos(lane_entry<TP>(q, t), i, stride));
    if (E == 2) {
      const uint2 a = ld_stream_v2(base + lpos(lane_entry<TP>(q, t), i, stride));
      const uint2 b = ld_stream_v2(base + lpos(lane_entry<TP>(q + 2, t), i, stride));
      return make_uint4(a.x, a.y, b.x, b.y);
    }
    return make_uint4(one(lane_entry<TP>(q, t)), one(lane_entry<TP>(q + 1, t)), one(lane_entry<TP>(q + 2, t)),
                      one(lane_entry<TP>(q + 3, t)));
  }
};
// Streamed through L2 only (ld.global.cg): for kernels that rewrite the
// list while they run (k_batch builds lists and reads them in one launch),
// where the read-only path may not see those writes.
__device__ __forceinline__ unsigned ld_cg_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint2 ld_cg_v2(const unsigned* p) {
  uint2 v;
  asm volatile("ld.global.cg.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ uint4 ld_cg_v4(const unsigned* p) {
  uint4 v;
  asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}
struct IdxStreamedCg {
  const unsigned* base;
  unsigned i;
  size_t stride;
  __device__ __forceinline__ unsigned one(unsigned k) const { return ld_cg_u32(base + lpos(k, i, stride)); }
  template <int TP>
  __device__ __forceinline__ uint4 group(unsigned q, unsigned t) const {
    constexpr unsigned E = 8 / TP;
    if (E >= 4) return ld_cg_v4(base + lpos(lane_entry<TP>(q, t), i, stride));
    if (E == 2) {
      const uint2 a = ld_cg_v2(base + lpos(lane_entry<TP>(q, t), i, stride));
      const uint2 b = ld_cg_v2(base + lpos(lane_entry<TP>(q + 2, t), i, stride));
      return make_uint4(a.x, a.y, b.x, b.y);
    }
    return make_uint4(one(lane_entry<TP>(q, t)), one(lane_entry<TP>(q + 1, t)), one(lane_entry<TP>(q + 2, t)),
                      one(lane_entry<TP>(q + 3, t)));
  }
};
// A position through L1 with a plain (coherent) load, for data the running
// kernel itself rewrites.
__device__ __forceinline__ float4 ld_ca_f4(const float4* p) {
  float4 v;
  asm volatile("ld.global.ca.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}

// Staged: the tile's list blocks copied to shared memory, block b of slot lp
// at p[(b * pb + lp) * 8]; p points at this particle's first block.
struct IdxStaged {
  const unsigned* p;
  int bstride;  // pb * 8
  __device__ __forceinline__ unsigned one(unsigned k) const { return p[(k >> 3) * bstride + (k & 7u)]; }
  template <int TP>
  __device__ __forceinline__ uint4 group(unsigned q, unsigned t) const {
    constexpr unsigned E = 8 / TP;
    if (E >= 4) {
      const unsigned k = lane_entry<TP>(q, t);
      return *reinterpret_cast<const uint4*>(p + (k >> 3) * bstride + (k & 7u));
    }
    if (E == 2) {
      const unsigned k0 = lane_entry<TP>(q, t), k1 = lane_entry<TP>(q + 2, t);
      const uint2 a = *reinterpret_cast<const uint2*>(p + (k0 >> 3) * bstride + (k0 & 7u));
      const uint2 b = *reinterpret_cast<const uint2*>(p + (k1 >> 3) * bstride + (k1 & 7u));
      return make_uint4(a.x, a.y, b.x, b.y);
    }
    return make_uint4(one(lane_entry<TP>(q, t)), one(lane_entry<TP>(q + 1, t)), one(lane_entry<TP>(q + 2, t)),
                      one(lane_entry<TP>(q + 3, t)));
  }
};
// Window: the 16-bit window list (offsets into the tile's position window),
// in the list's layout.
struct IdxWindow {
  const unsigned short* base;
  unsigned i;
  size_t stride;
  __device__ __forceinline__ unsigned one(unsigned k) const { return ld_stream_u16(base + lpos(k, i, stride)); }
  template <int TP>
  __device__ __forceinline__ uint4 group(unsigned q, unsigned t) const {
    constexpr unsigned E = 8 / TP;
    if (E >= 4) {
      // four 16-bit entries = 8 bytes
      const uint2 w = ld_stream_v2(reinterpret_cast<const unsigned*>(base + lpos(lane_entry<TP>(q, t), i, stride)));
      return make_uint4(w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16);
    }
    if (E == 2) {
      const unsigned a = ld_stream(reinterpret_cast<const unsigned*>(base + lpos(lane_entry<TP>(q, t), i, stride)));
      const unsigned b =
          ld_stream(reinterpret_cast<const unsigned*>(base + lpos(lane_entry<TP>(q + 2, t), i, stride)));
      return make_uint4(a & 0xffffu, a >> 16, b & 0xffffu, b >> 16);
    }
    return make_uint4(one(lane_entry<TP>(q, t)), one(lane_entry<TP>(q + 1, t)), one(lane_entry<TP>(q + 2, t)),
                      one(lane_entry<TP>(q + 3, t)));
  }
};

// Window, staged: the tile's 16-bit window-list blocks copied to shared
// memory, block b of slot lp at p[(b * pb + lp) * 8]; p points at this
// particle's first block.
struct IdxWindowStaged {
  const unsigned short* p;
  int bstride;  // pb * 8
  __device__ __forceinline__ unsigned one(unsigned k) const { return p[(k >> 3) * bstride + (k & 7u)]; }
  template <int TP>
  __device__ __forceinline__ uint4 group(unsigned q, unsigned t) const {
    constexpr unsigned E = 8 / TP;
    if (E >= 4) {
      const unsigned k = lane_entry<TP>(q, t);
      const uint2 w = *reinterpret_cast<const uint2*>(p + (k >> 3) * bstride + (k & 7u));
      return make_uint4(w.x & 0xffffu, w.x >> 16, w.y & 0xffffu, w.y >> 16);
    }
    if (E == 2) {
      const unsigned k0 = lane_entry<TP>(q, t), k1 = lane_entry<TP>(q + 2, t);
      const unsigned a = *reinterpret_cast<const unsigned*>(p + (k0 >> 3) * bstride + (k0 & 7u));
      const unsigned b = *reinterpret_cast<const unsigned*>(p + (k1 >> 3) * bstride + (k1 & 7u));
      return make_uint4(a & 0xffffu, a >> 16, b & 0xffffu, b >> 16);
    }
    return make_uint4(one(lane_entry<TP>(q, t)), one(lane_entry<TP>(q + 1, t)), one(lane_entry<TP>(q + 2, t)),
                      one(lane_entry<TP>(q + 3, t)));
  }
};

// Neighbour-position readers: gathered from global memory (through L1), or
// from the tile's position window in shared memory.
struct PosGlobal {
  const float4* __restrict__ p;
  __device__ __forceinline__ float4 operator()(unsigned j) const { return __ldg(p + j); }
};
// Positions that other blocks of the same launch rewrite (k_steps): plain
// L1-cached loads (no __restrict__, so never the read-only path), ordered
// after the step barrier's acquire.
struct PosCoherent {
  const float4* p;
  __device__ __forceinline__ float4 operator()(unsigned j) const { return p[j]; }
};
template <bool B, class T, class F> struct Pick { using type = T; };
template <class T, class F> struct Pick<false, T, F> { using type = F; };

struct PosWindow {
  const float4* p;
  __device__ __forceinline__ float4 operator()(unsigned j) const { return p[j]; }
};

// The neighbour loop of one thread: its entries (lane_entry) in groups of
// four -- one vector load of list entries, four neighbour positions in
// flight -- then the remaining ones singly.  Only entries below nn are read.
template <int TP, bool STRESS, bool WRAP, int POT, class Idx, class Pos, class Rows>
__device__ __forceinline__ void force_loop(PairAcc& A, const Idx& idx, const Pos& pos, unsigned lane_t, unsigned nn,
                                           const float4& ri, const Rows& prow, float Lx, float Ly, float Lz,
                                           float iLx, float iLy, float iLz) {
  const unsigned cnt = lane_count<TP>(nn, lane_t);
  unsigned q = 0;
  for (; q + 4 <= cnt; q += 4) {
    const uint4 j = idx.template group<TP>(q, lane_t);
    const float4 r0 = pos(j.x), r1 = pos(j.y), r2 = pos(j.z), r3 = pos(j.w);
    lj_pair<STRESS, WRAP, POT>(A, ri, r0, prow, Lx, Ly, Lz, iLx, iLy, iLz);
    lj_pair<STRESS, WRAP, POT>(A, ri, r1, prow, Lx, Ly, Lz, iLx, iLy, iLz);
    lj_pair<STRESS, WRAP, POT>(A, ri, r2, prow, Lx, Ly, Lz, iLx, iLy, iLz);
    lj_pair<STRESS, WRAP, POT>(A, ri, r3, prow, Lx, Ly, Lz, iLx, iLy, iLz);
  }
  for (; q < cnt; ++q) {
    const float4 r0 = pos(idx.one(lane_entry<TP>(q, lane_t)));
    lj_pair<STRESS, WRAP, POT>(A, ri, r0, prow, Lx, Ly, Lz, iLx, iLy, iLz);
  }
}

// The loop for the replica's pair function and type count (block-uniform)
// and minimum-image need.  REG: single-type LJ 12-6 replicas hold their row
// in registers (3.5 % faster at N = 1M; for two types the selects cost more
// than the shared-memory lookups they replace, 40.2 vs 37.6 us at KA 65536).
template <int TP, bool STRESS, bool REG, class Idx, class Pos>
__device__ __forceinline__ void force_loop_any(bool fast, int pot, int nt, PairAcc& A, const Idx& idx, const Pos& pos,
                                               unsigned lane_t, unsigned nn, const float4& ri, const float* prow,
                                               float Lx, float Ly, float Lz, float iLx, float iLy, float iLz) {
#define FL(W, P, ROWS) force_loop<TP, STRESS, W, P>(A, idx, pos, lane_t, nn, ri, ROWS, Lx, Ly, Lz, iLx, iLy, iLz)
  const RowsShared sh{prow};
  if (pot == POT_LJ_12_6) {
    if (REG && nt == 1) {
      const RowsLJ<1> rg(prow);
      if (fast) FL(false, POT_LJ_12_6, rg);
      else FL(true, POT_LJ_12_6, rg);
    } else {
      if (fast) FL(false, POT_LJ_12_6, sh);
      else FL(true, POT_LJ_12_6, sh);
    }
  } else if (pot == POT_LJ_12_6_SMOOTH_2_4) {
    if (fast) FL(false, POT_LJ_12_6_SMOOTH_2_4, sh);
    else FL(true, POT_LJ_12_6_SMOOTH_2_4, sh);
  } else {
    if (fast) FL(false, POT_IPL_N, sh);
    else FL(true, POT_IPL_N, sh);
  }
#undef FL
}

// Shared memory of k_force: [packed pair table, kParSmemFloats]
// [MODE 1: list tile | MODE 2: position window, win_cap float4]; after the
// neighbour loop the block reduction's scratch (force_red_bytes) overlays it.
constexpr int kParSmemFloats = kMaxTypes * kMaxTypes * kParStride;
__host__ __device__ constexpr int force_red_bytes(int threads) {
  return ((threads + 31) / 32) * kNPart * (int)sizeof(double) + threads * (int)sizeof(double);
}
// k_steps keeps the pair table (of the engine's largest type count) at the
// start of its dynamic shared memory; the reduction scratch follows it.
__host__ __device__ inline int persist_table_bytes(const EngArgs& a) {
  return (a.max_types * a.max_types * kParStride * (int)sizeof(float) + 15) & ~15;
}
constexpr unsigned kWaitPolls = 1u << 22;

enum { FM_STREAMED = 0, FM_STAGED = 1, FM_WINDOW = 2 };

// One tile of pb particles per block, tp threads per particle.  MODE selects
// how the neighbours are read:
//   FM_STREAMED  list entries and neighbour positions read from global memory
//                inside the loop (positions through L1);
//   FM_STAGED    the tile's list rows copied to shared memory first (TMA bulk
//                copies), positions gathered from global memory;
//   FM_WINDOW    the tile's position window (every slot segment holding a
//                listed neighbour of the tile) copied to shared memory with one
//                TMA bulk copy per segment, and the 16-bit window list read
//                from global memory: every neighbour position comes from shared
//                memory.  Tiles without a window (wmeta < 0) stream.
// One tile of the force kernels (see k_force).  PERSIST: inside k_steps,
// where other blocks rewrite positions and replica state between steps of
// the same launch, so those are read through coherent loads (no read-only
// path) and the state fields past L1.
// The replica-state fields a step reads.  In k_steps the previous step's
// finalizer (on another SM) wrote them, so thread 0 reads them past L1 once
// per tile and the block shares them through shared memory.
struct StepView {
  int overflow, rbuf, abuf, first;  // first: the tile's first slot
  long long steps_left, run_step, steps;
  double M, P[3], xi;
};

__device__ __forceinline__ void load_view(StepView& v, const RepState* S) {
  v.overflow = __ldcg(&S->overflow);
  v.rbuf = __ldcg(&S->rbuf);
  v.abuf = __ldcg(&S->abuf);
  v.steps_left = __ldcg(&S->steps_left);
  v.run_step = __ldcg(&S->run_step);
  v.steps = __ldcg(&S->steps);
  v.M = __ldcg(&S->M);
  v.P[0] = __ldcg(&S->P[0]);
  v.P[1] = __ldcg(&S->P[1]);
  v.P[2] = __ldcg(&S->P[2]);
  v.xi = __ldcg(&S->xi);
}

// Per-thread state that k_steps keeps in registers for a launch (no rebuild,
// hence no re-sort, happens inside one): the particle's list length and, in
// its integrating thread, the velocity, image counts and build-time position.
struct PersistRegs {
  float4 v, lr;
  int4 im;
  unsigned nn;
};

// COH (k_batch): positions and lists that the same launch rewrites are read
// with coherent loads (no read-only path); bpar: the batch rebuild-list parity
// passed to finish_step.
template <int TP, bool FUSED, bool STRESS, int MODE, bool PERSIST, bool COH = false>
__device__ __forceinline__ bool force_tile(const EngArgs& a, int tile, unsigned char* s_dyn, double* s_blk,
                                           double* s_tot, uint64_t& s_bar, unsigned& s_rows,
                                           const StepView* pv = nullptr, int gpar = 0,
                                           const RepDev* prep = nullptr, PersistRegs* pr = nullptr,
                                           unsigned* wdone = nullptr, int bpar = -1) {
  float* s_par = reinterpret_cast<float*>(s_dyn);
  unsigned* s_idx = reinterpret_cast<unsigned*>(s_dyn + kParSmemFloats * sizeof(float));
  float4* s_win = reinterpret_cast<float4*>(s_dyn + kParSmemFloats * sizeof(float));
  unsigned short* s_wl = reinterpret_cast<unsigned short*>(s_win + a.win_cap);  // mode 2: staged window list
  // the block reduction's scratch reuses the start of the dynamic region once
  // every thread is past the neighbour loop (force_red_bytes); in k_steps it
  // follows the pair table, which stays loaded for the whole launch
  double* s_warp = reinterpret_cast<double*>(s_dyn + (PERSIST ? persist_table_bytes(a) : 0));
  double* s_scr = s_warp + (blockDim.x >> 5) * kNPart;
  const int rep = a.tile_rep[tile];
  // PERSIST: k_steps' shared-memory copy of the replica's descriptor
  const RepDev& R = PERSIST ? *prep : a.rep[rep];
  RepState* S = a.st + rep;
  // PERSIST: the block's view of its replica's state, kept by k_steps
  // (the buffer parity, step counters); xi and the momentum come from the
  // previous step's finalizer just before the integration
  __shared__ double s_xi, s_M, s_P[3];
#define SV(f) (PERSIST ? pv->f : S->f)
  const bool skip = (SV(overflow) != 0) || (FUSED && SV(steps_left) <= 0) || !R.active;
  if (!skip) {
    const int pb = blockDim.x / TP;
    const int first = PERSIST ? pv->first : a.tile_first[tile];
    const int pitch = a.idx_pitch;
    const int rb = SV(rbuf);
    const float4* rc = a.r[rb] + R.p0;
    const int2 wm = MODE == FM_WINDOW ? a.wmeta[tile] : make_int2(-1, -1);
    const bool use_bar = MODE == FM_STAGED || (MODE == FM_WINDOW && wm.x >= 0);
    if (use_bar) {
      if (threadIdx.x == 0) {
        s_rows = 0u;
        mbar_init(&s_bar, 1);
        mbar_fence_init();
      }
      __syncthreads();
    }
    if (MODE == FM_STAGED || (MODE == FM_WINDOW && wm.x >= 0 && a.wl_rows > 0)) {
      // 1. rows of the list this tile needs: the largest neighbour count in it
      {
        unsigned c = (threadIdx.x < pb && first + (int)threadIdx.x < R.n) ? a.nn[R.p0 + first + threadIdx.x] : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
        if ((threadIdx.x & 31) == 0 && c) atomicMax(&s_rows, c);
      }
      __syncthreads();
    }
    bool wl_staged = false;
    if (MODE == FM_STAGED) {
      const unsigned rows = min(s_rows, (unsigned)a.idx_rows);
      // 2. one TMA bulk copy per list block of 8 entries: slots [first, first+width)
      //    of blocks 0 .. ceil(rows/8)-1, each a contiguous run of width*32 bytes
      if (threadIdx.x < 32) {
        const unsigned width = (unsigned)min(pb, R.nbl_stride - first);
        const unsigned nblk = (rows + 7u) >> 3;
        if (threadIdx.x == 0) mbar_arrive_expect_tx(&s_bar, nblk * width * 32u);
        __syncwarp();
        const unsigned* src = a.nbl + R.nbl0 + (size_t)first * 8;
        for (unsigned b = threadIdx.x; b < nblk; b += 32)
          bulk_g2s(s_idx + b * pitch * 8, src + (size_t)b * R.nbl_stride * 8, width * 32u, &s_bar);
      }
    } else if (MODE == FM_WINDOW && wm.x >= 0) {
      // 1-2. one TMA bulk copy per window segment (16-byte aligned float4 runs),
      //      and, when the tile's list fits the staged rows, one per block of 8
      //      window-list entries (width*16 bytes)
      const unsigned wrows = a.wl_rows > 0 ? s_rows : 0u;
      wl_staged = a.wl_rows > 0 && wrows <= (unsigned)a.wl_rows;
      if (threadIdx.x < 32) {
        const unsigned width = (unsigned)min(pb, R.nbl_stride - first);
        const unsigned nblk = wl_staged ? (wrows + 7u) >> 3 : 0u;
        if (threadIdx.x == 0) mbar_arrive_expect_tx(&s_bar, (unsigned)wm.y * 16u + nblk * width * 16u);
        __syncwarp();
        const int4* seg = a.wseg + (size_t)tile * kWinSeg;
        for (int sgi = threadIdx.x; sgi < wm.x; sgi += 32) {
          const int4 sg = seg[sgi];
          bulk_g2s(s_win + sg.z, rc + sg.x, (unsigned)sg.y * 16u, &s_bar);
        }
        const unsigned short* src = a.wl + R.nbl0 + (size_t)first * 8;
        for (unsigned b = threadIdx.x; b < nblk; b += 32)
          bulk_g2s(s_wl + b * pitch * 8, src + (size_t)b * R.nbl_stride * 8, width * 16u, &s_bar);
      }
    }
    // 3. meanwhile: pair table and this particle's data
    const int nt = R.ntypes;
    if (!PERSIST)
      for (int k = threadIdx.x; k < nt * nt * kParStride; k += blockDim.x) s_par[k] = a.par[R.par0 + k];
    const int lp = threadIdx.x / TP, lane_t = threadIdx.x % TP;
    const int i = first + lp;
    const bool valid = i < R.n;
    const float Lx = R.L[0], Ly = R.L[1], Lz = R.L[2];
    const float iLx = R.invL[0], iLy = R.invL[1], iLz = R.invL[2];
    const float4 ri = valid ? ((PERSIST || COH) ? rc[i] : __ldg(rc + i)) : make_float4(0.f, 0.f, 0.f, 0.f);
    const int ti = valid ? __float_as_int(ri.w) : 0;
    const float* prow = s_par + ti * nt * kParStride;
    const unsigned nn = valid ? (PERSIST ? pr->nn : a.nn[R.p0 + i]) : 0u;
    const size_t lstride = (size_t)R.nbl_stride;
    const unsigned* lbase = a.nbl + R.nbl0;
    const unsigned short* wbase = a.wl + R.nbl0;
    // A particle farther than rc_max + 2 skin from every face of the box has
    // all its listed neighbours (within rc + skin at the build, each moved at
    // most skin/2 since) inside the box at their minimum image, so the
    // minimum-image correction is exactly zero; warps made only of such
    // particles skip it.
    const bool inner = fabsf(ri.x) < R.ilim[0] && fabsf(ri.y) < R.ilim[1] && fabsf(ri.z) < R.ilim[2];
    const bool fast = __all_sync(0xffffffffu, !valid || inner);
    PairAcc A;
    if (use_bar) {
      // 4. bounded wait for the copies (the barrier also publishes the pair table)
      const bool ok = __syncthreads_and(mbar_wait_bounded(&s_bar, 0, kWaitPolls));
      if (ok) {
        if (MODE == FM_STAGED)
          force_loop_any<TP, STRESS, false>(fast, R.potential, nt, A, IdxStaged{s_idx + lp * 8, pitch * 8}, PosGlobal{rc}, lane_t, nn, ri, prow,
                                     Lx, Ly, Lz, iLx, iLy, iLz);
        else if (wl_staged)
          force_loop_any<TP, STRESS, false>(fast, R.potential, nt, A, IdxWindowStaged{s_wl + lp * 8, pitch * 8}, PosWindow{s_win}, lane_t, nn,
                                     ri, prow, Lx, Ly, Lz, iLx, iLy, iLz);
        else
          force_loop_any<TP, STRESS, false>(fast, R.potential, nt, A, IdxWindow{wbase, (unsigned)i, lstride}, PosWindow{s_win}, lane_t, nn, ri, prow,
                                     Lx, Ly, Lz, iLx, iLy, iLz);
      } else {
        // the copies did not land in time: record it for the host and wait
        // (bounded) for them before this block's shared memory is released
        if (threadIdx.x == 0) atomicExch(&S->err, 1);
        mbar_wait_bounded(&s_bar, 0, kWaitPolls);
      }
    } else {
      if (!PERSIST) __syncthreads();  // the pair table (k_steps loads it once per launch)
      using PosS = typename Pick<PERSIST || COH, PosCoherent, PosGlobal>::type;
      using IdxS = typename Pick<COH, IdxStreamedCg, IdxStreamed>::type;
      force_loop_any<TP, STRESS, true>(fast, R.potential, nt, A, IdxS{lbase, (unsigned)i, lstride}, PosS{rc}, lane_t, nn,
                                       ri, prow, Lx, Ly, Lz, iLx, iLy, iLz);
    }
    float fx = A.fx, fy = A.fy, fz = A.fz, uu = A.uu, ww = A.ww;
    double sxx = A.sxx, syy = A.syy, szz = A.szz, syz = A.syz, sxz = A.sxz, sxy = A.sxy;
    if (TP > 1) {
#pragma unroll
      for (int o = TP / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        uu += __shfl_xor_sync(0xffffffffu, uu, o);
        ww += __shfl_xor_sync(0xffffffffu, ww, o);
        if (STRESS) {
          sxx += __shfl_xor_sync(0xffffffffu, sxx, o);
          syy += __shfl_xor_sync(0xffffffffu, syy, o);
          szz += __shfl_xor_sync(0xffffffffu, szz, o);
          syz += __shfl_xor_sync(0xffffffffu, syz, o);
          sxz += __shfl_xor_sync(0xffffffffu, sxz, o);
          sxy += __shfl_xor_sync(0xffffffffu, sxy, o);
        }
      }
    }
    if constexpr (!PERSIST && !COH) {
      if (R.npot > 1) {
        // Sample::CalcF's potential loop (Sample.cu:335-336): the second
        // pair function's per-particle sums, over the same list (read from
        // global memory in every force mode), are added to the first's once
        // both are complete -- the store-then-accumulate of
        // PairPotential.cu:370-388
        PairAcc B;
        const float* prow1 = a.par + R.par1 + ti * nt * kParStride;
        force_loop_any<TP, STRESS, false>(fast, R.potential1, nt, B, IdxStreamed{lbase, (unsigned)i, lstride},
                                          PosGlobal{rc}, lane_t, nn, ri, prow1, Lx, Ly, Lz, iLx, iLy, iLz);
        if (TP > 1) {
#pragma unroll
          for (int o = TP / 2; o > 0; o >>= 1) {
            B.fx += __shfl_xor_sync(0xffffffffu, B.fx, o);
            B.fy += __shfl_xor_sync(0xffffffffu, B.fy, o);
            B.fz += __shfl_xor_sync(0xffffffffu, B.fz, o);
            B.uu += __shfl_xor_sync(0xffffffffu, B.uu, o);
            B.ww += __shfl_xor_sync(0xffffffffu, B.ww, o);
            if (STRESS) {
              B.sxx += __shfl_xor_sync(0xffffffffu, B.sxx, o);
              B.syy += __shfl_xor_sync(0xffffffffu, B.syy, o);
              B.szz += __shfl_xor_sync(0xffffffffu, B.szz, o);
              B.syz += __shfl_xor_sync(0xffffffffu, B.syz, o);
              B.sxz += __shfl_xor_sync(0xffffffffu, B.sxz, o);
              B.sxy += __shfl_xor_sync(0xffffffffu, B.sxy, o);
            }
          }
        }
        fx += B.fx; fy += B.fy; fz += B.fz; uu += B.uu; ww += B.ww;
        if (STRESS) {
          sxx += B.sxx; syy += B.syy; szz += B.szz; syz += B.syz; sxz += B.sxz; sxy += B.sxy;
        }
      }
    }
    if constexpr (PERSIST && FUSED) {
      // the block's first warp past its neighbour loop waits (bounded) for
      // the previous step's finalizer, which stores the step count last, with
      // release; the other warps are still in their loops meanwhile
      if ((threadIdx.x & 31u) == 0 && atomicAdd(wdone, 1u) == 0u) {
        const unsigned long long want = (unsigned long long)pv->steps;
        for (unsigned it = 0; ld_acquire_u64(reinterpret_cast<const unsigned long long*>(&S->steps)) < want; ++it) {
          if (it >= kWaitPolls) {
            atomicExch(&a.pctl->err, 1);
            break;
          }
          __nanosleep(32);
        }
        s_xi = __ldcg(&S->xi);
        s_M = __ldcg(&S->M);
        s_P[0] = __ldcg(&S->P[0]);
        s_P[1] = __ldcg(&S->P[1]);
        s_P[2] = __ldcg(&S->P[2]);
      }
      __syncthreads();
    }
#define SVS(f, pf) (PERSIST ? (pf) : S->f)
    double acc[kNPart];
#pragma unroll
    for (int k = 0; k < kNPart; ++k) acc[k] = 0.0;
    bool exceed = false;
    if (valid && lane_t == 0) {
      const float4 fo = make_float4(fx, fy, fz, 0.5f * uu);
      const size_t gi = (size_t)R.p0 + i;
      a.f[gi] = fo;
      a.w[gi] = make_float4(0.f, (float)sxz, (float)sxy, ww);
      if (STRESS) a.sts[gi] = make_float4((float)sxx, (float)syy, (float)szz, (float)syz);
      acc[P_PE] = (double)fo.w;
      acc[P_W] = (double)ww;
      if (FUSED) {
        const int ab = SV(abuf);
        float4 v = PERSIST ? pr->v : a.v[ab][gi];
        int4 im = PERSIST ? pr->im : a.im[ab][gi];
        const bool do_reset = R.reset_interval > 0 && (SV(run_step) % R.reset_interval) == 0;
        float3 vs = make_float3(0.f, 0.f, 0.f);
        const double M = SVS(M, s_M);
        if (do_reset && M > 0.0)
          vs = make_float3((float)(SVS(P[0], s_P[0]) / M), (float)(SVS(P[1], s_P[1]) / M),
                           (float)(SVS(P[2], s_P[2]) / M));
        float4 rn;
        integrate_one(R, (float)SVS(xi, s_xi), vs, do_reset, ri, fo, v, im, rn, acc, exceed,
                      PERSIST ? pr->lr : a.last_r[gi]);
        a.v[ab][gi] = v;
        a.im[ab][gi] = im;
        if (PERSIST) {
          pr->v = v;
          pr->im = im;
        }
        a.r[rb ^ 1][gi] = rn;
      }
    }
    // every thread is past the neighbour loop: the pair table (and the staged
    // tile) may be overwritten by the reduction scratch
    const int ex = __syncthreads_or(exceed);
    if constexpr (PERSIST) {
      // the rebuild request and "steps left" go with the block's arrival
      if (threadIdx.x == 0) {
        if (ex) S->rebuild = 1;
        s_step_tally += (ex ? (1ull << kTallyRebuildShift) : 0ull) +
                        (pv->steps_left > 1 ? (1ull << kTallyMoreShift) : 0ull);
      }
      // the tile's partial sums; k_steps reduces them after the block's
      // barrier arrival (the arrival releases them)
      block_sum8(acc, s_warp, s_blk);
      if (threadIdx.x < kNPart)
        a.tpart[(size_t)gpar * a.tpart_half + (size_t)tile * kNPart + threadIdx.x] = s_blk[threadIdx.x];
    } else {
      if (FUSED && ex && threadIdx.x == 0) atomicAdd(&S->exceed, 1);
      block_sum8(acc, s_warp, s_blk);
      if (replica_reduce(a, rep, R, tile - R.tile0, s_blk, s_scr, s_tot)) {
        if (FUSED) {
          finish_step(a, rep, R, S, s_tot, true, bpar);
        } else if (threadIdx.x == 0) {
          S->pe = s_tot[P_PE];
          S->vir = s_tot[P_W] / 6.0;
        }
      }
    }
#undef SVS
  }
#undef SV
  return !skip;
}

// One tile of pb particles per block, tp threads per particle.  MODE selects
// how the neighbours are read:
//   FM_STREAMED  list entries and neighbour positions read from global memory
//                inside the loop (positions through L1);
//   FM_STAGED    the tile's list rows copied to shared memory first (TMA bulk
//                copies), positions gathered from global memory;
//   FM_WINDOW    the tile's position window (every slot segment holding a
//                listed neighbour of the tile) copied to shared memory with one
//                TMA bulk copy per segment, and the 16-bit window list read
//                from global memory: every neighbour position comes from shared
//                memory.  Tiles without a window (wmeta < 0) stream.
template <int TP, bool FUSED, bool STRESS, int MODE>
__global__ void __launch_bounds__(kMaxBlock) k_force(EngArgs a, int has_cond, cudaGraphConditionalHandle h) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ double s_blk[kNPart], s_tot[kNPart];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ unsigned s_rows;
  __shared__ int s_tile;
  // SM tiles (streamed mode): a grid of at most as many blocks as fit at once;
  // each block claims tiles from its SM's region of the tile range, so the
  // tiles an SM processes are neighbours in space and share its L1
  const bool sm_tiles = MODE == FM_STREAMED && a.nreg > 0;
  int tile = blockIdx.x;
  for (;;) {
    if (sm_tiles) {
      __syncthreads();  // the previous tile is done with shared memory
      if (threadIdx.x < 32) {
        const int t = claim_tile(a);
        if (threadIdx.x == 0) s_tile = t;
      }
      __syncthreads();
      tile = s_tile;
      if (tile < 0) break;
    }
    force_tile<TP, FUSED, STRESS, MODE, false>(a, tile, s_dyn, s_blk, s_tot, s_bar, s_rows);
    if (!sm_tiles) break;
  }
  grid_final(a, has_cond, h);
}

// End of one step of k_steps: a grid barrier.  Every block arrives once its
// tiles are done (the replica finalizers after their finish_step); the last
// one to arrive resets the barrier and decides whether the launch goes on:
// not when a list rebuild is due (the graph's rebuild node runs first), the
// step budget of the graph launch is spent, or no replica has steps left; it
// then sets the graph's loop condition.  The others wait for the decision,
// at most kBarrierPolls polls; a wait that gives up records the error and
// ends the graph's loop, so every block returns.
constexpr unsigned kBarrierPolls = 1u << 22;  // > 0.25 s of 64 ns sleeps

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}

// The persistent loop's condition, when k_steps runs inside the step graph;
// an eager (profiling) launch passes a zero handle and the host decides.
__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle h, unsigned v) {
  if (h) cudaGraphSetConditional(h, v);
}

// Waits (bounded) until the grid barrier of generation gen is released;
// false when the wait gave up (recorded, and the graph's loop ended).
__device__ bool barrier_wait(PersistCtl* c, unsigned gen, cudaGraphConditionalHandle h_loop) {
  for (unsigned it = 0;; ++it) {
    if (ld_acquire_u32(&c->gen) != gen) break;
    if (it >= kBarrierPolls) {
      atomicExch(&c->err, 1);
      set_loop(h_loop, 0u);
      return false;
    }
    __nanosleep(64);
  }
  __threadfence();
  return true;
}

// Grid barrier at the start of k_steps; the last block to arrive zeroes the
// step-barrier words before it releases the others.
__device__ bool setup_barrier(const EngArgs& a, cudaGraphConditionalHandle h_loop) {
  PersistCtl* c = a.pctl;
  const unsigned gen = ld_acquire_u32(&c->gen);
  const unsigned long long n = atom_add_acq_rel_u64(&c->arrive, 1ull) + 1ull;
  if ((n & kTallyArriveMask) == gridDim.x) {
    c->arrive = 0ull;
    c->word[0] = 0ull;
    c->word[1] = 0ull;
    st_release_u32(&c->gen, gen + 1u);
    return true;
  }
  return barrier_wait(c, gen, h_loop);
}

// The step barrier needs no release step.  Steps alternate between two
// words (step s uses word[s & 1]); each word only grows during a launch (the
// setup barrier zeroes both).  A block adds, in one release/acquire atomic,
// its arrival (low 24 bits) and its finalizer's tallies (s_step_tally:
// replicas that still have steps, next 20 bits; rebuild requests, top 20),
// then polls the word until the step's arrivals are complete.  Nothing else
// can reach that word before every block has left this barrier (the next
// contributions to it come two steps later), so every block reads the same
// totals and takes the same decision: go on unless a rebuild is due, the
// budget (counted down by every block alike) is spent, no replica has steps
// left, or the launch has run kMaxLaunchSteps steps (the words' fields would
// otherwise carry).  The block whose arrival completed the step sets the
// graph's loop condition and, when stopping, the budget of the next launch.
// seen[w]: the totals of word w at its previous barrier.
constexpr int kMaxLaunchSteps = 4096;

__device__ unsigned long long step_arrive(const EngArgs& a, int step) {
  const unsigned long long mine = 1ull + s_step_tally;
  return atom_add_acq_rel_u64(&a.pctl->word[step & 1], mine) + mine;
}

__device__ int step_decide(const EngArgs& a, int step, int budget, unsigned long long* seen, unsigned long long now,
                           cudaGraphConditionalHandle h_loop) {
  PersistCtl* c = a.pctl;
  const int w = step & 1;
  const unsigned long long base = seen[w];
  const bool last = ((now - base) & kTallyArriveMask) == gridDim.x;
  if (!last) {
    for (unsigned it = 0;; ++it) {
      now = ld_acquire_u64(&c->word[w]);
      if (((now - base) & kTallyArriveMask) == gridDim.x) break;
      if (it >= kBarrierPolls) {
        atomicExch(&c->err, 1);
        set_loop(h_loop, 0u);
        return 0;
      }
      __nanosleep(32);
    }
  }
  seen[w] = now;
  const unsigned long long d = now - base;
  const unsigned more = (unsigned)((d >> kTallyMoreShift) & kTallyField);
  const unsigned any = (unsigned)((d >> kTallyRebuildShift) & kTallyField);
  const int cap = min(kMaxLaunchSteps, (int)(kTallyField / (unsigned)(a.nrep + 1)));
  const int go = any == 0 && more > 0 && budget > 0 && step + 1 < cap;
  if (last && !go) {
    c->budget = budget;  // for the launch after the rebuild
    set_loop(h_loop, (more > 0 && budget > 0) ? 1u : 0u);
  }
  return go;
}

// Many fused steps in one cooperative launch (every block resident): block b
// works tile b of a step, then the grid meets at the step barrier.  The
// launch ends when a list rebuild is due, the step budget is spent or no
// replica has steps left; the step graph's loop then runs the rebuild and
// launches it again.  Positions, forces, the thermostat and every reduction
// are those of k_force<TP, true, false, FM_STREAMED>, bit for bit.  (A tile
// order that spread each SM's tiles over the box measured 0.3 us per step
// slower than block order.)
template <int TP>
__global__ void __maxnreg__(72) k_steps(EngArgs a, cudaGraphConditionalHandle h_loop) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ double s_blk[kNPart], s_tot[kNPart];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ unsigned s_rows;
  __shared__ int s_go;
  PersistCtl* c = a.pctl;
  if (threadIdx.x == 0) {
    s_go = __ldcg(&c->err) == 0;
    if (!s_go && blockIdx.x == 0) set_loop(h_loop, 0u);
    if (s_go) s_go = setup_barrier(a, h_loop);
  }
  __syncthreads();
  // the launch's step budget (written before the launch, or by the previous
  // launch's last block), counted down by every block alike
  int budget = __ldcg(&c->budget);
  unsigned long long seen[2] = {0ull, 0ull};  // thread 0: the step words' totals so far
  // one tile per block (the engine uses k_steps only when every tile has a
  // resident block); the block's view of its replica's state
  __shared__ StepView s_view;
  // the replica's descriptor and pair table, which no step changes, once for
  // the launch
  __shared__ __align__(16) RepDev s_rep;
  __shared__ unsigned s_wdone;  // warps of the block past their neighbour loop this step
  const int tile = blockIdx.x;
  const bool has_tile = tile < a.ntiles;
  const int rep_id = has_tile ? a.tile_rep[tile] : 0;
  if (has_tile) {
    if (threadIdx.x == 0) {
      load_view(s_view, a.st + a.tile_rep[tile]);
      s_view.first = a.tile_first[tile];
    }
    const RepDev& R = a.rep[a.tile_rep[tile]];
    static_assert(sizeof(RepDev) % sizeof(int) == 0, "descriptor copied as words");
    for (int k = threadIdx.x; k < (int)(sizeof(RepDev) / sizeof(int)); k += blockDim.x)
      reinterpret_cast<int*>(&s_rep)[k] = reinterpret_cast<const int*>(&R)[k];
    float* s_par = reinterpret_cast<float*>(s_dyn);
    for (int k = threadIdx.x; k < R.ntypes * R.ntypes * kParStride; k += blockDim.x) s_par[k] = a.par[R.par0 + k];
  }
  __syncthreads();
  PersistRegs pr{};
  if (has_tile) {
    const int i = s_view.first + (int)threadIdx.x / TP;
    if (i < s_rep.n) {
      const size_t gi = (size_t)s_rep.p0 + i;
      pr.nn = a.nn[gi];
      if (threadIdx.x % TP == 0) {
        pr.v = a.v[s_view.abuf][gi];
        pr.im = a.im[s_view.abuf][gi];
        pr.lr = a.last_r[gi];
      }
    }
  }
  double* s_red = reinterpret_cast<double*>(s_dyn + persist_table_bytes(a)) + (blockDim.x >> 5) * kNPart;
  for (int step = 0; s_go; ++step) {
    if (threadIdx.x == 0) {
      s_step_tally = 0ull;
      s_wdone = 0u;
    }
    __syncthreads();
    bool stepped = false;
    if (has_tile)
      stepped = force_tile<TP, true, false, FM_STREAMED, true>(a, tile, s_dyn, s_blk, s_tot, s_bar, s_rows, &s_view,
                                                               step & 1, &s_rep, &pr, &s_wdone);
    budget -= 1;
    __syncthreads();  // the tile's partial sums are written
    unsigned long long now = 0ull;
    if (threadIdx.x == 0) now = step_arrive(a, step);
    // the replica reduction and the step's finish, between the arrival and
    // the barrier's completion
    if (stepped && post_reduce(a, tile, rep_id, s_rep, step & 1, s_red, s_tot))
      finish_step_persist(a, s_rep, a.st + rep_id, s_tot);
    if (threadIdx.x == 0) {
      s_go = step_decide(a, step, budget, seen, now, h_loop);
      if (stepped) {
        s_view.rbuf ^= 1;
        if (s_view.steps_left > 0) s_view.steps_left -= 1;
        s_view.run_step += 1;
        s_view.steps += 1;
      }
    }
    __syncthreads();
  }
}

// Start of the persistent step graph: whether its loop runs at all.
__global__ void k_gate_loop(EngArgs a, cudaGraphConditionalHandle h_loop) {
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  const int nrep = __ldcg(&a.pctl->lay_nrep);  // the layout in effect (not the captured one)
  for (int r = threadIdx.x; r < nrep; r += blockDim.x)
    if (a.rep[r].active && !a.st[r].overflow && a.st[r].steps_left > 0) s_any = 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    PersistCtl* c = a.pctl;
    c->arrive = 0ull;
    cudaGraphSetConditional(h_loop, (s_any && c->budget > 0 && c->err == 0) ? 1u : 0u);
  }
}

// IntegratorNVT::Integrate alone (forces already in f).  Particle p of the
// tile sits on thread p*tp, as in k_force, so the FP64 reduction tree (and
// hence every bit of the result) is the same as the fused step's.
__global__ void __launch_bounds__(kMaxBlock) k_integrate(EngArgs a, int tp) {
  __shared__ double s_warp[(kMaxBlock / 32) * kNPart];
  __shared__ double s_scr[kMaxBlock];
  __shared__ double s_blk[kNPart], s_tot[kNPart];
  const int tile = blockIdx.x;
  const int rep = a.tile_rep[tile];
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  if (S->overflow || !R.active) return;
  const int i = a.tile_first[tile] + threadIdx.x / tp;
  double acc[kNPart];
#pragma unroll
  for (int k = 0; k < kNPart; ++k) acc[k] = 0.0;
  bool exceed = false;
  const int rb = S->rbuf, ab = S->abuf;
  if (i < R.n && threadIdx.x % tp == 0) {
    const size_t gi = (size_t)R.p0 + i;
    float4 r = a.r[rb][gi], f = a.f[gi], v = a.v[ab][gi];
    int4 im = a.im[ab][gi];
    float4 rn;
    integrate_one(R, (float)S->xi, make_float3(0.f, 0.f, 0.f), false, r, f, v, im, rn, acc, exceed, a.last_r[gi]);
    acc[P_PE] = 0.0; acc[P_W] = 0.0;
    a.v[ab][gi] = v; a.im[ab][gi] = im; a.r[rb ^ 1][gi] = rn;
  }
  const int ex = __syncthreads_or(exceed);
  if (ex && threadIdx.x == 0) atomicAdd(&S->exceed, 1);
  block_sum8(acc, s_warp, s_blk);
  if (replica_reduce(a, rep, R, tile - R.tile0, s_blk, s_scr, s_tot)) {
    if (threadIdx.x == 0) {
      double pe = S->pe, vir = S->vir;
      finish_step(a, rep, R, S, s_tot, false);
      S->pe = pe; S->vir = vir;
    }
  }
}

// Total momentum and mass of the current velocities (calculateMomentum +
// sumIdenticalArrays, IntegratorNVT.cu:176-183, 462-471), FP64.
// Tiles tile0 .. tile0 + gridDim.x - 1 (all tiles, or one replica's).
__global__ void __launch_bounds__(kMaxBlock) k_momentum(EngArgs a, int tp, int tile0) {
  __shared__ double s_warp[(kMaxBlock / 32) * kNPart];
  __shared__ double s_scr[kMaxBlock];
  __shared__ double s_blk[kNPart], s_tot[kNPart];
  const int tile = tile0 + blockIdx.x;
  const int rep = a.tile_rep[tile];
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  if (!R.active) return;
  const int i = a.tile_first[tile] + threadIdx.x / tp;
  double acc[kNPart];
#pragma unroll
  for (int k = 0; k < kNPart; ++k) acc[k] = 0.0;
  if (i < R.n && threadIdx.x % tp == 0) {
    const float4 v = a.v[S->abuf][(size_t)R.p0 + i];
    const double m = 1.0 / (double)v.w;
    acc[P_PX] = m * v.x; acc[P_PY] = m * v.y; acc[P_PZ] = m * v.z; acc[P_M] = m;
  }
  block_sum8(acc, s_warp, s_blk);
  if (replica_reduce(a, rep, R, tile - R.tile0, s_blk, s_scr, s_tot)) {
    if (threadIdx.x == 0) {
      S->P[0] = s_tot[P_PX]; S->P[1] = s_tot[P_PY]; S->P[2] = s_tot[P_PZ]; S->M = s_tot[P_M];
    }
  }
}

// zeroTotalMomentum (IntegratorNVT.cu:444-458) with the FP64 momentum.
__global__ void k_apply_zero_momentum(EngArgs a) {
  const int tile = blockIdx.x;
  const int rep = a.tile_rep[tile];
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  if (!R.active || S->M <= 0.0) return;
  const int i = a.tile_first[tile] + threadIdx.x;
  if (i >= R.n) return;
  const size_t gi = (size_t)R.p0 + i;
  float4 v = a.v[S->abuf][gi];
  v.x -= (float)(S->P[0] / S->M); v.y -= (float)(S->P[1] / S->M); v.z -= (float)(S->P[2] / S->M);
  a.v[S->abuf][gi] = v;
}

// Original particle ids 0..n-1 (a replica's slot order before its first sort).
__global__ void k_iota(unsigned* ids, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ids[i] = (unsigned)i;
}

// Sets the queued step counts of all replicas (lock-step run start).
__global__ void k_set_steps(EngArgs a, long long nsteps, int reset_run_step) {
  const int rep = blockIdx.x * blockDim.x + threadIdx.x;
  if (rep >= a.nrep) return;
  if (!a.rep[rep].active) return;
  a.st[rep].steps_left = nsteps;
  if (reset_run_step) a.st[rep].run_step = 0;
}

// Adds queued steps to one replica (in stream order, after the work queued
// before it).
__global__ void k_queue_steps(RepState* s, long long nsteps) { s->steps_left += nsteps; }

// An enlarged list is in place: the replica's overflow flag is cleared and
// its list is due (in stream order).
__global__ void k_clear_overflow(RepState* s) {
  s->overflow = 0;
  s->rebuild = 1;
}

// Within a run only replicas that step again are rebuilt (a replica whose
// queue is empty keeps its flag until it steps or CalcF runs), as the
// batched kernels do.
__device__ __forceinline__ bool rb_active(const EngArgs& a, int rep) {
  const RepState* S = a.st + rep;
  return a.rep[rep].active && S->rebuild && !S->overflow && (!a.rb_steps_only || S->steps_left > 0);
}

// Gate: publishes "any replica flagged for rebuild" to the first conditional node.
__global__ void k_gate(EngArgs a, cudaGraphConditionalHandle h) {
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < a.nrep; r += blockDim.x)
    if (rb_active(a, r)) s_any = 1;
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h, s_any ? 1u : 0u);
}

// The gate's decision written to memory (for a host that takes it instead of
// a conditional graph node).
__global__ void k_gate_flag(EngArgs a, int* out) {
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < a.nrep; r += blockDim.x)
    if (rb_active(a, r)) s_any = 1;
  __syncthreads();
  if (threadIdx.x == 0) *out = s_any;
}

// ---------------------------------------------------------------------------
// Neighbour-list rebuild (NeighborList::CalculateNBL_Sorting, NeighborList.cu:717-781).
// Grid = tiles, block = pb (one thread per slot).  Every kernel returns at once
// for replicas that are not flagged, so the same sequence serves batches.
// ---------------------------------------------------------------------------

__device__ __forceinline__ int cell_chunk(const RepDev& R) { return (R.ncell + R.ntiles - 1) / R.ntiles; }

// (1) zero cell counts of this tile's chunk of the replica's cells
__global__ void k_rb_clear(EngArgs a) {
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  // the replica's first tile also resets the per-build maximum list length
  if (tile == R.tile0 && threadIdx.x == 0) a.st[rep].actual_max_nbrs = 0;
  if (R.nb_method != NB_CELLS) return;
  const int ch = cell_chunk(R), lt = tile - R.tile0;
  const int c0 = lt * ch, c1 = min(R.ncell, c0 + ch);
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) a.cnt[R.cell0 + c] = 0;
}

// (2) cell key per particle (calculateCellIndices, NeighborList.cu:1142-1172) and
//     its arrival rank in the cell
__global__ void k_rb_count(EngArgs a) {
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  if (R.nb_method != NB_CELLS) return;
  const int i = a.tile_first[tile] + threadIdx.x;
  if (i >= R.n) return;
  const size_t gi = (size_t)R.p0 + i;
  const float4 r = a.r[a.st[rep].rbuf][gi];
  const int cx = cell_coord(r.x, R.invL[0], R.nc[0]);
  const int cy = cell_coord(r.y, R.invL[1], R.nc[1]);
  const int cz = cell_coord(r.z, R.invL[2], R.nc[2]);
  const int key = cx + cy * R.nc[0] + cz * R.nc[0] * R.nc[1];
  a.key[gi] = key;
  a.slot[gi] = atomicAdd(&a.cnt[R.cell0 + key], 1);
}

// (3a) chunk-local exclusive prefix of cell counts; chunk total per tile
__global__ void k_rb_scan_local(EngArgs a) {
  __shared__ int s_w[kMaxBlock / 32];
  __shared__ int s_carry;
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  if (R.nb_method != NB_CELLS) return;
  const int ch = cell_chunk(R), lt = tile - R.tile0;
  const int c0 = lt * ch, c1 = min(R.ncell, c0 + ch);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = c0; base < c1; base += blockDim.x) {
    const int c = base + threadIdx.x;
    const int x = c < c1 ? a.cnt[R.cell0 + c] : 0;
    int incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    int woff = 0;
    for (int w = 0; w < wid; ++w) woff += s_w[w];
    const int carry = s_carry;
    if (c < c1) a.cstart[R.cell0 + c] = carry + woff + incl - x;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) {
      int tot = 0;
      for (int w = 0; w < nw; ++w) tot += s_w[w];
      s_carry = carry + tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) a.ctot[tile] = s_carry;
}

// (3b) exclusive prefix of chunk totals over the replica's tiles (block per
//      replica): thread t sums a run of consecutive tiles (its loads all in
//      flight together), the block scans the run sums, and each thread
//      writes its run's prefixes
constexpr int kScanRun = 8;  // tiles per thread and pass
__global__ void k_rb_scan_tiles(EngArgs a) {
  __shared__ int s_w[32];
  __shared__ int s_carry;
  const int rep = blockIdx.x;
  if (rep >= a.nrep || !rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  if (R.nb_method != NB_CELLS) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int* __restrict__ tot = a.ctot + R.tile0;
  int* __restrict__ pref = a.cpref + R.tile0;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < R.ntiles; base += blockDim.x * kScanRun) {
    const int t0 = base + threadIdx.x * kScanRun;
    int x[kScanRun];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanRun; ++k) {
      x[k] = t0 + k < R.ntiles ? tot[t0 + k] : 0;
      sum += x[k];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    int woff = 0;
    for (int w = 0; w < wid; ++w) woff += s_w[w];
    const int carry = s_carry;
    int run = carry + woff + incl - sum;
#pragma unroll
    for (int k = 0; k < kScanRun; ++k) {
      if (t0 + k < R.ntiles) pref[t0 + k] = run;
      run += x[k];
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) {
      int t = 0;
      for (int w = 0; w < nw; ++w) t += s_w[w];
      s_carry = carry + t;
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int cell_begin(const EngArgs& a, const RepDev& R, int c, int ch) {
  return a.cstart[R.cell0 + c] + a.cpref[R.tile0 + c / ch];
}

// (4) scatter particle ids to their cell buckets (arrival order)
__global__ void k_rb_scatter(EngArgs a) {
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  if (R.nb_method != NB_CELLS) return;
  const int i = a.tile_first[tile] + threadIdx.x;
  if (i >= R.n) return;
  const size_t gi = (size_t)R.p0 + i;
  const int key = a.key[gi];
  const int pos = cell_begin(a, R, key, cell_chunk(R)) + a.slot[gi];
  a.order[(size_t)R.p0 + pos] = (unsigned)i;
}

// (5) order each bucket by old index: the result equals a stable sort by key
//     (thrust::sort_by_key on (cellIndex, iota), Sample.h:174-188).  Also
//     turns cstart into each cell's absolute first slot (cstart + the chunk's
//     prefix), which the list build reads without a division.
constexpr int kFixRegs = 8;  // buckets up to this size are sorted in registers
__global__ void k_rb_fix(EngArgs a) {
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  if (R.nb_method != NB_CELLS) return;
  const int ch = cell_chunk(R), lt = tile - R.tile0;
  const int c0 = lt * ch, c1 = min(R.ncell, c0 + ch);
  const int pref = a.cpref[R.tile0 + lt];
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    const int b = a.cstart[R.cell0 + c] + pref, m = a.cnt[R.cell0 + c];
    a.cstart[R.cell0 + c] = b;
    unsigned* o = a.order + (size_t)R.p0 + b;
    if (m <= kFixRegs) {
      // the bucket in registers (padding sorts last), odd-even transposition
      unsigned x[kFixRegs];
#pragma unroll
      for (int k = 0; k < kFixRegs; ++k) x[k] = k < m ? o[k] : 0xffffffffu;
#pragma unroll
      for (int r = 0; r < kFixRegs; ++r)
#pragma unroll
        for (int k = r & 1; k + 1 < kFixRegs; k += 2) {
          const unsigned lo = min(x[k], x[k + 1]), hi = max(x[k], x[k + 1]);
          x[k] = lo;
          x[k + 1] = hi;
        }
#pragma unroll
      for (int k = 0; k < kFixRegs; ++k)
        if (k < m) o[k] = x[k];
      continue;
    }
    for (int p = 1; p < m; ++p) {
      unsigned x = o[p];
      int q = p - 1;
      while (q >= 0 && o[q] > x) { o[q + 1] = o[q]; --q; }
      o[q + 1] = x;
    }
  }
}

// (6) gather r, v, images, unsorted index into the sorted order
//     (ParticleData::UpdateAfterSorting, ParticleData.cu:493-528); the last
//     block of the replica flips the buffer parities
__global__ void k_rb_permute(EngArgs a) {
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  if (R.nb_method != NB_CELLS) return;
  RepState* S = a.st + rep;
  const int s = a.tile_first[tile] + threadIdx.x;
  const int rb = S->rbuf, ab = S->abuf;
  if (s < R.n) {
    const size_t gs = (size_t)R.p0 + s;
    const size_t go = (size_t)R.p0 + a.order[gs];
    a.r[rb ^ 1][gs] = a.r[rb][go];
    a.v[ab ^ 1][gs] = a.v[ab][go];
    a.im[ab ^ 1][gs] = a.im[ab][go];
    a.uidx[ab ^ 1][gs] = a.uidx[ab][go];
  }
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned c = atomicAdd(&a.rctr[rep], 1u);
    s_last = (c == (unsigned)(R.ntiles - 1));
    if (s_last) {
      a.rctr[rep] = 0u;
      S->rbuf = rb ^ 1;
      S->abuf = ab ^ 1;
    }
  }
}

// (7) sorted 5x5x5 cell scan (calculateNBL_CellsSorted, NeighborList.cu:1204-1319):
//     neighbours in the reference's order (dz, dy, dx, ascending slot).
//     LP lanes share one particle.  Its 25 (dz, dy) rows are contiguous slot
//     ranges (two when a row wraps); each round the LP lanes test LP
//     consecutive candidates and append the accepted ones in candidate order
//     (ballot + prefix count), so the list is the reference's entry for entry.
//     All groups of a warp run the same number of rounds per range (the warp
//     maximum), so the warp never diverges.  The tile's list is assembled in
//     shared memory and written row by row with TMA bulk stores (a
//     column-major row of the tile is one contiguous slot run).
constexpr int kCs2Floats = kMaxTypes * kMaxTypes;

// Position window of a tile (built with the list, read by k_force FM_WINDOW).
// The tile's particles are consecutive in cell-key order, so they lie in at
// most a few cell rows (y, z) -- its base rows -- each over an x-interval
// [xa, xb] of cells.  Every listed neighbour of a particle lies in the 25 rows
// (y+dy, z+dz), |dy|,|dz| <= 2, at x-cells within 2 of its own.  The window is
// the union, per neighbour row, of the x-intervals [xa-2, xb+2] (modulo the
// row length): a few slot segments (cells of one row are consecutive keys,
// hence consecutive slots).  Segments are kept sorted by first slot and
// numbered into the window in that order; a list entry j then becomes the
// window offset j + (offset - first slot) of its segment.
struct WinScratch {
  int rowid[kMaxBlock];  // base row y + z*ny of each particle of the tile
  int cx[kMaxBlock];     // x-cell of each particle
  int brow[kWinBase], bxa[kWinBase], bxb[kWinBase];
  int erow[25 * kWinBase];        // neighbour row of entry (base row, dz, dy)
  int eiv[25 * kWinBase][4];      // its x-cells as <= 2 linear intervals
  int em[25 * kWinBase];          // merged intervals (row leaders only)
  int eseg[25 * kWinBase];        // first segment number of a leader
  int ems[25 * kWinBase][8];      // <= 4 merged intervals [c0, c1)
  int ustart[kWinSeg], ulen[kWinSeg];
  int sstart[kWinSeg], slen[kWinSeg], soff[kWinSeg];
  int nseg, W;  // nseg < 0: the tile has no window
};

// Builds the tile's window into w (and wseg / wmeta).  Called by the whole
// block after rowid / cx of its np particles are written; warp 0 works.
__device__ void tile_window(const EngArgs& a, const RepDev& R, int tile, int np, WinScratch* w) {
  if (threadIdx.x >= 32) return;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x;
  const unsigned lt = (1u << lane) - 1u;
  const int nx = R.nc[0], ny = R.nc[1], nz = R.nc[2];
  bool bad = false;
  // W1: base rows = runs of equal rowid (x rises within a run)
  int nb = 0, nend = 0;
  for (int c0 = 0; c0 < np; c0 += 32) {
    const int p = c0 + lane;
    const bool in = p < np;
    const bool st = in && (p == 0 || w->rowid[p] != w->rowid[p - 1]);
    const bool en = in && (p == np - 1 || w->rowid[p] != w->rowid[p + 1]);
    const unsigned ms = __ballot_sync(FULL, st), me = __ballot_sync(FULL, en);
    const int rs = nb + __popc(ms & lt), re = nend + __popc(me & lt);
    if (st && rs < kWinBase) {
      w->brow[rs] = w->rowid[p];
      w->bxa[rs] = w->cx[p];
    }
    if (en && re < kWinBase) w->bxb[re] = w->cx[p];
    nb += __popc(ms);
    nend += __popc(me);
  }
  if (nb > kWinBase || nb == 0) bad = true;
  __syncwarp();
  const int ne = bad ? 0 : 25 * nb;
  // W2: entries (base row, dz, dy) -> neighbour row and x-intervals
  for (int e = lane; e < ne; e += 32) {
    const int k = e / 25, d = e % 25;
    const int dz = d / 5 - 2, dy = d % 5 - 2;
    const int by = w->brow[k] % ny, bz = w->brow[k] / ny;
    int y = by + dy;
    y += ((y < 0) - (y >= ny)) * ny;
    int z = bz + dz;
    z += ((z < 0) - (z >= nz)) * nz;
    w->erow[e] = y + z * ny;
    const int len = w->bxb[k] - w->bxa[k] + 5;
    int a0 = 0, b0 = nx, a1 = 0, b1 = 0;
    if (len < nx) {
      int s0 = w->bxa[k] - 2;
      if (s0 < 0) s0 += nx;
      a0 = s0;
      if (s0 + len <= nx) {
        b0 = s0 + len;
      } else {
        b0 = nx;
        b1 = s0 + len - nx;
      }
    }
    w->eiv[e][0] = a0; w->eiv[e][1] = b0; w->eiv[e][2] = a1; w->eiv[e][3] = b1;
  }
  __syncwarp();
  // W3: the first entry of each distinct row merges the row's intervals
  int badm = 0;
  for (int e = lane; e < ne; e += 32) {
    const int row = w->erow[e];
    bool leader = true;
    for (int e2 = 0; e2 < e; ++e2)
      if (w->erow[e2] == row) { leader = false; break; }
    int m = 0;
    if (leader) {
      int ia[2 * kWinBase], ib[2 * kWinBase], c = 0;
      for (int e2 = e; e2 < ne; ++e2) {
        if (w->erow[e2] != row) continue;
        for (int hh = 0; hh < 2; ++hh) {
          const int x0 = w->eiv[e2][2 * hh], x1 = w->eiv[e2][2 * hh + 1];
          if (x1 > x0 && c < 2 * kWinBase) {
            int t = c++;
            while (t > 0 && ia[t - 1] > x0) { ia[t] = ia[t - 1]; ib[t] = ib[t - 1]; --t; }
            ia[t] = x0; ib[t] = x1;
          }
        }
      }
      for (int t = 0; t < c; ++t) {
        if (m > 0 && ia[t] <= w->ems[e][2 * m - 1]) {
          w->ems[e][2 * m - 1] = max(w->ems[e][2 * m - 1], ib[t]);
        } else if (m < 4) {
          w->ems[e][2 * m] = ia[t];
          w->ems[e][2 * m + 1] = ib[t];
          ++m;
        } else {
          badm = 1;
        }
      }
    }
    w->em[e] = m;
  }
  bad = bad || __any_sync(FULL, badm);
  __syncwarp();
  // W4: segment numbers, and slot ranges from the cell starts
  int S = 0;
  for (int c0 = 0; c0 < ne; c0 += 32) {
    const int e = c0 + lane;
    const int m = e < ne ? w->em[e] : 0;
    int incl = m;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (e < ne) w->eseg[e] = S + incl - m;
    S += __shfl_sync(FULL, incl, 31);
  }
  if (S > kWinSeg) bad = true;
  __syncwarp();
  const int* __restrict__ cbeg = a.cstart + R.cell0;  // absolute first slot (k_rb_fix)
  const int* __restrict__ ccnt = a.cnt + R.cell0;
  if (!bad)
    for (int e = lane; e < ne; e += 32) {
      const int m = w->em[e], row = w->erow[e], b = w->eseg[e];
      for (int t = 0; t < m; ++t) {
        const int k0 = row * nx + w->ems[e][2 * t], k1 = row * nx + w->ems[e][2 * t + 1] - 1;
        const int s0 = cbeg[k0], s1 = cbeg[k1] + ccnt[k1];
        w->ustart[b + t] = s0;
        w->ulen[b + t] = s1 - s0;
      }
    }
  __syncwarp();
  // W5: non-empty segments in slot order (disjoint, so ranks by counting)
  int nseg = 0;
  if (!bad) {
    int cnt = 0;
    for (int sg = lane; sg < S; sg += 32) {
      if (w->ulen[sg] <= 0) continue;
      ++cnt;
      const int st = w->ustart[sg];
      int r = 0;
      for (int t = 0; t < S; ++t) r += (w->ulen[t] > 0) && (w->ustart[t] < st);
      w->sstart[r] = st;
      w->slen[r] = w->ulen[sg];
    }
    nseg = __reduce_add_sync(FULL, cnt);
  }
  __syncwarp();
  // W6: window offsets (exclusive prefix of the lengths in slot order)
  int W = 0;
  for (int c0 = 0; c0 < nseg; c0 += 32) {
    const int sg = c0 + lane;
    const int len = sg < nseg ? w->slen[sg] : 0;
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (sg < nseg) w->soff[sg] = W + incl - len;
    W += __shfl_sync(FULL, incl, 31);
  }
  if (W > a.win_cap) bad = true;
  if (!bad)
    for (int sg = lane; sg < nseg; sg += 32)
      a.wseg[(size_t)tile * kWinSeg + sg] = make_int4(w->sstart[sg], w->slen[sg], w->soff[sg], 0);
  if (lane == 0) {
    w->nseg = bad ? -1 : nseg;
    w->W = bad ? -1 : W;
    a.wmeta[tile] = make_int2(w->nseg, w->W);
  }
}

// The tile's window segments as the list build reads them (shared memory).
struct WinTable {
  int sstart[kWinSeg], slen[kWinSeg], soff[kWinSeg];
  int nseg;
};

// (6b) the position window of every tile (after the sort, before the list
//      build): one block per tile, pb threads
__global__ void __launch_bounds__(kMaxBlock) k_rb_window(EngArgs a) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  WinScratch* w = reinterpret_cast<WinScratch*>(s_dyn);
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!a.win_on || !rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  if (R.nb_method != NB_CELLS) {
    if (threadIdx.x == 0) a.wmeta[tile] = make_int2(-1, -1);  // no window for all pairs
    return;
  }
  const int first = a.tile_first[tile];
  const int np = min((int)blockDim.x, R.n - first);
  if ((int)threadIdx.x < np) {
    const float4 r = a.r[a.st[rep].rbuf][(size_t)R.p0 + first + threadIdx.x];
    const int cx = cell_coord(r.x, R.invL[0], R.nc[0]);
    const int cy = cell_coord(r.y, R.invL[1], R.nc[1]);
    const int cz = cell_coord(r.z, R.invL[2], R.nc[2]);
    w->rowid[threadIdx.x] = cy + cz * R.nc[1];
    w->cx[threadIdx.x] = cx;
  }
  __syncthreads();
  tile_window(a, R, tile, np, w);
}

// Window offset delta of the non-empty slot range [b, e) of one neighbour
// row part, which lies in one window segment by construction; a range that
// does not sets *bad (the tile then gets no window, so k_force never reads
// outside the staged window).
__device__ __forceinline__ int window_delta(const WinTable* w, int b, int e, int* bad) {
  int lo = 0, hi = w->nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (w->sstart[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  if (w->nseg <= 0 || b < w->sstart[lo] || e > w->sstart[lo] + w->slen[lo]) *bad = 1;
  return w->soff[lo] - w->sstart[lo];
}

//     SMEM_LIST = false writes the entries straight to the global list (one
//     lane per particle needs no shared-memory tile and keeps occupancy high).
template <int LP, bool SMEM_LIST, bool WIN>
__global__ void __launch_bounds__(kMaxBlock) k_rb_build(EngArgs a) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  float* s_cs2 = reinterpret_cast<float*>(s_dyn);
  unsigned* s_list = reinterpret_cast<unsigned*>(s_dyn + kCs2Floats * sizeof(float));
  __shared__ int s_max, s_winbad;
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  const int nt = R.ntypes;
  const int pb = blockDim.x / LP;
  // shared-memory list tile: block b (8 entries) of slot lp at s_list[(b * pb + lp) * 8]
  for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) s_cs2[k] = a.par[R.par0 + k * kParStride + 6];
  if (threadIdx.x == 0) {
    s_max = 0;
    s_winbad = 0;
  }
  __syncthreads();
  const int lp = threadIdx.x / LP, q = threadIdx.x % LP;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned gshift = lane & ~(unsigned)(LP - 1);
  const unsigned gbits = LP == 32 ? 0xffffffffu : ((1u << LP) - 1u);
  const unsigned below = (1u << (lane - gshift)) - 1u;
  const int first = a.tile_first[tile];
  const int i = first + lp;
  const bool valid = i < R.n;
  const float4* __restrict__ rc = a.r[S->rbuf] + R.p0;
  const int maxn = R.max_nbrs;
  const float4 ri = valid ? rc[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float* cs2 = s_cs2 + (valid ? __float_as_int(ri.w) : 0) * nt;
  const float Lx = R.L[0], Ly = R.L[1], Lz = R.L[2];
  const float iLx = R.invL[0], iLy = R.invL[1], iLz = R.invL[2];
  // this particle's list column, held in registers: the list stores below
  // cannot alias the replica table as far as the compiler can tell, so
  // reading R.nbl0 / R.nbl_stride in the loop would reload them after every store
  unsigned* __restrict__ lbase = a.nbl + R.nbl0;
  unsigned short* __restrict__ wbase = a.wl + R.nbl0;
  const size_t lstride = (size_t)R.nbl_stride;
  WinTable* ws = reinterpret_cast<WinTable*>(
      s_dyn + kCs2Floats * sizeof(float) + (SMEM_LIST ? (size_t)list_rows(a.idx_rows) * pb * sizeof(unsigned) : 0));
  bool win_ok = false;
  if (WIN) {
    // the tile's window segments (k_rb_window), sorted by first slot
    const int2 wm = a.wmeta[tile];
    const int ns = wm.x >= 0 ? min(wm.x, kWinSeg) : -1;
    for (int k = threadIdx.x; k < ns; k += blockDim.x) {
      const int4 sg = a.wseg[(size_t)tile * kWinSeg + k];
      ws->sstart[k] = sg.x;
      ws->slen[k] = sg.y;
      ws->soff[k] = sg.z;
    }
    if (threadIdx.x == 0) ws->nseg = ns;
    __syncthreads();
    win_ok = ws->nseg > 0;
  }
  int count = 0;
  // appends the accepted candidates of slots [b, e); every lane of the warp
  // calls it (invalid groups with an empty range).  With a window, entry j is
  // also written to the window list as j + delta.
  auto seg = [&](int b, int e, bool wrap, int delta) {
    int rounds = e > b ? (e - b + LP - 1) / LP : 0;
    rounds = __reduce_max_sync(0xffffffffu, rounds);
    for (int r = 0; r < rounds; ++r) {
      const int j = b + r * LP + q;
      bool in = false;
      if (j < e) {
        const float4 rj = __ldg(rc + j);
        float dx = ri.x - rj.x, dy = ri.y - rj.y, dz = ri.z - rj.z;
        if (wrap) {
          dx = mi_comp(dx, Lx, iLx);
          dy = mi_comp(dy, Ly, iLy);
          dz = mi_comp(dz, Lz, iLz);
        }
        in = (j != i) && dist2_ref(dx, dy, dz) < cs2[__float_as_int(rj.w)];
      }
      const unsigned g = (__ballot_sync(0xffffffffu, in) >> gshift) & gbits;
      if (in) {
        const int pos = count + __popc(g & below);
        if (pos < maxn) {
          if (SMEM_LIST) s_list[((pos >> 3) * pb + lp) * 8 + (pos & 7)] = (unsigned)j;
          else lbase[lpos((unsigned)pos, (unsigned)i, lstride)] = (unsigned)j;
          if (WIN && win_ok) wbase[lpos((unsigned)pos, (unsigned)i, lstride)] = (unsigned short)(j + delta);
        }
      }
      count += __popc(g);
    }
  };
  if (R.nb_method == NB_CELLS) {
    const int* __restrict__ cbeg = a.cstart + R.cell0;  // absolute first slot (k_rb_fix)
    const int* __restrict__ ccnt = a.cnt + R.cell0;
    const int nx = R.nc[0], ny = R.nc[1], nz = R.nc[2];
    const int cx = cell_coord(ri.x, iLx, nx), cy = cell_coord(ri.y, iLy, ny), cz = cell_coord(ri.z, iLz, nz);
    // With at least 7 cells per side and no wrapped cell among the 5x5x5,
    // every candidate is within 3/7 of a box length of the particle, so the
    // minimum-image step is exactly the identity; warps made only of such
    // particles skip it.
    const bool inner = nx >= 7 && ny >= 7 && nz >= 7 && cx >= 2 && cx < nx - 2 && cy >= 2 && cy < ny - 2 &&
                       cz >= 2 && cz < nz - 2;
    const bool wrap = !__all_sync(0xffffffffu, !valid || inner);
    // Cells farther from the particle than its largest list radius hold no
    // neighbour: rows (dz, dy) out of reach are skipped and each row's x-range
    // is trimmed at its ends, which leaves the list (and its order) unchanged.
    // The reach is the largest (rc + skin) of the particle's type plus 0.01;
    // the gaps are the exact distances from the particle to the cell faces.
    float reach2 = 0.f;
    for (int k = 0; k < nt; ++k) reach2 = fmaxf(reach2, cs2[k]);
    reach2 = sqrtf(reach2) + 0.01f;
    reach2 *= reach2;
    const float wx = Lx / nx, wy = Ly / ny, wz = Lz / nz;
    auto gap = [](float x, int c, int d, float w, float half) -> float {
      if (d > 0) return fmaxf(0.f, fmaf((float)(c + d), w, -half) - x);
      if (d < 0) return fmaxf(0.f, x - fmaf((float)(c + d + 1), w, -half));
      return 0.f;
    };
    for (int dz = -2; dz <= 2; ++dz) {
      int oz = cz + dz;
      oz += ((oz < 0) - (oz >= nz)) * nz;
      const float gz = gap(ri.z, cz, dz, wz, 0.5f * Lz);
      for (int dy = -2; dy <= 2; ++dy) {
        int oy = cy + dy;
        oy += ((oy < 0) - (oy >= ny)) * ny;
        const float gy = gap(ri.y, cy, dy, wy, 0.5f * Ly);
        const float gyz2 = fmaf(gy, gy, gz * gz);
        // the cells cx+dxl..cx+dxh of this row are consecutive keys, so
        // their particles are one slot range (two when the row wraps); the
        // scan order dx ascending, ascending slot, is the reference's
        int dxl = -2, dxh = 2;
        while (dxl < 0 && fmaf(gap(ri.x, cx, dxl, wx, 0.5f * Lx), gap(ri.x, cx, dxl, wx, 0.5f * Lx), gyz2) >= reach2)
          ++dxl;
        while (dxh > 0 && fmaf(gap(ri.x, cx, dxh, wx, 0.5f * Lx), gap(ri.x, cx, dxh, wx, 0.5f * Lx), gyz2) >= reach2)
          --dxh;
        const bool reach = gyz2 < reach2;
        const int row = oy * nx + oz * nx * ny;
        const int lo = cx + dxl, hi = cx + dxh;
        int b0 = 0, e0 = 0, b1 = 0, e1 = 0;
        if (valid && reach) {
          if (lo >= 0 && hi < nx) {
            const int c1 = row + hi;
            b0 = cbeg[row + lo];
            e0 = cbeg[c1] + ccnt[c1];
          } else {
            const int cw = row + nx - 1;
            const int ca = lo < 0 ? row + nx + lo : row + lo;  // first cell of the wrapped part order
            const int cb = lo < 0 ? row + hi : row + hi - nx;
            b0 = cbeg[ca];
            e0 = cbeg[cw] + ccnt[cw];
            b1 = cbeg[row];
            e1 = cbeg[cb] + ccnt[cb];
          }
        }
        const int d0 = WIN && win_ok && e0 > b0 ? window_delta(ws, b0, e0, &s_winbad) : 0;
        const int d1 = WIN && win_ok && e1 > b1 ? window_delta(ws, b1, e1, &s_winbad) : 0;
        seg(b0, e0, wrap, d0);
        seg(b1, e1, wrap, d1);
      }
    }
  } else {
    seg(0, valid ? R.n : 0, true, 0);  // all pairs (calculateNBL_N2 criterion), ascending j
  }
  if (valid && q == 0) {
    a.nn[(size_t)R.p0 + i] = (unsigned)min(count, maxn);
    a.last_r[(size_t)R.p0 + i] = ri;
    atomicMax(&s_max, count);
  }
  // write the tile's rows [0, rows) of the list: slots [first, first+width)
  if (SMEM_LIST) fence_async_shared();
  __syncthreads();
  if (WIN && win_ok && threadIdx.x == 0 && s_winbad) a.wmeta[tile] = make_int2(-1, -1);
  if (SMEM_LIST && threadIdx.x < 32) {
    const int nblk = (min(s_max, maxn) + 7) >> 3;
    const unsigned width = (unsigned)min(pb, R.nbl_stride - first);
    unsigned* dst = a.nbl + R.nbl0 + (size_t)first * 8;
    for (int b = threadIdx.x; b < nblk; b += 32)
      bulk_s2g(dst + (size_t)b * R.nbl_stride * 8, s_list + b * pb * 8, width * 32u);
    bulk_commit();
    bulk_wait_all();
  }
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    const int s_max_v = s_max;
    atomicMax(&S->actual_max_nbrs, s_max_v);
    if (s_max_v > R.max_nbrs) atomicExch(&S->overflow, 1);
    __threadfence();
    unsigned c = atomicAdd(&a.rctr[rep], 1u);
    s_last = (c == (unsigned)(R.ntiles - 1));
    if (s_last) {
      a.rctr[rep] = 0u;
      S->rebuild = 0;
      S->nrebuilds += 1;
    }
  }
}

// (7') The same list with one warp per cell.  The particles of a cell share
//      their 25 neighbour row parts, so the warp stages the candidates' slots
//      and positions in shared memory once (kCwCand at a time) and tests each
//      particle of the cell against 32 consecutive candidates per round;
//      ballot + prefix count append the accepted ones in candidate order, the
//      reference's order.  Every lane does useful work in every round but the
//      last of a particle.  All-pairs replicas use one part [0, n) for the
//      whole tile.
constexpr int kCwWarps = 4;   // warps per block
constexpr int kCwCand = 256;  // staged candidates per warp

__global__ void __launch_bounds__(kCwWarps * 32) k_rb_build_cw(EngArgs a) {
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(128) unsigned char s_dyn[];
  float* s_cs2 = reinterpret_cast<float*>(s_dyn);
  float4* s_pos = reinterpret_cast<float4*>(s_dyn + kCs2Floats * sizeof(float));  // [warp][kCwCand]
  int* s_slot = reinterpret_cast<int*>(s_pos + kCwWarps * kCwCand);                 // [warp][kCwCand]
  __shared__ int s_max;
  const int tile = blockIdx.x, rep = a.tile_rep[tile];
  if (!rb_active(a, rep)) return;
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  const int nt = R.ntypes;
  for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) s_cs2[k] = a.par[R.par0 + k * kParStride + 6];
  if (threadIdx.x == 0) s_max = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int first = a.tile_first[tile];
  const int last = (tile + 1 < R.tile0 + R.ntiles) ? a.tile_first[tile + 1] : R.n;
  const float4* __restrict__ rc = a.r[S->rbuf] + R.p0;
  const int maxn = R.max_nbrs;
  const float Lx = R.L[0], Ly = R.L[1], Lz = R.L[2];
  const float iLx = R.invL[0], iLy = R.invL[1], iLz = R.invL[2];
  const size_t lstride = (size_t)R.nbl_stride;
  unsigned* __restrict__ lbase = a.nbl + R.nbl0;
  float4* wpos = s_pos + warp * kCwCand;
  int* wslot = s_slot + warp * kCwCand;
  const bool cells = R.nb_method == NB_CELLS;
  const int nx = R.nc[0], ny = R.nc[1], nz = R.nc[2];
  const int* __restrict__ cbeg = a.cstart + R.cell0;  // absolute first slot (k_rb_fix)
  const int* __restrict__ ccnt = a.cnt + R.cell0;
  // units of work: the cells from the first to the last particle's (keys
  // ascend along the slots), or one unit for all pairs
  int k0 = 0, k1 = 0;
  if (cells && last > first) {
    const float4 rf = rc[first], rl = rc[last - 1];
    k0 = cell_coord(rf.x, iLx, nx) + cell_coord(rf.y, iLy, ny) * nx + cell_coord(rf.z, iLz, nz) * nx * ny;
    k1 = cell_coord(rl.x, iLx, nx) + cell_coord(rl.y, iLy, ny) * nx + cell_coord(rl.z, iLz, nz) * nx * ny;
  }
  int wmax = 0;
  for (int c = k0 + warp; c <= k1; c += kCwWarps) {
    const int p0 = cells ? max(cbeg[c], first) : first;
    const int p1 = cells ? min(cbeg[c] + ccnt[c], last) : last;
    if (p0 >= p1) continue;  // no particle of this tile in the cell
    // lane r < 25: row (dz, dy) = (r/5 - 2, r%5 - 2) as one or two slot parts
    int b0 = 0, e0 = 0, b1 = 0, e1 = 0;
    bool wrap = true;
    if (cells) {
      const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
      // no wrapped cell among the 5x5x5 and at least 7 cells a side: the
      // minimum-image step is exactly the identity
      wrap = !(nx >= 7 && ny >= 7 && nz >= 7 && cx >= 2 && cx < nx - 2 && cy >= 2 && cy < ny - 2 && cz >= 2 &&
               cz < nz - 2);
      if (lane < 25) {
        const int dz = lane / 5 - 2, dy = lane % 5 - 2;
        int oz = cz + dz;
        oz += ((oz < 0) - (oz >= nz)) * nz;
        int oy = cy + dy;
        oy += ((oy < 0) - (oy >= ny)) * ny;
        const int row = oy * nx + oz * nx * ny;
        const int lo = cx - 2, hi = cx + 2;
        if (lo >= 0 && hi < nx) {
          b0 = cbeg[row + lo];
          e0 = cbeg[row + hi] + ccnt[row + hi];
        } else {
          const int cw = row + nx - 1;
          const int ca = lo < 0 ? row + nx + lo : row + lo;
          const int cb = lo < 0 ? row + hi : row + hi - nx;
          b0 = cbeg[ca];
          e0 = cbeg[cw] + ccnt[cw];
          b1 = cbeg[row];
          e1 = cbeg[cb] + ccnt[cb];
        }
      }
    } else if (lane == 0) {
      e0 = R.n;
    }
    const int l0 = e0 - b0, len = l0 + (e1 - b1);
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    const int off = incl - len;                  // this lane's first candidate number
    const int M = __shfl_sync(FULL, incl, 31);   // candidates of the unit
    for (int pg = p0; pg < p1; pg += 32) {
      const int pe = min(p1, pg + 32);
      int cnt_reg = 0;  // lane k: count of particle pg + k
      for (int ch = 0; ch < M; ch += kCwCand) {
        const int mc = min(kCwCand, M - ch);
        __syncwarp();
        // candidate numbers [ch, ch + mc): each lane writes its own parts
        for (int v = max(off, ch); v < min(off + l0, ch + mc); ++v) wslot[v - ch] = b0 + (v - off);
        for (int v = max(off + l0, ch); v < min(off + len, ch + mc); ++v) wslot[v - ch] = b1 + (v - off - l0);
        __syncwarp();
        // the lane's position loads all in flight together
#pragma unroll
        for (int u = 0; u < kCwCand / 32; ++u) {
          const int v = lane + 32 * u;
          if (v < mc) wpos[v] = __ldg(rc + wslot[v]);
        }
        __syncwarp();
        // two particles at a time: each staged candidate is read once and
        // tested against both (the second is a copy of the first when the
        // cell has an odd count; its results are discarded)
        for (int p = pg; p < pe; p += 2) {
          const bool two = p + 1 < pe;
          const int p1 = two ? p + 1 : p;
          const float4 ra = rc[p], rb = rc[p1];
          const float* cs2a = s_cs2 + __float_as_int(ra.w) * nt;
          const float* cs2b = s_cs2 + __float_as_int(rb.w) * nt;
          int ca = __shfl_sync(FULL, cnt_reg, p - pg);
          int cb = __shfl_sync(FULL, cnt_reg, p1 - pg);
          for (int v0 = 0; v0 < mc; v0 += 32) {
            const int v = v0 + lane;
            bool ina = false, inb = false;
            int j = 0;
            if (v < mc) {
              j = wslot[v];
              const float4 rj = wpos[v];
              const int tj = __float_as_int(rj.w);
              float ax = ra.x - rj.x, ay = ra.y - rj.y, az = ra.z - rj.z;
              float bx = rb.x - rj.x, by = rb.y - rj.y, bz = rb.z - rj.z;
              if (wrap) {
                ax = mi_comp(ax, Lx, iLx);
                ay = mi_comp(ay, Ly, iLy);
                az = mi_comp(az, Lz, iLz);
                bx = mi_comp(bx, Lx, iLx);
                by = mi_comp(by, Ly, iLy);
                bz = mi_comp(bz, Lz, iLz);
              }
              ina = (j != p) && dist2_ref(ax, ay, az) < cs2a[tj];
              inb = two && (j != p1) && dist2_ref(bx, by, bz) < cs2b[tj];
            }
            const unsigned ga = __ballot_sync(FULL, ina), gb = __ballot_sync(FULL, inb);
            if (ina) {
              const int pos = ca + __popc(ga & lt);
              if (pos < maxn) lbase[lpos((unsigned)pos, (unsigned)p, lstride)] = (unsigned)j;
            }
            if (inb) {
              const int pos = cb + __popc(gb & lt);
              if (pos < maxn) lbase[lpos((unsigned)pos, (unsigned)p1, lstride)] = (unsigned)j;
            }
            ca += __popc(ga);
            cb += __popc(gb);
          }
          if (lane == p - pg) cnt_reg = ca;
          if (two && lane == p1 - pg) cnt_reg = cb;
        }
      }
      if (pg + lane < pe) {
        const int p = pg + lane;
        a.nn[(size_t)R.p0 + p] = (unsigned)min(cnt_reg, maxn);
        a.last_r[(size_t)R.p0 + p] = rc[p];
        wmax = max(wmax, cnt_reg);
      }
    }
  }
  wmax = __reduce_max_sync(FULL, wmax);
  if (lane == 0) atomicMax(&s_max, wmax);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int s_max_v = s_max;
    atomicMax(&S->actual_max_nbrs, s_max_v);
    if (s_max_v > R.max_nbrs) atomicExch(&S->overflow, 1);
    __threadfence();
    const unsigned cdone = atomicAdd(&a.rctr[rep], 1u);
    if (cdone == (unsigned)(R.ntiles - 1)) {
      a.rctr[rep] = 0u;
      S->rebuild = 0;
      S->nrebuilds += 1;
    }
  }
}

// (7'') The same list with one warp per cell and contiguous candidate runs:
//       the cell's candidates (its 25 row parts, numbered in the reference's
//       order) are cut into chunks of up to 32 * kRunMax, and lane l of the
//       warp takes the consecutive run [l K, (l + 1) K) of a chunk (K <= 16).
//       For two of the cell's particles at a time, a lane tests its run with
//       no cross-lane traffic, keeping one accept bit per candidate; one
//       exclusive scan of the lanes' accept counts then gives each lane the
//       list position of its first accepted candidate, and the lane writes its
//       accepted ones in run order.  Runs follow one another in candidate
//       order, so the list is the reference's entry for entry.  Only the
//       candidates' slots are staged (in shared memory, lane-major with an odd
//       stride so that a warp's reads are bank-conflict free); their
//       positions are read through L1, where the cell's other particles and
//       the neighbouring cells' warps find them again.
constexpr int kRunWarps = 4;                 // warps (cells in flight) per block
constexpr int kRunMax = 16;                  // candidates per lane per chunk
constexpr int kRunStride = kRunMax + 1;      // odd: conflict-free lane-major slots
constexpr int kRunChunk = 32 * kRunMax;      // candidates per chunk

struct Cs2One {
  float c0;
  __device__ __forceinline__ float operator()(int) const { return c0; }
};
struct Cs2Two {
  float c0, c1;
  __device__ __forceinline__ float operator()(int tj) const { return tj ? c1 : c0; }
};
struct Cs2Table {
  const float* row;
  __device__ __forceinline__ float operator()(int tj) const { return row[tj]; }
};

// Accept bits of a lane's run for G (4 or 2) of the cell's particles (a
// missing one repeats the last; its bits are unused): each candidate's
// position is read once and tested against all G.  G = 2 serves the last
// one or two particles of a cell, so that cells of 1, 2, 5 or 6 particles do
// not test padding copies.
template <bool WRAP, bool COH, int G, class CS2>
__device__ __forceinline__ void run_tests(const int* __restrict__ run, int nrun, const float4* rc,
                                          const float4 (&rp)[4], const int (&ip)[4], const CS2 (&cs)[4],
                                          float Lx, float Ly, float Lz, float iLx, float iLy, float iLz,
                                          unsigned (&bits)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) bits[q] = 0u;
#pragma unroll 2
  for (int k = 0; k < kRunMax; ++k) {
    if (k < nrun) {
      const int j = run[k];
      const float4 rj = COH ? ld_ca_f4(rc + j) : __ldg(rc + j);
      const int tj = __float_as_int(rj.w);
#pragma unroll
      for (int q = 0; q < G; ++q) {
        float dx = rp[q].x - rj.x, dy = rp[q].y - rj.y, dz = rp[q].z - rj.z;
        if (WRAP) {
          dx = mi_comp(dx, Lx, iLx);
          dy = mi_comp(dy, Ly, iLy);
          dz = mi_comp(dz, Lz, iLz);
        }
        if (dist2_ref(dx, dy, dz) < cs[q](tj) && j != ip[q]) bits[q] |= 1u << k;
      }
    }
  }
}

// Writes particle p's accepted candidates of this chunk: `bits` of the lane's
// run, after `cnt` entries already in p's list (32-bit offsets from the
// replica's list: entry k of slot p at (k/8) 8 stride + 8 p + k%8).
// Returns the chunk's total for p.
__device__ __forceinline__ int run_store(unsigned bits, const int* __restrict__ run, int cnt, int maxn,
                                         unsigned* __restrict__ lbase, unsigned p, unsigned stride8) {
  const int lane = threadIdx.x & 31;
  const int c = __popc(bits);
  int incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  unsigned pos = (unsigned)(cnt + incl - c);
  const unsigned pb = p << 3;
  while (bits) {
    const int k = __ffs(bits) - 1;
    bits &= bits - 1u;
    if (pos < (unsigned)maxn) lbase[(pos >> 3) * stride8 + pb + (pos & 7u)] = (unsigned)run[k];
    ++pos;
  }
  return __shfl_sync(0xffffffffu, incl, 31);
}

// The run build of one tile by the calling block (blockDim a multiple of 32:
// one cell per warp at a time).  s_cs2: the cut-off table (kCs2Floats),
// s_run: 32 * kRunStride ints per warp, s_max: one int.  COH: the positions
// and cell arrays were written earlier in the same launch (k_batch), so they
// are read with coherent loads.
// GRID: the block's warps claim cells of the whole replica from its counter
// (S->build_next) and list every particle of a claimed cell, so the work of
// all the replica's blocks evens out (cell method only); the tile's range
// then serves only the bookkeeping.
template <bool COH, bool GRID = false>
__device__ __forceinline__ void build_runs_tile(const EngArgs& a, int tile, float* s_cs2, int* s_run, int* s_max,
                                                int* s_last = nullptr, int* s_next = nullptr) {
  constexpr unsigned FULL = 0xffffffffu;
  const int rep = a.tile_rep[tile];
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  const int nt = R.ntypes;
  const int nwarps = blockDim.x >> 5;
  for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) s_cs2[k] = a.par[R.par0 + k * kParStride + 6];
  if (threadIdx.x == 0) {
    *s_max = 0;
    if (s_next) *s_next = nwarps;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int first = a.tile_first[tile];
  const int last = (tile + 1 < R.tile0 + R.ntiles) ? a.tile_first[tile + 1] : R.n;
  const float4* rc = a.r[COH ? __ldcg(&S->rbuf) : S->rbuf] + R.p0;
  const int maxn = R.max_nbrs;
  const unsigned stride8 = 8u * (unsigned)R.nbl_stride;
  unsigned* __restrict__ lbase = a.nbl + R.nbl0;
  int* wrun = s_run + warp * 32 * kRunStride;
  const int* run = wrun + lane * kRunStride;
  const bool cells = R.nb_method == NB_CELLS;
  const int nx = R.nc[0], ny = R.nc[1], nz = R.nc[2];
  const int* cbeg = a.cstart + R.cell0;  // absolute first slot (k_rb_fix / block_sort)
  const int* ccnt = a.cnt + R.cell0;
  // units of work: the cells from the first to the last particle's (keys
  // ascend along the slots), or one unit for all pairs
  int k0 = 0, k1 = 0;
  if (GRID) {
    k1 = R.ncell - 1;
  } else if (cells && last > first) {
    const float4 rf = rc[first], rl = rc[last - 1];
    const float iLx = R.invL[0], iLy = R.invL[1], iLz = R.invL[2];
    k0 = cell_coord(rf.x, iLx, nx) + cell_coord(rf.y, iLy, ny) * nx + cell_coord(rf.z, iLz, nz) * nx * ny;
    k1 = cell_coord(rl.x, iLx, nx) + cell_coord(rl.y, iLy, ny) * nx + cell_coord(rl.z, iLz, nz) * nx * ny;
  }
  int wmax = 0;
  // cells in order, each warp taking the next unclaimed one (s_next: the
  // warps' cells even out within the block), or every nwarps-th
  auto next_cell = [&](int c) -> int {
    if (GRID) {
      int v = 0;
      if (lane == 0) v = atomicAdd(&S->build_next, 1);
      return __shfl_sync(FULL, v, 0);
    }
    if (!s_next) return c + nwarps;
    int v = 0;
    if (lane == 0) v = atomicAdd(s_next, 1);
    return k0 + __shfl_sync(FULL, v, 0);
  };
  for (int c = GRID ? next_cell(0) : k0 + warp; c <= k1; c = next_cell(c)) {
    const int p0 = GRID ? cbeg[c] : cells ? max(cbeg[c], first) : first;
    const int p1 = GRID ? cbeg[c] + ccnt[c] : cells ? min(cbeg[c] + ccnt[c], last) : last;
    if (p0 >= p1) continue;  // no particle of this tile in the cell
    // lane r < 25: row (dz, dy) = (r/5 - 2, r%5 - 2) as one or two slot parts
    int b0 = 0, e0 = 0, b1 = 0, e1 = 0;
    bool wrap = true;
    if (cells) {
      const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
      // no wrapped cell among the 5x5x5 and at least 7 cells a side: the
      // minimum-image step is exactly the identity
      wrap = !(nx >= 7 && ny >= 7 && nz >= 7 && cx >= 2 && cx < nx - 2 && cy >= 2 && cy < ny - 2 && cz >= 2 &&
               cz < nz - 2);
      if (lane < 25) {
        const int dz = lane / 5 - 2, dy = lane % 5 - 2;
        int oz = cz + dz;
        oz += ((oz < 0) - (oz >= nz)) * nz;
        int oy = cy + dy;
        oy += ((oy < 0) - (oy >= ny)) * ny;
        const int row = oy * nx + oz * nx * ny;
        const int lo = cx - 2, hi = cx + 2;
        if (lo >= 0 && hi < nx) {
          b0 = cbeg[row + lo];
          e0 = cbeg[row + hi] + ccnt[row + hi];
        } else {
          // the row wraps: cells from the far end first (dx < 0), as the
          // reference's dx loop visits them
          const int cw = row + nx - 1;
          const int ca = lo < 0 ? row + nx + lo : row + lo;
          const int cb = lo < 0 ? row + hi : row + hi - nx;
          b0 = cbeg[ca];
          e0 = cbeg[cw] + ccnt[cw];
          b1 = cbeg[row];
          e1 = cbeg[cb] + ccnt[cb];
        }
      }
    } else if (lane == 0) {
      e0 = R.n;
    }
    const int l0 = e0 - b0, len = l0 + (e1 - b1);
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    const int off = incl - len;                 // this lane's first candidate number
    const int M = __shfl_sync(FULL, incl, 31);  // candidates of the unit
    for (int pg = p0; pg < p1; pg += 32) {
      const int pe = min(p1, pg + 32);
      int cnt_reg = 0;  // lane k: list length so far of particle pg + k
      for (int ch = 0; ch < M; ch += kRunChunk) {
        const int mc = min(kRunChunk, M - ch);
        const int K = (mc + 31) >> 5;  // run length of every lane but the last ones
        __syncwarp();
        // candidate number v of the chunk goes to lane v / K, place v % K:
        // each row lane writes its own parts' candidates, stepping the
        // (lane, place) pair instead of dividing per candidate
        {
          const int v0 = max(off, ch), v1 = min(off + len, ch + mc);
          if (v0 < v1) {
            int qk = (v0 - ch) / K, rk = (v0 - ch) - qk * K;
            for (int v = v0; v < v1; ++v) {
              wrun[qk * kRunStride + rk] = v - off < l0 ? b0 + (v - off) : b1 + (v - off - l0);
              if (++rk == K) {
                rk = 0;
                ++qk;
              }
            }
          }
        }
        __syncwarp();
        const int nrun = min(K, max(0, mc - lane * K));
        for (int p = pg; p < pe; p += 4) {
          // up to four of the cell's particles against the chunk
          float4 rp[4];
          int ip[4];
          const float* crow[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            ip[q] = min(p + q, pe - 1);
            rp[q] = rc[ip[q]];
            crow[q] = s_cs2 + __float_as_int(rp[q].w) * nt;
          }
          unsigned bits[4];
#define RUNS(W, T, MK)                                                                                    \
  {                                                                                                       \
    const T cs[4] = {MK(crow[0]), MK(crow[1]), MK(crow[2]), MK(crow[3])};                                 \
    if (pe - p <= 2)                                                                                      \
      run_tests<W, COH, 2>(run, nrun, rc, rp, ip, cs, R.L[0], R.L[1], R.L[2], R.invL[0], R.invL[1], R.invL[2], bits); \
    else                                                                                                  \
      run_tests<W, COH, 4>(run, nrun, rc, rp, ip, cs, R.L[0], R.L[1], R.L[2], R.invL[0], R.invL[1], R.invL[2], bits); \
  }
#define ONE(c) Cs2One{(c)[0]}
#define TWO(c) Cs2Two{(c)[0], (c)[1]}
#define TAB(c) Cs2Table{(c)}
          if (nt == 1) {
            if (wrap) RUNS(true, Cs2One, ONE) else RUNS(false, Cs2One, ONE)
          } else if (nt == 2) {
            if (wrap) RUNS(true, Cs2Two, TWO) else RUNS(false, Cs2Two, TWO)
          } else {
            if (wrap) RUNS(true, Cs2Table, TAB) else RUNS(false, Cs2Table, TAB)
          }
#undef RUNS
#undef ONE
#undef TWO
#undef TAB
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (p + q < pe) {
              const int cq = __shfl_sync(FULL, cnt_reg, p + q - pg);
              const int tot = run_store(bits[q], run, cq, maxn, lbase, (unsigned)(p + q), stride8);
              if (lane == p + q - pg) cnt_reg = cq + tot;
            }
          }
        }
      }
      if (pg + lane < pe) {
        const int p = pg + lane;
        a.nn[(size_t)R.p0 + p] = (unsigned)min(cnt_reg, maxn);
        a.last_r[(size_t)R.p0 + p] = rc[p];
        wmax = max(wmax, cnt_reg);
      }
    }
  }
  wmax = __reduce_max_sync(FULL, wmax);
  if (lane == 0) atomicMax(s_max, wmax);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int s_max_v = *s_max;
    atomicMax(&S->actual_max_nbrs, s_max_v);
    if (s_max_v > R.max_nbrs) {
      atomicExch(&S->overflow, 1);
      if (COH) s_step_tally += 1ull << kTallyRebuildShift;  // k_batch: the launch stops at the step's end
    }
    __threadfence();
    const unsigned cdone = atomicAdd(&a.rctr[rep], 1u);
    if (s_last) *s_last = cdone == (unsigned)(R.ntiles - 1);
    if (cdone == (unsigned)(R.ntiles - 1)) {
      a.rctr[rep] = 0u;
      if (GRID) S->build_next = 0;
      S->nrebuilds += 1;
      // the replica's lists are complete: released to k_batch's force items
      st_release_u32(reinterpret_cast<unsigned*>(&S->rebuild), 0u);
    }
  }
}

// k_batch's call of the build: kept out of line so that its registers do
// not add to those of k_batch's force path.
__device__ __noinline__ void build_runs_tile_batch(const EngArgs& a, int tile, float* s_cs2, int* s_run, int* s_max) {
  build_runs_tile<true>(a, tile, s_cs2, s_run, s_max);
}
// k_flow's: also reports whether this item's build was the replica's last;
// cell-method replicas claim cells replica-wide (an item queued late finds
// the cells taken and ends at once), others by the block's counter s_next.
__device__ __noinline__ void build_runs_tile_flow(const EngArgs& a, int tile, float* s_cs2, int* s_run, int* s_max,
                                                  int* s_last, int* s_next) {
  if (a.rep[a.tile_rep[tile]].nb_method == NB_CELLS) build_runs_tile<true, true>(a, tile, s_cs2, s_run, s_max, s_last);
  else build_runs_tile<true>(a, tile, s_cs2, s_run, s_max, s_last, s_next);
}

__global__ void __launch_bounds__(kRunWarps * 32) k_rb_build_runs(EngArgs a) {
  __shared__ float s_cs2[kCs2Floats];
  __shared__ int s_run[kRunWarps * 32 * kRunStride];
  __shared__ int s_max, s_next;
  const int rep = a.tile_rep[blockIdx.x];
  if (!rb_active(a, rep)) return;
  if (a.rep[rep].nb_method == NB_CELLS) build_runs_tile<false, true>(a, blockIdx.x, s_cs2, s_run, &s_max);
  else build_runs_tile<false>(a, blockIdx.x, s_cs2, s_run, &s_max, nullptr, &s_next);
}

// ---------------------------------------------------------------------------
// Batched persistent launch (k_batch): many replicas, any number of tiles
// per block, list rebuilds inside the launch.
// ---------------------------------------------------------------------------

// Block-wide exclusive scan of one int per thread (blockDim a multiple of
// 32, at most 1024); returns the thread's exclusive prefix, *total the sum.
// s_w: 33 ints of shared memory.
__device__ __forceinline__ int block_excl_scan(int x, int* s_w, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[wid] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int w = 0; w < nw; ++w) {
      const int t = s_w[w];
      s_w[w] = run;
      run += t;
    }
    s_w[32] = run;
  }
  __syncthreads();
  const int out = s_w[wid] + incl - x;
  *total = s_w[32];
  __syncthreads();
  return out;
}

// The stable cell-key sort of one replica by the calling block, the same
// permutation as the sort kernels (k_rb_clear .. k_rb_permute; RUMD's
// thrust::sort_by_key on (cell key, current slot), Sample.h:174-188):
// count with an arrival rank per cell, exclusive scan of the counts into
// absolute cell starts, scatter, order each bucket by current slot, gather
// r, v, images and ids into the other buffers, flip the parities, and
// publish the sort (release) under `epoch`.  s_w: 33 ints of shared memory.
__device__ __noinline__ void block_sort(const EngArgs& a, int rep, unsigned epoch, int* s_w) {
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  const int tid = threadIdx.x, bd = blockDim.x;
  if (R.nb_method == NB_CELLS) {
    const int rb = __ldcg(&S->rbuf), ab = __ldcg(&S->abuf);
    const int n = R.n, ncell = R.ncell;
    const size_t p0 = (size_t)R.p0;
    int* cnt = a.cnt + R.cell0;
    int* cst = a.cstart + R.cell0;
    for (int c = tid; c < ncell; c += bd) cnt[c] = 0;
    __syncthreads();
    // cell key (calculateCellIndices, NeighborList.cu:1142-1172) and arrival
    // rank; a thread keeps kSortIlp particles' loads and atomics in flight
    constexpr int kSortIlp = 8;
    for (int i0 = tid; i0 < n; i0 += bd * kSortIlp) {
      float4 r[kSortIlp];
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) {
        const int i = i0 + u * bd;
        r[u] = i < n ? a.r[rb][p0 + i] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      int key[kSortIlp], sl[kSortIlp];
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) {
        key[u] = cell_coord(r[u].x, R.invL[0], R.nc[0]) + cell_coord(r[u].y, R.invL[1], R.nc[1]) * R.nc[0] +
                 cell_coord(r[u].z, R.invL[2], R.nc[2]) * R.nc[0] * R.nc[1];
        sl[u] = i0 + u * bd < n ? atomicAdd(&cnt[key[u]], 1) : 0;
      }
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) {
        const int i = i0 + u * bd;
        if (i < n) {
          a.key[p0 + i] = key[u];
          a.slot[p0 + i] = sl[u];
        }
      }
    }
    __syncthreads();
    // absolute first slot of every cell: thread t owns the cells
    // [t K, (t + 1) K), loads their counts together, and one block scan of
    // the threads' totals gives every run's first slot
    const int K = (ncell + bd - 1) / bd;
    {
      constexpr int kCh = 8;
      const int c0 = tid * K, c1 = min(ncell, c0 + K);
      int tot = 0;
      for (int cb = c0; cb < c1; cb += kCh) {
        int x[kCh];
#pragma unroll
        for (int u = 0; u < kCh; ++u) x[u] = cb + u < c1 ? cnt[cb + u] : 0;
#pragma unroll
        for (int u = 0; u < kCh; ++u) tot += x[u];
      }
      int all;
      int run = block_excl_scan(tot, s_w, &all);
      for (int cb = c0; cb < c1; cb += kCh) {
        int x[kCh];
#pragma unroll
        for (int u = 0; u < kCh; ++u) x[u] = cb + u < c1 ? cnt[cb + u] : 0;
#pragma unroll
        for (int u = 0; u < kCh; ++u)
          if (cb + u < c1) {
            cst[cb + u] = run;
            run += x[u];
          }
      }
    }
    __syncthreads();
    for (int i0 = tid; i0 < n; i0 += bd * kSortIlp) {
      int key[kSortIlp], sl[kSortIlp];
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) {
        const int i = i0 + u * bd;
        key[u] = i < n ? a.key[p0 + i] : 0;
        sl[u] = i < n ? a.slot[p0 + i] : 0;
      }
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) key[u] = cst[key[u]];
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) {
        const int i = i0 + u * bd;
        if (i < n) a.order[p0 + key[u] + sl[u]] = (unsigned)i;
      }
    }
    __syncthreads();
    // each bucket by current slot: the result is the stable sort by key.  A
    // thread takes its run of cells kFixCells at a time; buckets of up to
    // kFixRegs slots are loaded together into registers, sorted by an
    // odd-even transposition network and stored back (larger ones:
    // insertion sort in place)
    {
      constexpr int kFixCells = 2;
      const int c0 = tid * K, c1 = min(ncell, c0 + K);
      for (int cb = c0; cb < c1; cb += kFixCells) {
        int m[kFixCells], b[kFixCells];
        unsigned x[kFixCells][kFixRegs];
#pragma unroll
        for (int u = 0; u < kFixCells; ++u) {
          const int c = cb + u;
          m[u] = c < c1 ? cnt[c] : 0;
          b[u] = c < c1 ? cst[c] : 0;
        }
#pragma unroll
        for (int u = 0; u < kFixCells; ++u)
#pragma unroll
          for (int k = 0; k < kFixRegs; ++k)
            x[u][k] = (k < m[u] && m[u] <= kFixRegs && m[u] > 1) ? a.order[p0 + b[u] + k] : 0xffffffffu;
#pragma unroll
        for (int u = 0; u < kFixCells; ++u) {
          if (m[u] <= 1) continue;
          if (m[u] <= kFixRegs) {
#pragma unroll
            for (int r = 0; r < kFixRegs; ++r)
#pragma unroll
              for (int k = r & 1; k + 1 < kFixRegs; k += 2) {
                const unsigned lo = min(x[u][k], x[u][k + 1]), hi = max(x[u][k], x[u][k + 1]);
                x[u][k] = lo;
                x[u][k + 1] = hi;
              }
#pragma unroll
            for (int k = 0; k < kFixRegs; ++k)
              if (k < m[u]) a.order[p0 + b[u] + k] = x[u][k];
          } else {
            unsigned* o = a.order + p0 + b[u];
            for (int q = 1; q < m[u]; ++q) {
              const unsigned v = o[q];
              int k = q - 1;
              while (k >= 0 && o[k] > v) {
                o[k + 1] = o[k];
                --k;
              }
              o[k + 1] = v;
            }
          }
        }
      }
    }
    __syncthreads();
    // ParticleData::UpdateAfterSorting (ParticleData.cu:493-528)
    for (int s0 = tid; s0 < n; s0 += bd * kSortIlp) {
      unsigned o[kSortIlp];
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) {
        const int sl = s0 + u * bd;
        o[u] = sl < n ? a.order[p0 + sl] : 0u;
      }
#pragma unroll
      for (int u = 0; u < kSortIlp; ++u) {
        const int sl = s0 + u * bd;
        if (sl < n) {
          const size_t gs = p0 + sl, go = p0 + o[u];
          a.r[rb ^ 1][gs] = a.r[rb][go];
          a.v[ab ^ 1][gs] = a.v[ab][go];
          a.im[ab ^ 1][gs] = a.im[ab][go];
          a.uidx[ab ^ 1][gs] = a.uidx[ab][go];
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      S->rbuf = rb ^ 1;
      S->abuf = ab ^ 1;
    }
  }
  if (tid == 0) {
    S->actual_max_nbrs = 0;  // the per-build maximum (k_rb_clear)
    __threadfence();
    st_release_u32(&S->sort_done, epoch);
  }
  __syncthreads();
}

// Bounded wait of thread 0 until *p == want (acquire); false when it gave up.
__device__ __forceinline__ bool wait_eq_u32(const unsigned* p, unsigned want) {
  for (unsigned it = 0; ld_acquire_u32(p) != want; ++it) {
    if (it >= kWaitPolls) return false;
    __nanosleep(64);
  }
  return true;
}

// Bounded wait of thread 0 until *p >= want (acquire); false when it gave up.
__device__ __forceinline__ bool wait_ge_u32(const unsigned* p, unsigned want) {
  for (unsigned it = 0; ld_acquire_u32(p) < want; ++it) {
    if (it >= kWaitPolls) return false;
    __nanosleep(64);
  }
  return true;
}

// ---------------------------------------------------------------------------
// The split sort of k_batch: the stable cell-key sort of a large replica as
// phase items that any blocks take, one item per tile (or per the tile's
// share of the cells), so that a 32k-particle replica sorts in a few
// microseconds per phase instead of one block running all of it.  The
// phases are those of block_sort and of the sort kernels:
//   0 clear the cell counts of a chunk of cells        (C items)
//   1 cell key and arrival rank of a tile's particles  (C items)
//   2 absolute cell starts (one block scan)            (1 item)
//   3 scatter a tile's particles to their buckets      (C items)
//   4 order a chunk of cells' buckets by current slot
//     and gather r, v, images and ids of their slots   (C items)
// where C is the replica's tile count.  Each finished item adds one to the
// replica's sort_items (acquire-release); an item of phase p waits (bounded)
// until the items of the earlier phases are all counted: split_sort_need.
// The last item of phase 4 flips the buffer parities, resets the count and
// publishes the sort under the step's epoch, as block_sort does.  The
// permutation is the same stable sort.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned split_sort_need(int phase, unsigned C) {
  return phase == 0 ? 0u : phase == 1 ? C : phase == 2 ? 2u * C : phase == 3 ? 2u * C + 1u : 3u * C + 1u;
}
__device__ __forceinline__ unsigned split_sort_items(unsigned C) { return 4u * C + 1u; }

__device__ __forceinline__ int cell_key_of(const RepDev& R, const float4& r) {
  // calculateCellIndices (NeighborList.cu:1142-1172)
  return cell_coord(r.x, R.invL[0], R.nc[0]) + cell_coord(r.y, R.invL[1], R.nc[1]) * R.nc[0] +
         cell_coord(r.z, R.invL[2], R.nc[2]) * R.nc[0] * R.nc[1];
}

// Orders bucket o[0, m) ascending (slot indices): small buckets in registers
// by an odd-even transposition network, larger ones by insertion in place.
__device__ __forceinline__ void order_bucket(unsigned* o, int m) {
  if (m <= 1) return;
  if (m <= kFixRegs) {
    unsigned x[kFixRegs];
#pragma unroll
    for (int k = 0; k < kFixRegs; ++k) x[k] = k < m ? o[k] : 0xffffffffu;
#pragma unroll
    for (int r = 0; r < kFixRegs; ++r)
#pragma unroll
      for (int k = r & 1; k + 1 < kFixRegs; k += 2) {
        const unsigned lo = min(x[k], x[k + 1]), hi = max(x[k], x[k + 1]);
        x[k] = lo;
        x[k + 1] = hi;
      }
#pragma unroll
    for (int k = 0; k < kFixRegs; ++k)
      if (k < m) o[k] = x[k];
    return;
  }
  for (int q = 1; q < m; ++q) {
    const unsigned v = o[q];
    int k = q - 1;
    while (k >= 0 && o[k] > v) {
      o[k + 1] = o[k];
      --k;
    }
    o[k + 1] = v;
  }
}

// One item of phase `phase` (chunk: the tile / cell chunk index within the
// replica).  rb, ab: the replica's buffer parities before the sort.
__device__ __noinline__ void split_sort_item(const EngArgs& a, int rep, int phase, int chunk, int rb, int ab,
                                             int* s_w) {
  const RepDev& R = a.rep[rep];
  const size_t p0 = (size_t)R.p0;
  int* cnt = a.cnt + R.cell0;
  int* cst = a.cstart + R.cell0;
  const int tid = threadIdx.x, bd = blockDim.x;
  const int ch = cell_chunk(R);
  const int c0 = min(R.ncell, chunk * ch), c1 = min(R.ncell, c0 + ch);
  const int tile = R.tile0 + chunk;
  const int i0 = a.tile_first[tile];
  const int i1 = chunk + 1 < R.ntiles ? a.tile_first[tile + 1] : R.n;
  if (phase == 0) {
    for (int c = c0 + tid; c < c1; c += bd) cnt[c] = 0;
  } else if (phase == 1) {
    for (int i = i0 + tid; i < i1; i += bd) {
      const int key = cell_key_of(R, a.r[rb][p0 + i]);
      a.key[p0 + i] = key;
      a.slot[p0 + i] = atomicAdd(&cnt[key], 1);
    }
  } else if (phase == 2) {
    // absolute first slot of every cell: thread t owns a run of cells, one
    // block scan of the runs' totals
    const int ncell = R.ncell;
    const int K = (ncell + bd - 1) / bd;
    constexpr int kCh = 8;
    const int e0 = tid * K, e1 = min(ncell, e0 + K);
    int tot = 0;
    for (int cb = e0; cb < e1; cb += kCh) {
      int x[kCh];
#pragma unroll
      for (int u = 0; u < kCh; ++u) x[u] = cb + u < e1 ? cnt[cb + u] : 0;
#pragma unroll
      for (int u = 0; u < kCh; ++u) tot += x[u];
    }
    int all;
    int run = block_excl_scan(tot, s_w, &all);
    for (int cb = e0; cb < e1; cb += kCh) {
      int x[kCh];
#pragma unroll
      for (int u = 0; u < kCh; ++u) x[u] = cb + u < e1 ? cnt[cb + u] : 0;
#pragma unroll
      for (int u = 0; u < kCh; ++u)
        if (cb + u < e1) {
          cst[cb + u] = run;
          run += x[u];
        }
    }
  } else if (phase == 3) {
    for (int i = i0 + tid; i < i1; i += bd) a.order[p0 + cst[a.key[p0 + i]] + a.slot[p0 + i]] = (unsigned)i;
  } else {
    // buckets of the chunk's cells by current slot (= the stable sort), then
    // the gather of their slots (ParticleData::UpdateAfterSorting,
    // ParticleData.cu:493-528)
    for (int c = c0 + tid; c < c1; c += bd) order_bucket(a.order + p0 + cst[c], cnt[c]);
    __syncthreads();
    const int s0 = c0 < R.ncell ? cst[c0] : R.n;
    const int s1 = c1 < R.ncell ? cst[c1] : R.n;
    for (int sl = s0 + tid; sl < s1; sl += bd) {
      const size_t gs = p0 + sl, go = p0 + a.order[gs];
      a.r[rb ^ 1][gs] = a.r[rb][go];
      a.v[ab ^ 1][gs] = a.v[ab][go];
      a.im[ab ^ 1][gs] = a.im[ab][go];
      a.uidx[ab ^ 1][gs] = a.uidx[ab][go];
    }
  }
}

constexpr int kBatchMaxRep = 1024;   // replicas whose rebuild list a block holds in shared memory
// Tiles of the other replicas claimed between the sorts and the builds: two
// thirds of the tiles (on the 256-replica batch: 566, 548, 535 us per step
// for a third, a half, two thirds), but no more than the tiles left once the
// listed replicas' are taken out.
__device__ __forceinline__ int batch_first_tiles(int ntiles, int t2) {
  return min(2 * ntiles / 3, max(0, ntiles - t2));
}
constexpr int kBatchMaxN = 65536;    // particles per replica (one block sorts a replica)
constexpr int kBatchEpochSteps = 4096;  // epochs: launch generation * this + step + 1

// Shared memory of k_batch after the tile's dynamic region: the step's
// rebuild list (replica ids) and the prefix of their tile counts, and a bit
// per replica that is on it.
struct BatchShared {
  int list[kBatchMaxRep];
  int pref[kBatchMaxRep + 1];
  int spref[kBatchMaxRep + 1];  // prefix of the split-sort chunks (tiles of the replicas sorted in phases)
  int slist[kBatchMaxRep];      // replicas sorted by one block each
  int blist[kBatchMaxRep];      // replicas sorted in phases
  unsigned bits[kBatchMaxRep / 32];
  int scan[33];
};

// Every MD step of many replicas in one cooperative launch.  Per step the
// blocks claim work items in ticket order (one atomic counter):
//   1. the stable sort of each replica on the step's rebuild list (one block
//      sorts one replica, block_sort);
//   2. the fused force + Nose-Hoover tile of every tile of the other
//      replicas (force_tile, as k_force);
//   3. the list build of every tile of the listed replicas (build_runs_tile),
//      each after its replica's sort (bounded wait on sort_done);
//   4. their fused force + Nose-Hoover tiles, each after all of its
//      replica's builds (bounded wait on the replica's rebuild flag, which
//      the last build clears with release).
// Every wait is on an item with an earlier ticket, taken by a running block
// that does not wait on later items, so the claims always progress.  A
// replica's arithmetic is that of the other paths (the same sort, list,
// per-tile sums and reduction tree), whatever block runs which item.  The
// replica finalizers put the replicas whose lists are due on the next step's
// rebuild list (two lists alternated by step parity) and tally "steps left";
// one grid barrier ends each step, after which every block takes the same
// decision: stop when no replica has steps left, the budget is spent, a list
// overflowed (the host repairs it) or a wait gave up.
template <int TP>
__global__ void __maxnreg__(64) k_batch(EngArgs a, cudaGraphConditionalHandle h_loop) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ double s_blk[kNPart], s_tot[kNPart];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ unsigned s_rows;
  __shared__ int s_go, s_item, s_ok, s_max;
  // the loop's bookkeeping, kept out of registers for the force path: the
  // launch generation, the step budget, the tickets of the steps so far, the
  // step barrier words' totals, the step's rebuild-list size and its tiles
  __shared__ unsigned s_gen, s_base;
  __shared__ int s_budget, s_nf, s_t2;
  __shared__ int s_ns, s_nb, s_cs;  // the step's one-block sorts, split sorts and their chunks
  __shared__ int s_ntiles, s_nrep;  // the layout in effect (not the captured one)
  __shared__ unsigned long long s_seen[2];
  BatchShared* bs = reinterpret_cast<BatchShared*>(s_dyn + a.bshared_off);
  PersistCtl* c = a.pctl;
  if (threadIdx.x == 0) {
    s_ntiles = __ldcg(&c->lay_ntiles);
    s_nrep = __ldcg(&c->lay_nrep);
    s_go = __ldcg(&c->err) == 0;
    if (!s_go && blockIdx.x == 0) set_loop(h_loop, 0u);
  }
  __syncthreads();
  // setup barrier; its last block zeroes the step words and the tickets and
  // puts the replicas whose lists are due on the first step's rebuild list
  if (s_go) {
    if (threadIdx.x == 0) {
      s_gen = ld_acquire_u32(&c->gen);
      const unsigned long long nnow = atom_add_acq_rel_u64(&c->arrive, 1ull) + 1ull;
      s_item = (nnow & kTallyArriveMask) == gridDim.x;
    }
    __syncthreads();
    if (s_item) {
      if (threadIdx.x == 0) {
        c->word[0] = 0ull;
        c->word[1] = 0ull;
        c->ticket = 0u;
        c->readers = 0u;
        c->fcnt[0] = c->fcnt[1] = 0;
        c->ftiles[0] = c->ftiles[1] = 0;
        *a.any_rebuild = 0;
      }
      __syncthreads();
      for (int r = threadIdx.x; r < s_nrep; r += blockDim.x) {
        const RepState* S = a.st + r;
        if (a.rep[r].active && S->rebuild && !S->overflow && S->steps_left > 0) {
          const int pos = atomicAdd(&c->fcnt[0], 1);
          a.flist[pos] = r;
          atomicAdd(&c->ftiles[0], a.rep[r].ntiles);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        c->arrive = 0ull;
        __threadfence();
        st_release_u32(&c->gen, s_gen + 1u);
      }
    } else if (threadIdx.x == 0) {
      s_go = barrier_wait(c, s_gen, h_loop);
    }
    if (threadIdx.x == 0) {
      s_budget = __ldcg(&c->budget);
      s_base = 0u;
      s_seen[0] = s_seen[1] = 0ull;
    }
    __syncthreads();
  }
  for (int step = 0; s_go; ++step) {
    const int par = step & 1;
    // the step's rebuild list: every block reads the same one (its last
    // reader clears it for reuse two steps on)
    if (threadIdx.x == 0) {
      s_step_tally = 0ull;
      s_nf = min(__ldcg(&c->fcnt[par]), kBatchMaxRep);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kBatchMaxRep / 32; k += blockDim.x) bs->bits[k] = 0u;
    __syncthreads();
    {
      const int nf = s_nf;
      int run = 0, srun = 0, brun = 0;
      for (int k0 = 0; k0 < nf; k0 += blockDim.x) {
        const int k = k0 + threadIdx.x;
        const int r = k < nf ? __ldcg(a.flist + (size_t)par * a.rctr_half + k) : 0;
        const int nt = k < nf ? a.rep[r].ntiles : 0;
        // replicas of at least split_tiles tiles (cell method) sort in phases
        const int big = (k < nf && nt >= a.split_tiles && a.rep[r].nb_method == NB_CELLS) ? 1 : 0;
        int tot, stot, btot;
        const int ex = block_excl_scan(nt, bs->scan, &tot);
        const int sex = block_excl_scan(big ? nt : 0, bs->scan, &stot);
        const int bex = block_excl_scan(big, bs->scan, &btot);
        if (k < nf) {
          bs->list[k] = r;
          bs->pref[k] = run + ex;
          bs->spref[k] = srun + sex;
          if (big) bs->blist[brun + bex] = r;
          else bs->slist[k - (brun + bex)] = r;
          atomicOr(&bs->bits[r >> 5], 1u << (r & 31));
        }
        run += tot;
        srun += stot;
        brun += btot;
      }
      if (threadIdx.x == 0) {
        bs->pref[nf] = run;
        bs->spref[nf] = srun;
        s_cs = srun;
        s_nb = brun;
        s_ns = nf - brun;
        s_t2 = run;  // tiles of the listed replicas
        __threadfence();
        if (atomicAdd(&c->readers, 1u) == gridDim.x - 1) {
          c->readers = 0u;
          c->fcnt[par] = 0;
          c->ftiles[par] = 0;
        }
      }
    }
    __syncthreads();
    // claim items until the step's are gone (each block overshoots once).
    // Ticket order: [one-block sorts] [split sorts: phases 0, 1, 2]
    // [a third of the first q tiles] [split phase 3] [a third] [split phase 4]
    // [the last third] [builds] [the remaining tiles] [the listed replicas'
    // force tiles]: force tiles of the other replicas between the split
    // phases keep blocks busy while a phase's items complete, the first
    // tiles give the sorts time, the remaining ones the builds.  Every wait
    // is on items with earlier tickets.
    for (;;) {
      if (threadIdx.x == 0) s_item = (int)(atomicAdd(&c->ticket, 1u) - s_base);
      __syncthreads();
      const unsigned it = (unsigned)s_item;
      const int t2 = s_t2, nf = s_nf, ntiles = s_ntiles;
      const int ns = s_ns, nb = s_nb, cs = s_cs;
      const int so = ns + 4 * cs + nb;  // sort items
      const int q = batch_first_tiles(ntiles, t2);
      const unsigned epoch = s_gen * kBatchEpochSteps + (unsigned)step + 1u;
      if (it >= (unsigned)(so + ntiles + 2 * t2)) break;
      // the sort segment [0, so + q): split phases 0-2 end at e2, then a
      // third of the first tiles, phase 3 from b3, a third, phase 4 from b4,
      // the last third from e4
      const int f1 = q / 3, f2 = q / 3;
      const int e2 = ns + 2 * cs + nb, b3 = e2 + f1, b4 = b3 + cs + f2, e4 = b4 + cs;
      int phase = -1, j = 0, tile = -1;
      if (it < (unsigned)ns) {
        phase = 5;  // a one-block sort
      } else if (it < (unsigned)e2) {
        j = (int)it - ns;
        if (j < cs) phase = 0;
        else if ((j -= cs) < cs) phase = 1;
        else { j -= cs; phase = 2; }
      } else if (it < (unsigned)b3) {
        tile = (int)it - e2;
      } else if (it < (unsigned)(b3 + cs)) {
        j = (int)it - b3;
        phase = 3;
      } else if (it < (unsigned)b4) {
        tile = f1 + ((int)it - b3 - cs);
      } else if (it < (unsigned)e4) {
        j = (int)it - b4;
        phase = 4;
      } else if (it < (unsigned)(so + q)) {
        tile = f1 + f2 + ((int)it - e4);
      } else if (it >= (unsigned)(so + q + t2) && it < (unsigned)(so + ntiles + t2)) {
        tile = (int)it - so - t2;
      }
      const bool tile_item = tile >= 0;
      if (phase == 5) {
        block_sort(a, bs->slist[it], epoch, bs->scan);
      } else if (phase >= 0) {
        // a split-sort item: its replica and chunk
        int r, chunk = 0;
        if (phase == 2) {
          r = bs->blist[j];
        } else {
          int lo = 0, hi = nf - 1;  // the listed replica whose chunk range holds j
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (bs->spref[mid] <= j) lo = mid;
            else hi = mid - 1;
          }
          r = bs->list[lo];
          chunk = j - bs->spref[lo];
        }
        RepState* S = a.st + r;
        const unsigned C = (unsigned)a.rep[r].ntiles;
        if (threadIdx.x == 0) {
          s_ok = wait_ge_u32(&S->sort_items, split_sort_need(phase, C));
          if (!s_ok) {
            atomicExch(&c->err, 1);
            s_step_tally += 1ull << kTallyRebuildShift;
          }
          s_max = __ldcg(&S->rbuf) | (__ldcg(&S->abuf) << 1);  // the parities before the sort
        }
        __syncthreads();
        if (s_ok) {
          split_sort_item(a, r, phase, chunk, s_max & 1, s_max >> 1, bs->scan);
          __syncthreads();
          if (threadIdx.x == 0) {
            const unsigned done = atom_add_acq_rel(&S->sort_items, 1u) + 1u;
            if (done == split_sort_items(C)) {
              // the last item: flip the parities, reset the count, publish
              S->rbuf = (s_max & 1) ^ 1;
              S->abuf = (s_max >> 1) ^ 1;
              S->actual_max_nbrs = 0;  // the per-build maximum (k_rb_clear)
              S->sort_items = 0u;
              __threadfence();
              st_release_u32(&S->sort_done, epoch);
            }
          }
        }
      } else if (tile_item) {
        const int r = a.tile_rep[tile];
        if (!((bs->bits[r >> 5] >> (r & 31)) & 1u))
          force_tile<TP, true, false, FM_STREAMED, false, true>(a, tile, s_dyn, s_blk, s_tot, s_bar, s_rows, nullptr,
                                                                0, nullptr, nullptr, nullptr, par ^ 1);
      } else {
        const bool build = it < (unsigned)(so + q + t2);
        const int k = build ? (int)it - so - q : (int)it - so - ntiles - t2;
        int lo = 0, hi = nf - 1;  // the listed replica holding flagged tile k
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (bs->pref[mid] <= k) lo = mid;
          else hi = mid - 1;
        }
        const int r = bs->list[lo];
        const int tile = a.rep[r].tile0 + (k - bs->pref[lo]);
        RepState* S = a.st + r;
        if (threadIdx.x == 0) {
          s_ok = build ? wait_eq_u32(&S->sort_done, epoch)
                       : wait_eq_u32(reinterpret_cast<const unsigned*>(&S->rebuild), 0u);
          if (!s_ok) {
            // recorded for the host and tallied with the barrier arrival, so
            // that every block stops after this step
            atomicExch(&c->err, 1);
            s_step_tally += 1ull << kTallyRebuildShift;
          }
        }
        __syncthreads();
        if (s_ok) {
          if (build) {
            float* s_cs2 = reinterpret_cast<float*>(s_dyn);
            int* s_run = reinterpret_cast<int*>(s_dyn + kCs2Floats * sizeof(float));
            build_runs_tile_batch(a, tile, s_cs2, s_run, &s_max);
          } else {
            force_tile<TP, true, false, FM_STREAMED, false, true>(a, tile, s_dyn, s_blk, s_tot, s_bar, s_rows,
                                                                  nullptr, 0, nullptr, nullptr, nullptr, par ^ 1);
          }
        }
      }
      __syncthreads();
    }
    // step barrier: arrival + "steps left" and overflow tallies
    if (threadIdx.x == 0) {
      s_base += (unsigned)(s_ns + 4 * s_cs + s_nb + s_ntiles + 2 * s_t2) + gridDim.x;
      const int budget = --s_budget;
      const unsigned long long mine = 1ull + s_step_tally;
      const unsigned long long now = atom_add_acq_rel_u64(&c->word[par], mine) + mine;
      const unsigned long long base_w = s_seen[par];
      const bool last = ((now - base_w) & kTallyArriveMask) == gridDim.x;
      unsigned long long tot = now;
      int ok = 1;
      if (!last) {
        for (unsigned it = 0;; ++it) {
          tot = ld_acquire_u64(&c->word[par]);
          if (((tot - base_w) & kTallyArriveMask) == gridDim.x) break;
          if (it >= kBarrierPolls) {
            atomicExch(&c->err, 1);
            set_loop(h_loop, 0u);
            ok = 0;
            break;
          }
          __nanosleep(32);
        }
      }
      s_seen[par] = tot;
      const unsigned long long d = tot - base_w;
      const unsigned more = (unsigned)((d >> kTallyMoreShift) & kTallyField);
      // list overflows and waits that gave up: the host repairs or reports
      const unsigned stop = (unsigned)((d >> kTallyRebuildShift) & kTallyField);
      // steps per launch: the epochs' and the tally fields' range, and the
      // 32-bit ticket counter (at most nrep + 7 ntiles + grid tickets a step)
      const unsigned per_step = (unsigned)s_nrep + 7u * (unsigned)s_ntiles + gridDim.x;
      const int cap = min(min(kBatchEpochSteps - 2, (int)(kTallyField / (unsigned)(s_nrep + 1))),
                          (int)min(0x7fffffffu, 0xffffffffu / per_step));
      const int go = ok && stop == 0 && more > 0 && budget > 0 && step + 1 < cap;
      if (last && !go) {
        c->budget = budget;
        set_loop(h_loop, (stop == 0 && more > 0 && budget > 0) ? 1u : 0u);
      }
      s_go = go;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// k_flow: the same steps as k_batch, each replica stepping on its own.
// Work items go through one queue (a ring of slots in global memory); an
// item is queued only when everything it reads is complete, so no item
// waits:
//   * a replica's step: its force tiles (fused force + Nose-Hoover); the
//     replica's finalizer (the last tile's block) queues the next step's
//     items -- force tiles, or the sort when its list is due -- or, when the
//     replica has no steps left or has run the launch's budget, retires it
//     from the launch;
//   * a rebuild: the sort (one item for replicas below the split threshold,
//     else the five split phases, each phase's last item queueing the next),
//     then one build item per tile; the last build queues the force tiles.
// Items of one phase count down the replica's flow_left; the block that
// finishes the last queues the next phase.  Replicas therefore advance at
// their own pace: a large replica's rebuild no longer holds every other
// replica at a step barrier.  The queue's tickets are 64-bit and monotone
// across launches; a slot is published by a release store of its ticket + 1,
// and a consumer polls (bounded) for it, or for no replica left stepping,
// which ends the launch.  The arithmetic of a replica is that of k_batch and
// the per-step path (the same items), so results agree bit for bit.
// ---------------------------------------------------------------------------
constexpr unsigned kFlowForce = 0u, kFlowSort1 = 1u, kFlowSplit = 2u, kFlowBuild = 3u;

// Queues items idx = 0 .. n-1 of kind/phase for replica rep (all threads of
// the block; the caller has published the replica's state with a fence).
__device__ __forceinline__ void flow_push(const EngArgs& a, int rep, unsigned kind, unsigned phase, int n,
                                          unsigned long long* s_t0) {
  PersistCtl* c = a.pctl;
  if (threadIdx.x == 0) *s_t0 = atomicAdd(&c->qtail, (unsigned long long)n);
  __syncthreads();
  const unsigned long long t0 = *s_t0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const unsigned long long t = t0 + (unsigned long long)k;
    const unsigned slot = (unsigned)(t % a.qcap);
    a.fq[slot] = make_int2(rep, (int)((kind << 28) | (phase << 20) | (unsigned)k));
    st_release_u64(&a.fseq[slot], t + 1ull);
  }
  __syncthreads();
}

// A replica's next items: its force tiles, or (rebuild) the start of its sort.
__device__ void flow_start_step(const EngArgs& a, int rep, bool rebuild, unsigned long long* s_t0) {
  const RepDev& R = a.rep[rep];
  RepState* S = a.st + rep;
  unsigned kind = kFlowForce;
  int n = R.ntiles;
  if (rebuild) {
    if (R.nb_method == NB_CELLS && R.ntiles >= a.split_tiles) {
      kind = kFlowSplit;  // phase 0: one item per chunk
    } else {
      kind = kFlowSort1;
      n = 1;
    }
  }
  if (threadIdx.x == 0) {
    S->flow_left = n;
    __threadfence();
  }
  __syncthreads();
  flow_push(a, rep, kind, 0u, n, s_t0);
}

// Counts one finished item of the replica's phase; true in every thread of
// the block that finished the phase's last.
__device__ __forceinline__ bool flow_item_done(RepState* S, int* s_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    *s_flag = atomicSub(&S->flow_left, 1) == 1;
  }
  __syncthreads();
  return *s_flag != 0;
}

__device__ __forceinline__ void flow_retire(const EngArgs& a) {
  if (threadIdx.x == 0) {
    __threadfence();
    atomicSub(&a.pctl->active, 1);
  }
}

template <int TP>
__global__ void __maxnreg__(64) k_flow(EngArgs a, cudaGraphConditionalHandle h_loop) {
  extern __shared__ __align__(128) unsigned char s_dyn[];
  __shared__ double s_blk[kNPart], s_tot[kNPart];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ unsigned s_rows;
  __shared__ int s_go, s_last, s_max, s_flag, s_rep, s_code;
  __shared__ unsigned s_gen;
  __shared__ unsigned long long s_t0;
  __shared__ int s_scan[33];
  PersistCtl* c = a.pctl;
  if (threadIdx.x == 0) {
    s_go = __ldcg(&c->err) == 0;
    if (!s_go && blockIdx.x == 0) set_loop(h_loop, 0u);
  }
  __syncthreads();
  if (!s_go) return;
  // setup barrier; its last block aligns the queue's tickets, starts every
  // replica that has steps left and releases the others
  if (threadIdx.x == 0) {
    s_gen = ld_acquire_u32(&c->gen);
    const unsigned long long nnow = atom_add_acq_rel_u64(&c->arrive, 1ull) + 1ull;
    s_last = (nnow & kTallyArriveMask) == gridDim.x;
  }
  __syncthreads();
  if (s_last) {
    const int nrep = __ldcg(&c->lay_nrep);
    if (threadIdx.x == 0) {
      const unsigned long long h = __ldcg(&c->qhead), t = __ldcg(&c->qtail);
      c->qhead = c->qtail = h > t ? h : t;
      c->active = 0;
      c->ran = 0;
      c->exited = 0u;
      *a.any_rebuild = 0;
    }
    __syncthreads();
    for (int r = 0; r < nrep; ++r) {
      RepState* S = a.st + r;
      if (threadIdx.x == 0)
        s_flag = a.rep[r].active && !S->overflow && S->steps_left > 0 && a.rep[r].ntiles > 0;
      __syncthreads();
      if (s_flag) {
        if (threadIdx.x == 0) {
          S->launch_steps = 0;
          c->active += 1;
        }
        flow_start_step(a, r, S->rebuild != 0, &s_t0);
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      c->arrive = 0ull;
      __threadfence();
      st_release_u32(&c->gen, s_gen + 1u);
    }
  } else if (threadIdx.x == 0) {
    s_go = barrier_wait(c, s_gen, h_loop);
  }
  __syncthreads();
  while (s_go) {
    // the next item, or the end of the launch
    if (threadIdx.x == 0) {
      const unsigned long long t = atomicAdd(&c->qhead, 1ull);
      const unsigned slot = (unsigned)(t % a.qcap);
      int got = 0;
      for (unsigned it = 0;; ++it) {
        if (ld_acquire_u64(&a.fseq[slot]) == t + 1ull) {
          const int2 q = __ldcg(a.fq + slot);
          s_rep = q.x;
          s_code = q.y;
          got = 1;
          break;
        }
        if (ld_acquire_u32(reinterpret_cast<const unsigned*>(&c->active)) == 0u || __ldcg(&c->err)) break;
        if (it >= kBarrierPolls) {
          atomicExch(&c->err, 1);
          break;
        }
        __nanosleep(32);
      }
      s_go = got;
    }
    __syncthreads();
    if (!s_go) break;
    const int rep = s_rep;
    const unsigned code = (unsigned)s_code;
    const unsigned kind = code >> 28, phase = (code >> 20) & 0xffu;
    const int idx = (int)(code & 0xfffffu);
    const RepDev& R = a.rep[rep];
    RepState* S = a.st + rep;
    if (kind == kFlowForce) {
      if (threadIdx.x == 0) s_fin = -1;
      __syncthreads();
      force_tile<TP, true, false, FM_STREAMED, false, true>(a, R.tile0 + idx, s_dyn, s_blk, s_tot, s_bar, s_rows,
                                                            nullptr, 0, nullptr, nullptr, nullptr, kFlowPar);
      __syncthreads();
      const int fin = s_fin;
      if (fin == 0) flow_retire(a);
      else if (fin > 0) flow_start_step(a, rep, fin == 2, &s_t0);
    } else if (kind == kFlowSort1 || kind == kFlowSplit) {
      if (kind == kFlowSort1) {
        block_sort(a, rep, 0u, s_scan);
      } else {
        if (threadIdx.x == 0) s_max = __ldcg(&S->rbuf) | (__ldcg(&S->abuf) << 1);
        __syncthreads();
        split_sort_item(a, rep, (int)phase, idx, s_max & 1, s_max >> 1, s_scan);
      }
      if (flow_item_done(S, &s_flag)) {
        unsigned nkind = kFlowBuild, nphase = 0u;
        int n = R.ntiles;
        if (kind == kFlowSplit && phase < 4u) {
          nkind = kFlowSplit;
          nphase = phase + 1u;
          n = nphase == 2u ? 1 : R.ntiles;
        }
        if (threadIdx.x == 0) {
          if (kind == kFlowSplit && phase == 4u) {
            // the sort is complete: flip the parities (the per-build maximum
            // starts again, as k_rb_clear does)
            S->rbuf = (s_max & 1) ^ 1;
            S->abuf = (s_max >> 1) ^ 1;
            S->actual_max_nbrs = 0;
          }
          S->flow_left = n;
          __threadfence();
        }
        __syncthreads();
        flow_push(a, rep, nkind, nphase, n, &s_t0);
      }
    } else {
      float* s_cs2 = reinterpret_cast<float*>(s_dyn);
      int* s_run = reinterpret_cast<int*>(s_dyn + kCs2Floats * sizeof(float));
      build_runs_tile_flow(a, R.tile0 + idx, s_cs2, s_run, &s_max, &s_last, &s_flag);  // s_flag: cell claims
      __syncthreads();
      if (s_last) {
        // the replica's lists are complete: its force tiles, unless a list
        // overflowed (the replica leaves the launch; the host enlarges it)
        if (threadIdx.x == 0) s_flag = __ldcg(&S->overflow) != 0;
        __syncthreads();
        if (s_flag) {
          flow_retire(a);
        } else {
          if (threadIdx.x == 0) {
            S->flow_left = R.ntiles;
            __threadfence();
          }
          __syncthreads();
          flow_push(a, rep, kFlowForce, 0u, R.ntiles, &s_t0);
        }
      }
    }
    __syncthreads();
  }
  // the last block out: the unspent budget and the graph's loop decision
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&c->exited, 1u) == gridDim.x - 1) {
      const int budget = __ldcg(&c->budget) - __ldcg(&c->ran);
      const int nrep = __ldcg(&c->lay_nrep);
      int more = 0, ovf = 0;
      for (int r = 0; r < nrep; ++r) {
        const RepState* S = a.st + r;
        if (!a.rep[r].active || __ldcg(&S->steps_left) <= 0) continue;
        if (__ldcg(&S->overflow)) ovf = 1;
        else more = 1;
      }
      c->budget = budget;
      set_loop(h_loop, (more && !ovf && budget > 0 && __ldcg(&c->err) == 0) ? 1u : 0u);
    }
  }
}

}  // namespace b2md
