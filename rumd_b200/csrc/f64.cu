// Double-precision engine: the per-step path of RUMD (neighbour list, LJ pair
// forces, Nose-Hoover leap-frog, energy/virial/kinetic sums) computed in FP64
// throughout.  It is the analogue of RUMD rebuilt after changeToDouble.sh
// (changeToDouble.sh:1-189, which turns every float of the sources into a
// double) and serves as the accuracy oracle on the GPU for the FP32 engine:
// the same potential and integrator, evaluated without FP32 rounding.
//
// Algorithm, step by step (the order of Simulation.Run, Simulation.py:585-610,
// with IntegratorNVT::Integrate, IntegratorNVT.cu:64-92, 364-437):
//   1. every reset_interval steps: centre-of-mass velocity removed
//      (IntegratorNVT::SetMomentumToZero, IntegratorNVT.cu:176-183);
//   2. if a particle moved more than skin/2 since the last build: cell list
//      and full neighbour list within (rc_ij + skin)^2
//      (NeighborList::UpdateNBlist, NeighborList.cu:583-690);
//   3. pair forces, u_i (halved) and w_i = sum d^2 s (fij, PairPotential.h:1198-1244;
//      Pot_IPL_12_6::ComputeInteraction, PairPotential.h:161-168);
//   4. Nose-Hoover leap-frog with PBC wrap and image count, FP64 kinetic sums
//      (integrateNVTAlgorithm, IntegratorNVT.cu:364-418);
//   5. thermostat update xi += dt * omega^2 * min(KE2/(DOF T) - 1, 10)
//      (updateNVTThermostatState, IntegratorNVT.cu:426-437).
// The pair constants: rc, A12 and A6 come from the RUMD parameter table; the
// shifted-force / shifted-potential constants s(rc) rc and u(rc) are
// recomputed here in FP64 from them, as the double build's CopyParamsToGPU
// (PairPotential.cu:82-125) would.
//
// Layout: particles stay in the caller's order (no spatial sort).  Cells are
// at least rc_max + skin wide (27-cell stencil); boxes with fewer than three
// cells along a side use all pairs.  Within a cell, particles are listed in
// ascending index, so lists and sums are deterministic.  All sums are FP64
// with a fixed tree (block partials added in block order).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/rumd_b200.h"

namespace b2md_internal {
void set_last_error(const char* msg);
}

namespace {

constexpr int kB = 256;        // threads per block
constexpr int kMaxT = 16;      // particle types
constexpr int kNPartF64 = 4;   // per-block partials: pe, w, ke_t, ke2

struct F64Pair {
  double rc, rc2, a12, a6, cs, cu, nb2;  // cs = s(rc) rc, cu = u(rc), nb2 = (rc + skin)^2
};

struct F64Dev {  // device-resident scalars
  double xi, P[3], M, pe, W, ke_t, ke2;
  long long rebuilds, steps;
  int need, overflow;
};

struct F64Args {
  int n, ntypes, cutoff, max_nbrs, ncell, allpairs, thermo;
  int nc[3];
  double L[3], invL[3], dt, skin2_4, T, omega2, dof;
  double4 *r, *v, *f, *last_r;
  int4* im;
  int *cell, *cnt, *cstart, *cfill, *cidx;
  unsigned *nn, *nbl;
  double* part;
  F64Dev* st;
  const F64Pair* par;
};

__device__ __forceinline__ double mi64(double d, double L, double iL) { return d - L * rint(d * iL); }

__device__ __forceinline__ int type_of(const double4& r) { return (int)r.w; }

// Block sum of K doubles per thread (warp butterfly, then warps in order);
// the result is valid in s_out after the call.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* s_warp, double* s_out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) s_warp[wid * K + k] = x;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += s_warp[w * K + threadIdx.x];
    s_out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Sums partial columns [k0, k0+K) over `nblocks` rows of part (row stride
// kNPartF64) in a fixed order: thread t adds rows t, t+kB, ...; then the
// block adds the threads in order.
template <int K>
__device__ __forceinline__ void sum_partials(const F64Args& a, int nblocks, int k0, double* s_out) {
  __shared__ double s_warp[(kB / 32) * K];
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += a.part[(size_t)b * kNPartF64 + k0 + k];
  block_sum<K>(v, s_warp, s_out);
}

// ---- 1. momentum reset ----
__global__ void __launch_bounds__(kB) k64_momentum_part(F64Args a) {
  __shared__ double s_warp[(kB / 32) * 4], s_out[4];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (i < a.n) {
    const double4 vi = a.v[i];
    const double m = 1.0 / vi.w;
    v[0] = m * vi.x; v[1] = m * vi.y; v[2] = m * vi.z; v[3] = m;
  }
  block_sum<4>(v, s_warp, s_out);
  if (threadIdx.x < 4) a.part[(size_t)blockIdx.x * kNPartF64 + threadIdx.x] = s_out[threadIdx.x];
}

__global__ void __launch_bounds__(kB) k64_momentum_total(F64Args a, int nblocks) {
  __shared__ double s_out[4];
  sum_partials<4>(a, nblocks, 0, s_out);
  if (threadIdx.x == 0) {
    a.st->P[0] = s_out[0]; a.st->P[1] = s_out[1]; a.st->P[2] = s_out[2]; a.st->M = s_out[3];
  }
}

__global__ void __launch_bounds__(kB) k64_momentum_apply(F64Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n || !(a.st->M > 0.0)) return;
  const double iM = 1.0 / a.st->M;
  double4 v = a.v[i];
  v.x -= a.st->P[0] * iM; v.y -= a.st->P[1] * iM; v.z -= a.st->P[2] * iM;
  a.v[i] = v;
}

// ---- 2. neighbour list (each kernel returns at once unless a build is due) ----
__device__ __forceinline__ int cell_of(const F64Args& a, const double4& r) {
  int c[3];
  const double x[3] = {r.x, r.y, r.z};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int k = (int)floor((x[d] * a.invL[d] + 0.5) * a.nc[d]);
    c[d] = k < 0 ? 0 : (k >= a.nc[d] ? a.nc[d] - 1 : k);
  }
  return c[0] + a.nc[0] * (c[1] + a.nc[1] * c[2]);
}

__global__ void __launch_bounds__(kB) k64_rb_clear(F64Args a) {
  if (!a.st->need || a.allpairs) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < a.ncell; c += gridDim.x * blockDim.x) a.cnt[c] = 0;
}

__global__ void __launch_bounds__(kB) k64_rb_count(F64Args a) {
  if (!a.st->need || a.allpairs) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int c = cell_of(a, a.r[i]);
  a.cell[i] = c;
  atomicAdd(&a.cnt[c], 1);
}

// exclusive scan of the cell counts by one block: each thread scans a
// contiguous chunk, the chunk totals are scanned in shared memory
__global__ void __launch_bounds__(1024) k64_rb_scan(F64Args a) {
  if (!a.st->need || a.allpairs) return;
  __shared__ int s_tot[1024];
  const int chunk = (a.ncell + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * chunk, e = min(a.ncell, b + chunk);
  int s = 0;
  for (int c = b; c < e; ++c) s += a.cnt[c];
  s_tot[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const int t = threadIdx.x >= (unsigned)o ? s_tot[threadIdx.x - o] : 0;
    __syncthreads();
    s_tot[threadIdx.x] += t;
    __syncthreads();
  }
  int run = s_tot[threadIdx.x] - s;  // exclusive prefix of this chunk
  for (int c = b; c < e; ++c) {
    a.cstart[c] = run;
    a.cfill[c] = run;
    run += a.cnt[c];
  }
}

__global__ void __launch_bounds__(kB) k64_rb_fill(F64Args a) {
  if (!a.st->need || a.allpairs) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  a.cidx[atomicAdd(&a.cfill[a.cell[i]], 1)] = i;
}

// particles of each cell in ascending index (insertion sort; a few per cell)
__global__ void __launch_bounds__(kB) k64_rb_sort(F64Args a) {
  if (!a.st->need || a.allpairs) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < a.ncell; c += gridDim.x * blockDim.x) {
    int* p = a.cidx + a.cstart[c];
    const int m = a.cnt[c];
    for (int k = 1; k < m; ++k) {
      const int x = p[k];
      int q = k - 1;
      while (q >= 0 && p[q] > x) {
        p[q + 1] = p[q];
        --q;
      }
      p[q + 1] = x;
    }
  }
}

__global__ void __launch_bounds__(kB) k64_rb_build(F64Args a) {
  if (!a.st->need) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double4 ri = a.r[i];
  const F64Pair* row = a.par + type_of(ri) * a.ntypes;
  unsigned count = 0;
  auto test = [&](int j) {
    if (j == i) return;
    const double4 rj = a.r[j];
    const double dx = mi64(ri.x - rj.x, a.L[0], a.invL[0]);
    const double dy = mi64(ri.y - rj.y, a.L[1], a.invL[1]);
    const double dz = mi64(ri.z - rj.z, a.L[2], a.invL[2]);
    if (dx * dx + dy * dy + dz * dz < row[type_of(rj)].nb2) {
      if ((int)count < a.max_nbrs) a.nbl[(size_t)count * a.n + i] = (unsigned)j;
      ++count;
    }
  };
  if (a.allpairs) {
    for (int j = 0; j < a.n; ++j) test(j);
  } else {
    const int c = a.cell[i];
    const int cx = c % a.nc[0], cy = (c / a.nc[0]) % a.nc[1], cz = c / (a.nc[0] * a.nc[1]);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int ox = (cx + dx + a.nc[0]) % a.nc[0], oy = (cy + dy + a.nc[1]) % a.nc[1];
          const int oz = (cz + dz + a.nc[2]) % a.nc[2];
          const int o = ox + a.nc[0] * (oy + a.nc[1] * oz);
          const int b = a.cstart[o], e = b + a.cnt[o];
          for (int s = b; s < e; ++s) test(a.cidx[s]);
        }
  }
  a.nn[i] = min(count, (unsigned)a.max_nbrs);
  if ((int)count > a.max_nbrs) a.st->overflow = 1;
  a.last_r[i] = ri;
}

__global__ void k64_rb_done(F64Args a) {
  if (a.st->need) {
    a.st->need = 0;
    a.st->rebuilds += 1;
  }
}

// ---- 3. pair forces ----
__global__ void __launch_bounds__(kB) k64_forces(F64Args a) {
  __shared__ double s_warp[(kB / 32) * 2], s_out[2];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2] = {0.0, 0.0};
  if (i < a.n) {
    const double4 ri = a.r[i];
    const F64Pair* row = a.par + type_of(ri) * a.ntypes;
    double fx = 0.0, fy = 0.0, fz = 0.0, u = 0.0, w = 0.0;
    const unsigned nn = a.nn[i];
    for (unsigned k = 0; k < nn; ++k) {
      const double4 rj = a.r[a.nbl[(size_t)k * a.n + i]];
      const double dx = mi64(ri.x - rj.x, a.L[0], a.invL[0]);
      const double dy = mi64(ri.y - rj.y, a.L[1], a.invL[1]);
      const double dz = mi64(ri.z - rj.z, a.L[2], a.invL[2]);
      const double d2 = dx * dx + dy * dy + dz * dz;
      const F64Pair& p = row[type_of(rj)];
      if (d2 < p.rc2) {
        const double i2 = 1.0 / d2, i6 = i2 * i2 * i2, t = p.a12 * i6;
        double s = i6 * i2 * (12.0 * t + 6.0 * p.a6);
        double uu = i6 * (t + p.a6);
        if (a.cutoff == B2MD_CUTOFF_SF) {
          const double r = sqrt(d2);
          s -= p.cs / r;
          uu += p.cs * (r - p.rc) - p.cu;
        } else if (a.cutoff == B2MD_CUTOFF_SP) {
          uu -= p.cu;
        }
        fx += dx * s; fy += dy * s; fz += dz * s;
        u += uu; w += d2 * s;
      }
    }
    a.f[i] = make_double4(fx, fy, fz, 0.5 * u);
    acc[0] = 0.5 * u;
    acc[1] = w;
  }
  block_sum<2>(acc, s_warp, s_out);
  if (threadIdx.x < 2) a.part[(size_t)blockIdx.x * kNPartF64 + threadIdx.x] = s_out[threadIdx.x];
}

// ---- 4. Nose-Hoover leap-frog ----
__global__ void __launch_bounds__(kB) k64_integrate(F64Args a) {
  __shared__ double s_warp[(kB / 32) * 2], s_out[2];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[2] = {0.0, 0.0};
  if (i < a.n) {
    const double factor = a.thermo ? 0.5 * a.st->xi * a.dt : 0.0;
    const double plus = 1.0 / (1.0 + factor), minus = 1.0 - factor;
    const double4 f = a.f[i];
    double4 v = a.v[i], r = a.r[i];
    int4 im = a.im[i];
    const double vb = v.x * v.x + v.y * v.y + v.z * v.z;
    v.x = plus * (minus * v.x + v.w * f.x * a.dt);
    v.y = plus * (minus * v.y + v.w * f.y * a.dt);
    v.z = plus * (minus * v.z + v.w * f.z * a.dt);
    r.x += v.x * a.dt; r.y += v.y * a.dt; r.z += v.z * a.dt;
    const double kx = rint(r.x * a.invL[0]), ky = rint(r.y * a.invL[1]), kz = rint(r.z * a.invL[2]);
    r.x -= a.L[0] * kx; r.y -= a.L[1] * ky; r.z -= a.L[2] * kz;
    im.x += (int)kx; im.y += (int)ky; im.z += (int)kz;
    a.v[i] = v; a.r[i] = r; a.im[i] = im;
    const double vf = v.x * v.x + v.y * v.y + v.z * v.z;
    const double m = 1.0 / v.w;
    acc[0] = 0.25 * m * (vb + vf);
    acc[1] = m * vf;
    const double4 lr = a.last_r[i];
    const double ex = mi64(r.x - lr.x, a.L[0], a.invL[0]), ey = mi64(r.y - lr.y, a.L[1], a.invL[1]);
    const double ez = mi64(r.z - lr.z, a.L[2], a.invL[2]);
    if (ex * ex + ey * ey + ez * ez > a.skin2_4) a.st->need = 1;
  }
  block_sum<2>(acc, s_warp, s_out);
  if (threadIdx.x < 2) a.part[(size_t)blockIdx.x * kNPartF64 + 2 + threadIdx.x] = s_out[threadIdx.x];
}

// ---- 5. totals, thermostat, energy log ----
__global__ void __launch_bounds__(kB) k64_finish(F64Args a, int nblocks, int integrated, double* elog) {
  __shared__ double s_out[4];
  sum_partials<4>(a, nblocks, 0, s_out);
  if (threadIdx.x != 0) return;
  F64Dev* S = a.st;
  S->pe = s_out[0];
  S->W = s_out[1] / 6.0;
  if (!integrated) return;
  S->ke_t = s_out[2];
  S->ke2 = s_out[3];
  if (a.thermo) {
    double dev = s_out[3] / (a.dof * a.T) - 1.0;
    if (dev > 10.0) dev = 10.0;
    S->xi += a.dt * a.omega2 * dev;
  }
  S->steps += 1;
  if (elog) {
    elog[0] = S->pe;
    elog[1] = S->W;
    elog[2] = S->ke_t;
    elog[3] = S->xi;
  }
}

}  // namespace

struct b2md_f64 {
  int device = 0;
  cudaStream_t stream = nullptr;
  F64Args a = {};
  F64Dev* st = nullptr;
  F64Pair* par = nullptr;
  int reset_interval = 100;
  bool have_state = false;
  std::vector<void*> bufs;
};

namespace {

std::string f64_errmsg;

int f64_fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  f64_errmsg = buf;
  b2md_internal::set_last_error(f64_errmsg.c_str());
  return code;
}

#define F64_CK(x)                                                                       \
  do {                                                                                  \
    cudaError_t err_ = (x);                                                             \
    if (err_ != cudaSuccess)                                                            \
      return f64_fail(B2MD_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(err_));           \
  } while (0)

template <class T>
int f64_alloc(b2md_f64* h, T*& p, size_t count) {
  void* q = nullptr;
  cudaError_t err = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (err != cudaSuccess) return f64_fail(B2MD_ERR_NOMEM, "b2md_f64: cudaMalloc of %zu bytes failed: %s",
                                          count * sizeof(T), cudaGetErrorString(err));
  h->bufs.push_back(q);
  p = static_cast<T*>(q);
  return B2MD_OK;
}

int nblocks(const b2md_f64* h) { return (h->a.n + kB - 1) / kB; }

// step 2 + 3: list (when due) and forces; the launches of one step
int launch_forces(b2md_f64* h) {
  const F64Args& a = h->a;
  const int B = nblocks(h), s_cells = std::max(1, std::min((a.ncell + kB - 1) / kB, 4096));
  cudaStream_t s = h->stream;
  k64_rb_clear<<<s_cells, kB, 0, s>>>(a);
  k64_rb_count<<<B, kB, 0, s>>>(a);
  k64_rb_scan<<<1, 1024, 0, s>>>(a);
  k64_rb_fill<<<B, kB, 0, s>>>(a);
  k64_rb_sort<<<s_cells, kB, 0, s>>>(a);
  k64_rb_build<<<B, kB, 0, s>>>(a);
  k64_rb_done<<<1, 1, 0, s>>>(a);
  k64_forces<<<B, kB, 0, s>>>(a);
  F64_CK(cudaGetLastError());
  return B2MD_OK;
}

int read_dev(b2md_f64* h, F64Dev* out) {
  F64_CK(cudaMemcpyAsync(out, h->st, sizeof(F64Dev), cudaMemcpyDeviceToHost, h->stream));
  F64_CK(cudaStreamSynchronize(h->stream));
  return B2MD_OK;
}

int check_overflow(b2md_f64* h) {
  F64Dev d;
  int rc = read_dev(h, &d);
  if (rc) return rc;
  if (d.overflow)
    return f64_fail(B2MD_ERR_OVERFLOW, "b2md_f64: a particle has more than %d neighbours within rc + skin; "
                                       "the run is invalid (create the engine with a larger max_nbrs)",
                    h->a.max_nbrs);
  return B2MD_OK;
}

}  // namespace

extern "C" {

int b2md_f64_create(int device, int n, int ntypes, const double* box3, const float* params, int cutoff_method,
                    double skin, int max_nbrs, b2md_f64** out) {
  if (!out || !box3 || !params) return f64_fail(B2MD_ERR_ARG, "b2md_f64_create: null argument");
  *out = nullptr;
  if (n < 2) return f64_fail(B2MD_ERR_ARG, "b2md_f64_create: n must be >= 2");
  if (ntypes < 1 || ntypes > kMaxT) return f64_fail(B2MD_ERR_ARG, "b2md_f64_create: ntypes must be 1..%d", kMaxT);
  if (cutoff_method < 0 || cutoff_method > 2)
    return f64_fail(B2MD_ERR_ARG, "b2md_f64_create: cut-off method must be NS, SP or SF");
  if (!(skin >= 0.0)) return f64_fail(B2MD_ERR_ARG, "b2md_f64_create: skin must be >= 0");
  for (int d = 0; d < 3; ++d)
    if (!(box3[d] > 0.0)) return f64_fail(B2MD_ERR_ARG, "b2md_f64_create: box lengths must be positive");
  // pair constants in FP64 from rc = p0, A12 = p1, A6 = p2 of the RUMD table
  std::vector<F64Pair> pars((size_t)ntypes * ntypes);
  double rc_max = 0.0;
  for (int k = 0; k < ntypes * ntypes; ++k) {
    const float* p = params + (size_t)k * 12;
    F64Pair& q = pars[k];
    q.rc = p[0]; q.a12 = p[1]; q.a6 = p[2];
    if (!(q.rc > 0.0)) return f64_fail(B2MD_ERR_ARG, "b2md_f64_create: pair %d has no positive cut-off", k);
    q.rc2 = q.rc * q.rc;
    const double i2 = 1.0 / q.rc2, i6 = i2 * i2 * i2;
    q.cu = i6 * (q.a12 * i6 + q.a6);
    q.cs = i6 * i2 * (12.0 * q.a12 * i6 + 6.0 * q.a6) * q.rc;
    q.nb2 = (q.rc + skin) * (q.rc + skin);
    rc_max = std::max(rc_max, q.rc);
  }
  b2md_f64* h = new b2md_f64();
  h->device = device;
  F64Args& a = h->a;
  a.n = n; a.ntypes = ntypes; a.cutoff = cutoff_method;
  a.allpairs = 0;
  a.ncell = 1;
  for (int d = 0; d < 3; ++d) {
    a.L[d] = box3[d];
    a.invL[d] = 1.0 / box3[d];
    a.nc[d] = (int)std::floor(box3[d] / (rc_max + skin));
    if (a.nc[d] < 3) a.allpairs = 1;
    a.ncell *= std::max(a.nc[d], 1);
  }
  const double vol = box3[0] * box3[1] * box3[2];
  const double est = n / vol * 4.0 / 3.0 * M_PI * std::pow(rc_max + skin, 3.0);
  a.max_nbrs = max_nbrs > 0 ? max_nbrs : (int)std::min<double>(n - 1, 1.6 * est + 32.0);
  a.skin2_4 = 0.25 * skin * skin;
  a.dt = 0.005; a.T = 1.0; a.omega2 = 4.0 * M_PI * M_PI / (0.2 * 0.2); a.thermo = 1;
  a.dof = 3.0 * n - 3.0;
  int rc = B2MD_OK;
  auto done = [&](int code) {
    if (code) { b2md_f64_destroy(h); return code; }
    *out = h;
    return B2MD_OK;
  };
  if (cudaSetDevice(device) != cudaSuccess) return done(f64_fail(B2MD_ERR_CUDA, "b2md_f64_create: bad device %d", device));
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    return done(f64_fail(B2MD_ERR_CUDA, "b2md_f64_create: stream creation failed"));
  const size_t nb = (size_t)((n + kB - 1) / kB);
  if ((rc = f64_alloc(h, a.r, n)) || (rc = f64_alloc(h, a.v, n)) || (rc = f64_alloc(h, a.f, n)) ||
      (rc = f64_alloc(h, a.last_r, n)) || (rc = f64_alloc(h, a.im, n)) || (rc = f64_alloc(h, a.cell, n)) ||
      (rc = f64_alloc(h, a.cnt, a.ncell)) || (rc = f64_alloc(h, a.cstart, a.ncell)) ||
      (rc = f64_alloc(h, a.cfill, a.ncell)) || (rc = f64_alloc(h, a.cidx, n)) || (rc = f64_alloc(h, a.nn, n)) ||
      (rc = f64_alloc(h, a.nbl, (size_t)a.max_nbrs * n)) || (rc = f64_alloc(h, a.part, nb * kNPartF64)) ||
      (rc = f64_alloc(h, h->st, 1)) || (rc = f64_alloc(h, h->par, pars.size())))
    return done(rc);
  a.st = h->st;
  a.par = h->par;
  if (cudaMemcpy(h->par, pars.data(), pars.size() * sizeof(F64Pair), cudaMemcpyHostToDevice) != cudaSuccess)
    return done(f64_fail(B2MD_ERR_CUDA, "b2md_f64_create: parameter upload failed"));
  F64Dev d0 = {};
  d0.need = 1;
  if (cudaMemcpy(h->st, &d0, sizeof d0, cudaMemcpyHostToDevice) != cudaSuccess)
    return done(f64_fail(B2MD_ERR_CUDA, "b2md_f64_create: state upload failed"));
  return done(B2MD_OK);
}

int b2md_f64_destroy(b2md_f64* h) {
  if (!h) return B2MD_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (void* p : h->bufs) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return B2MD_OK;
}

int b2md_f64_set_state(b2md_f64* h, const double* pos4, const double* vel4, const int* im3) {
  if (!h || !pos4 || !vel4) return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_state: null argument");
  const int n = h->a.n;
  std::vector<double4> r(n), v(n);
  std::vector<int4> im(n);
  for (int i = 0; i < n; ++i) {
    const double t = pos4[4 * i + 3];
    if (!(t >= 0.0 && t < h->a.ntypes && t == std::floor(t)))
      return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_state: particle %d has type %g (want 0..%d)", i, t,
                      h->a.ntypes - 1);
    if (!(vel4[4 * i + 3] > 0.0)) return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_state: particle %d: 1/m must be > 0", i);
    r[i] = make_double4(pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2], t);
    v[i] = make_double4(vel4[4 * i], vel4[4 * i + 1], vel4[4 * i + 2], vel4[4 * i + 3]);
    im[i] = im3 ? make_int4(im3[3 * i], im3[3 * i + 1], im3[3 * i + 2], 0) : make_int4(0, 0, 0, 0);
  }
  F64_CK(cudaSetDevice(h->device));
  F64_CK(cudaMemcpyAsync(h->a.r, r.data(), n * sizeof(double4), cudaMemcpyHostToDevice, h->stream));
  F64_CK(cudaMemcpyAsync(h->a.v, v.data(), n * sizeof(double4), cudaMemcpyHostToDevice, h->stream));
  F64_CK(cudaMemcpyAsync(h->a.im, im.data(), n * sizeof(int4), cudaMemcpyHostToDevice, h->stream));
  const int one = 1;
  F64_CK(cudaMemcpyAsync(&h->st->need, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  F64_CK(cudaStreamSynchronize(h->stream));
  h->have_state = true;
  return B2MD_OK;
}

int b2md_f64_set_integrator(b2md_f64* h, double dt, double target_T, double tau, int thermostat_on,
                            int reset_interval) {
  if (!h) return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_integrator: null engine");
  if (!(dt > 0.0)) return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_integrator: dt must be > 0");
  if (thermostat_on && !(target_T > 0.0 && tau > 0.0))
    return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_integrator: thermostat needs T > 0 and tau > 0");
  if (reset_interval < 0) return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_integrator: reset_interval must be >= 0");
  h->a.dt = dt;
  h->a.T = target_T;
  h->a.thermo = thermostat_on ? 1 : 0;
  h->a.omega2 = thermostat_on ? 4.0 * M_PI * M_PI / (tau * tau) : 0.0;
  h->reset_interval = reset_interval;
  return B2MD_OK;
}

int b2md_f64_set_xi(b2md_f64* h, double xi) {
  if (!h) return f64_fail(B2MD_ERR_ARG, "b2md_f64_set_xi: null engine");
  F64_CK(cudaSetDevice(h->device));
  F64_CK(cudaMemcpyAsync(&h->st->xi, &xi, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  F64_CK(cudaStreamSynchronize(h->stream));
  return B2MD_OK;
}

int b2md_f64_calc_f(b2md_f64* h) {
  if (!h) return f64_fail(B2MD_ERR_ARG, "b2md_f64_calc_f: null engine");
  if (!h->have_state) return f64_fail(B2MD_ERR_STATE, "b2md_f64_calc_f: no state set");
  F64_CK(cudaSetDevice(h->device));
  int rc = launch_forces(h);
  if (rc) return rc;
  k64_finish<<<1, kB, 0, h->stream>>>(h->a, nblocks(h), 0, nullptr);
  F64_CK(cudaGetLastError());
  return check_overflow(h);
}

int b2md_f64_run(b2md_f64* h, long long nsteps, double* energies) {
  if (!h) return f64_fail(B2MD_ERR_ARG, "b2md_f64_run: null engine");
  if (nsteps < 0) return f64_fail(B2MD_ERR_ARG, "b2md_f64_run: nsteps must be >= 0");
  if (!h->have_state) return f64_fail(B2MD_ERR_STATE, "b2md_f64_run: no state set");
  F64_CK(cudaSetDevice(h->device));
  double* d_log = nullptr;
  if (energies && nsteps > 0) F64_CK(cudaMalloc(&d_log, (size_t)nsteps * 4 * sizeof(double)));
  const int B = nblocks(h);
  int rc = B2MD_OK;
  for (long long k = 0; k < nsteps && rc == B2MD_OK; ++k) {
    if (h->reset_interval > 0 && k % h->reset_interval == 0) {
      k64_momentum_part<<<B, kB, 0, h->stream>>>(h->a);
      k64_momentum_total<<<1, kB, 0, h->stream>>>(h->a, B);
      k64_momentum_apply<<<B, kB, 0, h->stream>>>(h->a);
    }
    rc = launch_forces(h);
    if (rc) break;
    k64_integrate<<<B, kB, 0, h->stream>>>(h->a);
    k64_finish<<<1, kB, 0, h->stream>>>(h->a, B, 1, d_log ? d_log + 4 * k : nullptr);
    if (cudaGetLastError() != cudaSuccess) rc = f64_fail(B2MD_ERR_CUDA, "b2md_f64_run: launch failed");
    if (rc == B2MD_OK && (k + 1) % 256 == 0) rc = check_overflow(h);
  }
  if (rc == B2MD_OK) rc = check_overflow(h);
  if (rc == B2MD_OK && d_log) {
    if (cudaMemcpy(energies, d_log, (size_t)nsteps * 4 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = f64_fail(B2MD_ERR_CUDA, "b2md_f64_run: energy copy failed");
  }
  if (d_log) cudaFree(d_log);
  return rc;
}

int b2md_f64_get(b2md_f64* h, int field, void* out) {
  if (!h || !out) return f64_fail(B2MD_ERR_ARG, "b2md_f64_get: null argument");
  const int n = h->a.n;
  F64_CK(cudaSetDevice(h->device));
  F64_CK(cudaStreamSynchronize(h->stream));
  if (field == B2MD_F64_POS || field == B2MD_F64_VEL || field == B2MD_F64_FORCE) {
    const double4* src = field == B2MD_F64_POS ? h->a.r : (field == B2MD_F64_VEL ? h->a.v : h->a.f);
    F64_CK(cudaMemcpy(out, src, n * sizeof(double4), cudaMemcpyDeviceToHost));
    return B2MD_OK;
  }
  if (field == B2MD_F64_IMAGES) {
    std::vector<int4> im(n);
    F64_CK(cudaMemcpy(im.data(), h->a.im, n * sizeof(int4), cudaMemcpyDeviceToHost));
    int* o = static_cast<int*>(out);
    for (int i = 0; i < n; ++i) { o[3 * i] = im[i].x; o[3 * i + 1] = im[i].y; o[3 * i + 2] = im[i].z; }
    return B2MD_OK;
  }
  return f64_fail(B2MD_ERR_ARG, "b2md_f64_get: unknown field %d", field);
}

int b2md_f64_stats(b2md_f64* h, double* out) {
  if (!h || !out) return f64_fail(B2MD_ERR_ARG, "b2md_f64_stats: null argument");
  F64_CK(cudaSetDevice(h->device));
  F64Dev d;
  int rc = read_dev(h, &d);
  if (rc) return rc;
  out[0] = d.pe; out[1] = d.W; out[2] = d.ke_t; out[3] = d.ke2; out[4] = d.xi;
  out[5] = (double)d.rebuilds; out[6] = (double)d.steps;
  return B2MD_OK;
}

}  // extern "C"
