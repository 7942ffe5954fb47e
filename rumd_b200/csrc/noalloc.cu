// LJ forces, potential energy and virial of one configuration without any
// device allocation.
//
// Some callers cannot allocate device memory when they call this library:
// a host application that owns every device buffer and hands a plugin only
// pointers to its own buffers, or a real-time loop that must not call
// cudaMalloc/cudaFree because those may synchronise the device and take
// unbounded time.  b2md_forces_noalloc serves them: the caller passes device
// pointers to its own inputs and outputs, and the only scratch memory (the
// per-block FP64 partial sums of the energy and virial and a completion
// counter) is a fixed, statically allocated array in this library's device
// image, sized for at most kNoAllocMaxParticles particles.
//
// The array exists once per GPU that loads the library and lives until the
// process exits.  Every call shares it, so calls whose kernels overlap on the
// GPU (different streams, no ordering between them) race on it; order them on
// one stream or with events.  The completion counter is cleared at the start
// of every call; the partial sums are overwritten before they are read.
//
// Host code cannot use the array's name as a device address (it names a
// host-side stand-in).  The first call on a device, with that device current,
// looks the address up with cudaGetSymbolAddress and keeps it together with
// the device's current CUDA context; a later call in another context (after
// cudaDeviceReset, say, which unloads the module and so moves the array)
// looks it up again.  Make the first call on a device before any stream
// capture, since the lookup is not a stream operation.
//
// The pair sum uses the minimum-image convention, which counts each pair once;
// that equals the periodic sum only while every cut-off is at most half of
// every box length, so larger cut-offs are rejected.
//
// Its results match b2md_calc_f for the same configuration: the same pair
// function (shifted-force / shifted-potential / plain LJ), all pairs within
// the cut-off under the minimum-image convention, per-particle energies halved.
#include <cstdio>
#include <mutex>

#include "../../include/rumd_b200.h"
#include "pbc_math.cuh"

namespace {

constexpr int kNoAllocMaxParticles = 65536;
constexpr int kNoAllocBlock = 128;
constexpr int kNoAllocMaxBlocks = kNoAllocMaxParticles / kNoAllocBlock;
constexpr int kNoAllocMaxTypes = 8;
constexpr int kRow = 8;  // rc^2, A12, A6, c_s, c_u0, c_ur, unused x2

struct NoAllocScratch {
  double part[kNoAllocMaxBlocks][2];  // per-block sums of u_i and w_i
  unsigned counter;                    // blocks finished in this call
};

// The scratch: a fixed array in the library's device image (no allocation).
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

struct PairTable {
  float p[kNoAllocMaxTypes * kNoAllocMaxTypes * kRow];
};

// Device address of g_noalloc_scratch per device, looked up once per device
// and context (the context the address was found in is kept beside it).
std::mutex g_mu;
NoAllocScratch* g_scratch_ptr[64] = {};
void* g_scratch_ctx[64] = {};

__global__ void __launch_bounds__(kNoAllocBlock)
    k_forces_noalloc(const float4* __restrict__ pos, int n, float3 L, float3 iL, int ntypes, PairTable tab,
                     float4* __restrict__ force, double* __restrict__ sums, NoAllocScratch* scr) {
  __shared__ float4 s_r[kNoAllocBlock];
  __shared__ float s_tab[kNoAllocMaxTypes * kNoAllocMaxTypes * kRow];
  __shared__ double s_red[kNoAllocBlock / 32][2];
  __shared__ int s_last;
  for (int k = threadIdx.x; k < ntypes * ntypes * kRow; k += blockDim.x) s_tab[k] = tab.p[k];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const float4 ri = valid ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  const int ti = __float_as_int(ri.w);
  const bool type_ok = ti >= 0 && ti < ntypes;
  float fx = 0.f, fy = 0.f, fz = 0.f, uu = 0.f, ww = 0.f;
  // all pairs, j staged through shared memory one block-width at a time
  for (int base = 0; base < n; base += blockDim.x) {
    __syncthreads();
    if (base + threadIdx.x < n) s_r[threadIdx.x] = pos[base + threadIdx.x];
    __syncthreads();
    const int m = min((int)blockDim.x, n - base);
    if (!valid || !type_ok) continue;
    const float* row = s_tab + ti * ntypes * kRow;
    for (int k = 0; k < m; ++k) {
      const float4 rj = s_r[k];
      const int tj = __float_as_int(rj.w);
      if (base + k == i || tj < 0 || tj >= ntypes) continue;
      const float dx = b2md::mi_comp(ri.x - rj.x, L.x, iL.x);
      const float dy = b2md::mi_comp(ri.y - rj.y, L.y, iL.y);
      const float dz = b2md::mi_comp(ri.z - rj.z, L.z, iL.z);
      const float d2 = b2md::dist2_ref(dx, dy, dz);
      const float* q = row + tj * kRow;
      if (d2 < q[0]) {
        // 1/r by rsqrt plus one Newton-Raphson step; the cut-off method is
        // folded into c_s, c_u0, c_ur as in the engine's pair rows
        float y = b2md::rsqrt_approx(d2);
        y = y * __fmaf_rn(-0.5f * d2 * y, y, 1.5f);
        const float i2 = y * y, i6 = i2 * i2 * i2, t = q[1] * i6;
        const float s = __fmaf_rn(-q[3], y, i6 * i2 * __fmaf_rn(12.f, t, 6.f * q[2]));
        uu += __fmaf_rn(i6, t + q[2], __fmaf_rn(q[5], d2 * y, q[4]));
        fx = __fmaf_rn(dx, s, fx);
        fy = __fmaf_rn(dy, s, fy);
        fz = __fmaf_rn(dz, s, fz);
        ww = __fmaf_rn(d2, s, ww);
      }
    }
  }
  if (valid) {
    const float nanf_ = __int_as_float(0x7fc00000);
    force[i] = type_ok ? make_float4(fx, fy, fz, 0.5f * uu) : make_float4(nanf_, nanf_, nanf_, nanf_);
  }
  // FP64 block sums, then the last block adds the blocks in index order
  double u = valid && type_ok ? 0.5 * (double)uu : 0.0, w = valid && type_ok ? (double)ww : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    u += __shfl_xor_sync(0xffffffffu, u, o);
    w += __shfl_xor_sync(0xffffffffu, w, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_red[threadIdx.x >> 5][0] = u;
    s_red[threadIdx.x >> 5][1] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bu = 0.0, bw = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      bu += s_red[k][0];
      bw += s_red[k][1];
    }
    scr->part[blockIdx.x][0] = bu;
    scr->part[blockIdx.x][1] = bw;
    __threadfence();
    s_last = atomicAdd(&scr->counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    double su = 0.0, sw = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) {
      su += __ldcg(&scr->part[b][0]);
      sw += __ldcg(&scr->part[b][1]);
    }
    sums[0] = su;        // potential energy, sum of u_i
    sums[1] = sw / 6.0;  // virial W = sum w_i / 6
    scr->counter = 0u;
  }
}

// The current CUDA context (driver call cuCtxGetCurrent, fetched through the
// runtime so that the library needs no link to the driver library); null
// when it cannot be read.
void* current_context() {
  typedef int (*CtxGetCurrent)(void**);
  static CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Looks up (once per device and context, with that device current) the
// device address of the scratch array; host code may not use the symbol
// itself as a pointer.
NoAllocScratch* scratch_for_current_device(int* err) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    *err = B2MD_ERR_CUDA;
    return nullptr;
  }
  void* ctx = current_context();
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev] || !ctx || ctx != g_scratch_ctx[dev]) {
    // the lookup also makes the device's primary context current on this
    // thread when none was, so the context is read again after it
    NoAllocScratch* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_noalloc_scratch) != cudaSuccess || !p) {
      *err = B2MD_ERR_CUDA;
      return nullptr;
    }
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = current_context();
  }
  return g_scratch_ptr[dev];
}

}  // namespace

namespace b2md_internal {
void set_last_error(const char* msg);
}

namespace {
int noalloc_fail(int code, const char* msg) {
  b2md_internal::set_last_error(msg);
  return code;
}
}  // namespace

extern "C" int b2md_forces_noalloc(const float* pos4, int n, const float* box, int ntypes, const float* params,
                                   int cutoff_method, float* force4, double* sums, void* stream) {
  if (n < 2 || n > kNoAllocMaxParticles)
    return noalloc_fail(B2MD_ERR_ARG, "b2md_forces_noalloc: n must be between 2 and 65536 (the size of its "
                                      "fixed scratch array)");
  if (!pos4 || !box || !params || !force4 || !sums) return noalloc_fail(B2MD_ERR_ARG, "b2md_forces_noalloc: null pointer");
  if (ntypes < 1 || ntypes > kNoAllocMaxTypes) return noalloc_fail(B2MD_ERR_ARG, "b2md_forces_noalloc: ntypes must be 1..8");
  if (cutoff_method < 0 || cutoff_method > 2)
    return noalloc_fail(B2MD_ERR_ARG, "b2md_forces_noalloc: cutoff method must be NS, SP or SF");
  if (!(box[0] > 0.f) || !(box[1] > 0.f) || !(box[2] > 0.f))
    return noalloc_fail(B2MD_ERR_ARG, "b2md_forces_noalloc: box lengths must be positive");
  // minimum image counts one image per pair: exact only for rc <= L/2
  float rcmax = 0.f;
  for (int k = 0; k < ntypes * ntypes; ++k) rcmax = params[k * 12] > rcmax ? params[k * 12] : rcmax;
  const float lmin = fminf(box[0], fminf(box[1], box[2]));
  if (rcmax > 0.5f * lmin) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "b2md_forces_noalloc: cut-off %g exceeds half the smallest box length %g (the minimum-image sum "
             "would miss periodic images)", (double)rcmax, (double)lmin);
    return noalloc_fail(B2MD_ERR_ARG, msg);
  }
  // an error left by an earlier runtime call on this thread is not this
  // call's: clear it so that the launch check below sees only this launch
  (void)cudaGetLastError();
  int err = B2MD_OK;
  NoAllocScratch* scr = scratch_for_current_device(&err);
  if (!scr) return noalloc_fail(err, "b2md_forces_noalloc: cannot find the device address of the scratch array");
  // pack the RUMD table (T*T*12) into the kernel's rows, by value
  PairTable tab = {};
  for (int k = 0; k < ntypes * ntypes; ++k) {
    const float* p = params + k * 12;
    float* q = tab.p + k * kRow;
    const float rc = p[0], sc = p[10], uc = p[11];
    const bool sf = cutoff_method == B2MD_CUTOFF_SF, sp = cutoff_method == B2MD_CUTOFF_SP;
    q[0] = rc * rc;
    q[1] = p[1];
    q[2] = p[2];
    q[3] = sf ? sc : 0.f;
    q[4] = sf ? -(sc * rc + uc) : (sp ? -uc : 0.f);
    q[5] = sf ? sc : 0.f;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the completion counter must start at zero for every call
  const cudaError_t me = cudaMemsetAsync(&scr->counter, 0, sizeof(unsigned), s);
  if (me != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof(msg), "b2md_forces_noalloc: clearing the scratch counter failed: %s",
             cudaGetErrorName(me));
    return noalloc_fail(B2MD_ERR_CUDA, msg);
  }
  const float3 L = make_float3(box[0], box[1], box[2]);
  const float3 iL = make_float3(1.f / box[0], 1.f / box[1], 1.f / box[2]);
  const int blocks = (n + kNoAllocBlock - 1) / kNoAllocBlock;
  k_forces_noalloc<<<blocks, kNoAllocBlock, 0, s>>>(reinterpret_cast<const float4*>(pos4), n, L, iL, ntypes, tab,
                                                     reinterpret_cast<float4*>(force4), sums, scr);
  const cudaError_t le = cudaGetLastError();
  if (le != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof(msg), "b2md_forces_noalloc: launch failed: %s (%s)", cudaGetErrorName(le),
             cudaGetErrorString(le));
    return noalloc_fail(B2MD_ERR_CUDA, msg);
  }
  return B2MD_OK;
}
