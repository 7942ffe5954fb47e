// Box and cell arithmetic shared by the kernels and the parity probes.
//
// These are the reference's FP32 expressions (SimulationBox.h:111-125,
// NeighborList.cu:1106-1140) with the multiply-add contractions that nvcc
// applies to them written out explicitly, so that every neighbour-list and
// sort decision rounds exactly as the reference's device build does.
#pragma once
#include <cuda_runtime.h>

namespace b2md {

// Round to nearest, ties to even, for |x| < 2^22: adding and subtracting
// 1.5 * 2^23 rounds x to an integer in the IEEE addition itself (the sum's
// unit in the last place is 1), so the result equals rintf(x) bit for bit.
// Two adds on the FMA pipe instead of a round instruction on the slower
// conversion pipe.  __fadd_rn keeps the compiler from contracting or folding.
__device__ __forceinline__ float rint_small(float x) {
  const float M = 12582912.0f;  // 1.5 * 2^23
  return __fsub_rn(__fadd_rn(x, M), M);
}

__device__ __forceinline__ float mi_comp(float d, float L, float invL) {
  // dr -= L * rintf(dr * invL)   (SimulationBox.h:117-122); |dr * invL| < 1
  return __fmaf_rn(-L, rint_small(__fmul_rn(d, invL)), d);
}

__device__ __forceinline__ float dist2_ref(float dx, float dy, float dz) {
  // dx*dx + dy*dy + dz*dz as contracted by nvcc (SimulationBox.h:124)
  return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// Hardware approximate 1/sqrt(x) (one MUFU operation, denormals flushed);
// callers refine it with a Newton-Raphson step.  Arguments here are squared
// distances, far from the denormal range.
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Nose-Hoover leap-frog of one particle (integrateNVTAlgorithm,
// IntegratorNVT.cu:385-399, with applyBoundaryCondition, SimulationBox.h:140-155):
//   factor = xi dt / 2, plus = 1 / (1 + factor), minus = 1 - factor
//   v <- plus (minus v + (1/m) f dt);  r <- r + v dt;  k = rint(r / L);  r <- r - L k
// with the multiply-add contractions nvcc makes of those expressions written
// out, so that the result is the reference's bit for bit (checked by the
// parity probe against the expressions compiled as written).
struct NvtCoef {
  float plus, minus;
};
// factor = (0.5 xi) dt is never rounded on its own: nvcc fuses it into the
// two sums that use it, 1 + factor and 1 - factor.
__device__ __forceinline__ NvtCoef nvt_coef(float xi, float dt) {
  const float h = __fmul_rn(0.5f, xi);
  NvtCoef c;
  c.plus = __fdiv_rn(1.f, __fmaf_rn(h, dt, 1.f));
  c.minus = __fmaf_rn(-h, dt, 1.f);
  return c;
}
// One component: new velocity, position before the wrap, then the wrap.
// In minus * v + (1/m) f dt nvcc fuses the second product, ((1/m) f) dt,
// into the sum, not the first (2^20 random states: 0 mismatches this way,
// about 30 % the other way).
__device__ __forceinline__ float nvt_velocity(const NvtCoef& c, float v, float im, float f, float dt) {
  return __fmul_rn(c.plus, __fmaf_rn(__fmul_rn(im, f), dt, __fmul_rn(c.minus, v)));
}
__device__ __forceinline__ float nvt_position(float r, float vn, float dt) { return __fmaf_rn(vn, dt, r); }
__device__ __forceinline__ float wrap_image(float x, float invL) { return rintf(__fmul_rn(x, invL)); }
__device__ __forceinline__ float wrap_apply(float x, float L, float k) { return __fmaf_rn(-L, k, x); }

__device__ __forceinline__ int cell_coord(float x, float invL, int nc) {
  // calculateCellCoordinates (NeighborList.cu:1106-1133)
  float scaled = __fmaf_rn(x, invL, 0.5f);
  int c = __float2int_rz(__fmul_rn((float)nc, scaled));
  if (c == nc) c -= 1;
  else if (c < 0) c = 0;
  return c;
}

}  // namespace b2md
