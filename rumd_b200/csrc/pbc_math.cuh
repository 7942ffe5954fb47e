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

__device__ __forceinline__ int cell_coord(float x, float invL, int nc) {
  // calculateCellCoordinates (NeighborList.cu:1106-1133)
  float scaled = __fmaf_rn(x, invL, 0.5f);
  int c = __float2int_rz(__fmul_rn((float)nc, scaled));
  if (c == nc) c -= 1;
  else if (c < 0) c = 0;
  return c;
}

}  // namespace b2md
