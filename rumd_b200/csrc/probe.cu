// Arithmetic probes for the parity tests.  This translation unit is compiled
// with nvcc's default floating-point flags (multiply-add contraction on, IEEE
// division/sqrt), the same as the reference's device build, and evaluates
// the reference's expressions as written next to the engine's explicit forms.
#include "../../include/rumd_b200.h"
#include "pbc_math.cuh"


namespace {

__global__ void k_probe_dist2(const float4* a, const float4* b, float3 L, float3 iL, int n, float* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = a[i], q = b[i];
  // minimum image and squared distance as the reference source writes them
  // (SimulationBox.h:111-125)
  float x = p.x - q.x, y = p.y - q.y, z = p.z - q.z;
  x -= L.x * rintf(x * iL.x);
  y -= L.y * rintf(y * iL.y);
  z -= L.z * rintf(z * iL.z);
  out[2 * i] = x * x + y * y + z * z;
  out[2 * i + 1] = b2md::dist2_ref(b2md::mi_comp(p.x - q.x, L.x, iL.x), b2md::mi_comp(p.y - q.y, L.y, iL.y),
                                   b2md::mi_comp(p.z - q.z, L.z, iL.z));
}

__global__ void k_probe_cell(const float* x, int n, float iL, int nc, int* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // calculateCellCoordinates as written (NeighborList.cu:1106-1133), without the clamp
  float s = x[i] * iL + 0.5f;
  out[2 * i] = (int)(nc * s);
  float se = __fmaf_rn(x[i], iL, 0.5f);
  out[2 * i + 1] = __float2int_rz(__fmul_rn((float)nc, se));
}

}  // namespace

extern "C" int b2md_probe_dist2(const float* a4, const float* b4, const float* box, int npairs, float* out) {
  if (!a4 || !b4 || !box || !out || npairs <= 0) return B2MD_ERR_ARG;
  float4 *da = nullptr, *db = nullptr;
  float* dout = nullptr;
  size_t nb = (size_t)npairs * sizeof(float4);
  int rc = B2MD_OK;
  if (cudaMalloc(&da, nb) != cudaSuccess || cudaMalloc(&db, nb) != cudaSuccess ||
      cudaMalloc(&dout, 2 * (size_t)npairs * sizeof(float)) != cudaSuccess) {
    rc = B2MD_ERR_NOMEM;
  } else {
    cudaMemcpy(da, a4, nb, cudaMemcpyHostToDevice);
    cudaMemcpy(db, b4, nb, cudaMemcpyHostToDevice);
    float3 L = make_float3(box[0], box[1], box[2]);
    float3 iL = make_float3(1.f / box[0], 1.f / box[1], 1.f / box[2]);
    k_probe_dist2<<<(npairs + 255) / 256, 256>>>(da, db, L, iL, npairs, dout);
    if (cudaMemcpy(out, dout, 2 * (size_t)npairs * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = B2MD_ERR_CUDA;
  }
  cudaFree(da);
  cudaFree(db);
  cudaFree(dout);
  return rc;
}

extern "C" int b2md_probe_cell(const float* x, int n, float box, int nc, int* out) {
  if (!x || !out || n <= 0 || nc <= 0 || !(box > 0.f)) return B2MD_ERR_ARG;
  float* dx = nullptr;
  int* dout = nullptr;
  int rc = B2MD_OK;
  if (cudaMalloc(&dx, (size_t)n * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&dout, 2 * (size_t)n * sizeof(int)) != cudaSuccess) {
    rc = B2MD_ERR_NOMEM;
  } else {
    cudaMemcpy(dx, x, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    k_probe_cell<<<(n + 255) / 256, 256>>>(dx, n, 1.f / box, nc, dout);
    if (cudaMemcpy(out, dout, 2 * (size_t)n * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) rc = B2MD_ERR_CUDA;
  }
  cudaFree(dx);
  cudaFree(dout);
  return rc;
}
