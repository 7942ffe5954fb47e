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

// integrateNVTAlgorithm's update and wrap as the reference source writes them
// (IntegratorNVT.cu:385-399, SimulationBox.h:140-155), next to the engine's
// explicit forms.  out: 9 floats per particle each (v, r, image).
__global__ void k_probe_nvt(const float4* r, const float4* v, const float4* f, const float* xi, float dt, float3 L,
                            float3 iL, int n, float* ref, float* eng) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = r[i], u = v[i], g = f[i];
  {
    float4 my_position = p, my_velocity = u;
    const float4 my_force = g;
    float localThermostatState = xi[i];
    float timeStep = dt;
    float factor = 0.5f * localThermostatState * timeStep;
    float plus = 1.f / (1.f + factor);
    float minus = 1.f - factor;
    my_velocity.x = plus * (minus * my_velocity.x + my_velocity.w * my_force.x * timeStep);
    my_velocity.y = plus * (minus * my_velocity.y + my_velocity.w * my_force.y * timeStep);
    my_velocity.z = plus * (minus * my_velocity.z + my_velocity.w * my_force.z * timeStep);
    my_position.x += my_velocity.x * timeStep;
    my_position.y += my_velocity.y * timeStep;
    my_position.z += my_velocity.z * timeStep;
    float4 image = {rintf(my_position.x * iL.x), rintf(my_position.y * iL.y), rintf(my_position.z * iL.z), 0.f};
    my_position.x -= L.x * image.x;
    my_position.y -= L.y * image.y;
    my_position.z -= L.z * image.z;
    float* o = ref + 9 * (size_t)i;
    o[0] = my_velocity.x; o[1] = my_velocity.y; o[2] = my_velocity.z;
    o[3] = my_position.x; o[4] = my_position.y; o[5] = my_position.z;
    o[6] = image.x; o[7] = image.y; o[8] = image.z;
  }
  {
    const b2md::NvtCoef c = b2md::nvt_coef(xi[i], dt);
    const float vx = b2md::nvt_velocity(c, u.x, u.w, g.x, dt), vy = b2md::nvt_velocity(c, u.y, u.w, g.y, dt),
                vz = b2md::nvt_velocity(c, u.z, u.w, g.z, dt);
    float x = b2md::nvt_position(p.x, vx, dt), y = b2md::nvt_position(p.y, vy, dt), z = b2md::nvt_position(p.z, vz, dt);
    const float kx = b2md::wrap_image(x, iL.x), ky = b2md::wrap_image(y, iL.y), kz = b2md::wrap_image(z, iL.z);
    x = b2md::wrap_apply(x, L.x, kx);
    y = b2md::wrap_apply(y, L.y, ky);
    z = b2md::wrap_apply(z, L.z, kz);
    float* o = eng + 9 * (size_t)i;
    o[0] = vx; o[1] = vy; o[2] = vz;
    o[3] = x; o[4] = y; o[5] = z;
    o[6] = kx; o[7] = ky; o[8] = kz;
  }
}

}  // namespace

extern "C" int b2md_probe_nvt(const float* r4, const float* v4, const float* f4, const float* xi, float dt,
                              const float* box, int n, float* ref9, float* eng9) {
  if (!r4 || !v4 || !f4 || !xi || !box || !ref9 || !eng9 || n <= 0) return B2MD_ERR_ARG;
  float4 *dr = nullptr, *dv = nullptr, *df = nullptr;
  float *dxi = nullptr, *dref = nullptr, *deng = nullptr;
  const size_t nb = (size_t)n * sizeof(float4), no = (size_t)n * 9 * sizeof(float);
  int rc = B2MD_OK;
  if (cudaMalloc(&dr, nb) != cudaSuccess || cudaMalloc(&dv, nb) != cudaSuccess || cudaMalloc(&df, nb) != cudaSuccess ||
      cudaMalloc(&dxi, (size_t)n * sizeof(float)) != cudaSuccess || cudaMalloc(&dref, no) != cudaSuccess ||
      cudaMalloc(&deng, no) != cudaSuccess) {
    rc = B2MD_ERR_NOMEM;
  } else {
    cudaMemcpy(dr, r4, nb, cudaMemcpyHostToDevice);
    cudaMemcpy(dv, v4, nb, cudaMemcpyHostToDevice);
    cudaMemcpy(df, f4, nb, cudaMemcpyHostToDevice);
    cudaMemcpy(dxi, xi, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    const float3 L = make_float3(box[0], box[1], box[2]);
    const float3 iL = make_float3(1.f / box[0], 1.f / box[1], 1.f / box[2]);
    k_probe_nvt<<<(n + 255) / 256, 256>>>(dr, dv, df, dxi, dt, L, iL, n, dref, deng);
    if (cudaMemcpy(ref9, dref, no, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(eng9, deng, no, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = B2MD_ERR_CUDA;
  }
  cudaFree(dr);
  cudaFree(dv);
  cudaFree(df);
  cudaFree(dxi);
  cudaFree(dref);
  cudaFree(deng);
  return rc;
}

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
