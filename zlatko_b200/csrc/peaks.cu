// Measured throughput of the special-function unit (MUFU ex2), the ceiling that binds the fused
// exposure kernel (one exponential per merged bond term and path).  Each thread runs 8 independent
// chains of ex2.approx so the unit, not latency, limits the rate.
#include <cuda_runtime.h>

#include "../../include/zlatko_b200.h"

namespace {

__global__ void ex2Chains(float* out, int iters, float seed) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed * (1.0f + 0.01f * k) + 1e-3f * threadIdx.x;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      float r;
      asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a[k]));
      a[k] = r - 1.0f;  // stays in (-1, 1): no overflow
    }
  }
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" zk_status zk_peak_ex2(int device, double* giga_per_s) {
  if (!giga_per_s) return ZK_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return ZK_ERR_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int block = 256, grid = sms * 8, iters = 4096;
  float* out = nullptr;
  if (cudaMalloc(&out, static_cast<size_t>(grid) * block * sizeof(float)) != cudaSuccess) return ZK_ERR_OUT_OF_MEMORY;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ex2Chains<<<grid, block>>>(out, iters, 0.5f);  // warm-up
  cudaEventRecord(e0);
  for (int r = 0; r < 5; ++r) ex2Chains<<<grid, block>>>(out, iters, 0.25f + 0.01f * r);
  cudaEventRecord(e1);
  const cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return ZK_ERR_CUDA;
  *giga_per_s = 5.0 * grid * block * static_cast<double>(iters) * 8.0 / (ms * 1e-3) / 1e9;
  return ZK_OK;
}
