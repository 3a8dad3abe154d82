// probe.cu — FP32 FMA throughput probe: the roofline denominator for the
// FP32-pipe-bound correlation kernels, measured on the device in use.
#include <cuda_runtime.h>

#include "fxc.h"

namespace {

__global__ void fma_probe_kernel(float* out, int iters, float a, float b) {
  // 16 independent FMA chains per thread keep every FP32 lane busy.
  float r[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) r[i] = (float)(threadIdx.x + i) * 1e-3f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 16; ++i) r[i] = fmaf(r[i], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) s += r[i];
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

}  // namespace

extern "C" fxc_status fxc_probe_fp32_peak(int32_t device, double* tflops) {
  if (!tflops) return FXC_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return FXC_EINVAL;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return FXC_ECUDA;
  float* d = nullptr;
  if (cudaMalloc(&d, 16) != cudaSuccess) return FXC_ENOMEM;
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_probe_kernel<<<blocks, threads>>>(d, iters, 0.999f, 1e-4f);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    fma_probe_kernel<<<blocks, threads>>>(d, iters, 0.999f, 1e-4f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  cudaSetDevice(prev);
  if (err != cudaSuccess) return FXC_ECUDA;
  const double flops = 2.0 * 16.0 * (double)iters * (double)threads * (double)blocks;
  *tflops = flops / ((double)best * 1e-3) / 1e12;
  return FXC_OK;
}
