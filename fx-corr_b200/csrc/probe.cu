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

// ------------------------------------------------- design-choice probes
//
// Two measurements behind the FFT-8192 kernel's design, reported by
// fxc_probe_exchange and fxc_probe_mma_f16:
//  * the cost of redistributing a frame's 8192 complex values among a CTA's
//    512 threads (16 per thread) through padded shared memory, the exchange
//    between two radix-16 passes (store, barrier, strided load, barrier),
//    against the same number of values redistributed by warp shuffles (a
//    16 x 16 transpose within each half-warp, four butterfly stages of
//    shfl.xor; a shuffle moves one 32-bit word, so a complex value costs two);
//  * the throughput of the legacy warp-level tensor instruction
//    (mma.sync m16n8k16, f16 inputs, f32 accumulation) on this GPU, which
//    bounds a DFT-as-matrix-product radix stage written with it.

namespace {

constexpr int kExT = 512;
constexpr int kExStride = 8192 + 512;  // padded complex buffer (one pad per 16)

__global__ void __launch_bounds__(kExT, 1) exchange_smem_kernel(float* out, int iters) {
  extern __shared__ __align__(16) float2 xbuf[];
  const int t = threadIdx.x;
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = make_float2((float)(t + r), (float)(t - r));
  for (int it = 0; it < iters; ++it) {
    float2* dst = xbuf + 17 * t;  // cpad(16 t + r) = 17 t + r
#pragma unroll
    for (int r = 0; r < 16; ++r) dst[r] = v[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int j = t + kExT * r;
      v[r] = xbuf[j + (j >> 4)];
    }
    __syncthreads();
  }
  float s = 0.f;
#pragma unroll
  for (int r = 0; r < 16; ++r) s += v[r].x - v[r].y;
  if (s == 12345.678f) out[0] = s;
}

__device__ __forceinline__ float2 shfl_xor2(float2 a, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, a.x, m), __shfl_xor_sync(0xffffffffu, a.y, m));
}

__global__ void __launch_bounds__(kExT, 1) exchange_shfl_kernel(float* out, int iters) {
  const int t = threadIdx.x;
  const int lane = t & 31;
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = make_float2((float)(t + r), (float)(t - r));
  for (int it = 0; it < iters; ++it) {
    // 16 x 16 transpose within each half-warp: at stage s a lane trades the
    // half of its values whose index differs from its lane in bit s
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int m = 1 << s;
      const bool up = (lane & m) != 0;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        if (i & m) continue;
        const float2 send = up ? v[i] : v[i | m];
        const float2 got = shfl_xor2(send, m);
        if (up) v[i] = got;
        else v[i | m] = got;
      }
    }
  }
  float s = 0.f;
#pragma unroll
  for (int r = 0; r < 16; ++r) s += v[r].x - v[r].y;
  if (s == 12345.678f) out[0] = s;
}

__global__ void mma_f16_probe_kernel(float* out, int iters) {
  // eight independent accumulator tiles per warp keep the tensor pipe fed
  uint32_t a[4], b[2];
#pragma unroll
  for (int i = 0; i < 4; ++i) a[i] = 0x3c003c00u ^ (threadIdx.x << 2) ^ i;  // ~1.0 halves
#pragma unroll
  for (int i = 0; i < 2; ++i) b[i] = 0x38003800u ^ (threadIdx.x << 3) ^ i;
  float c[8][4];
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int i = 0; i < 4; ++i) c[k][i] = 0.f;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      asm volatile(
          "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 "
          "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
          : "+f"(c[k][0]), "+f"(c[k][1]), "+f"(c[k][2]), "+f"(c[k][3])
          : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int i = 0; i < 4; ++i) s += c[k][i];
  if (s == 12345.678f) out[0] = s;
}

// Best of `reps` timed launches (ms) of launch() after one warm-up.
template <typename F>
float best_ms(F launch, int reps) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  launch();
  float best = 1e30f;
  for (int rep = 0; rep < reps; ++rep) {
    cudaEventRecord(e0);
    launch();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

}  // namespace

extern "C" fxc_status fxc_probe_exchange(int32_t device, double* smem_ns, double* shfl_ns) {
  if (!smem_ns || !shfl_ns) return FXC_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return FXC_EINVAL;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return FXC_ECUDA;
  float* d = nullptr;
  if (cudaMalloc(&d, 16) != cudaSuccess) return FXC_ENOMEM;
  const int smem = kExStride * (int)sizeof(float2);
  cudaFuncSetAttribute(exchange_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int blocks = prop.multiProcessorCount, iters = 2048;
  const float a = best_ms([&] { exchange_smem_kernel<<<blocks, kExT, smem>>>(d, iters); }, 5);
  const float b = best_ms([&] { exchange_shfl_kernel<<<blocks, kExT>>>(d, iters); }, 5);
  const cudaError_t err = cudaGetLastError();
  cudaFree(d);
  cudaSetDevice(prev);
  if (err != cudaSuccess) return FXC_ECUDA;
  // time per redistribution of one frame's 8192 complex values on one SM
  *smem_ns = (double)a * 1e6 / iters;
  *shfl_ns = (double)b * 1e6 / iters;
  return FXC_OK;
}

extern "C" fxc_status fxc_probe_mma_f16(int32_t device, double* tflops) {
  if (!tflops) return FXC_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return FXC_EINVAL;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return FXC_ECUDA;
  float* d = nullptr;
  if (cudaMalloc(&d, 16) != cudaSuccess) return FXC_ENOMEM;
  const int threads = 256, blocks = prop.multiProcessorCount * 4, iters = 4096;
  const float ms = best_ms([&] { mma_f16_probe_kernel<<<blocks, threads>>>(d, iters); }, 5);
  const cudaError_t err = cudaGetLastError();
  cudaFree(d);
  cudaSetDevice(prev);
  if (err != cudaSuccess) return FXC_ECUDA;
  const double mmas = 8.0 * iters * (threads / 32.0) * blocks;
  *tflops = mmas * 2.0 * 16 * 8 * 16 / ((double)ms * 1e-3) / 1e12;
  return FXC_OK;
}
