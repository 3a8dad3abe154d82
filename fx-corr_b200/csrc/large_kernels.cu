// large_kernels.cu — correlation path for FFT lengths above one CTA's shared
// memory (N = C * M with M = 8192, C in {2, 4, 8}: N = 16384 .. 65536).
//
// The N-point complex FFT of z = x1 + i x2 runs as one decimation-in-frequency
// radix-C step over the frame followed by C shared-memory FFTs of M points:
//   y_q[m] = W_N^(m q) * sum_c z[m + M c] W_C^(c q),   Z[C k + q] = FFT_M(y_q)[k].
// Kernels, per batch of frames held in device scratch:
//   rows_fft_kernel<C>    C = 2: decode + shift + radix-C step + row FFT fused,
//                         one (frame, row) per CTA iteration, the frame's packed words
//                         staged in shared memory by bulk copies             -> Z
//   dif_staged_kernel<C>  C = 4, 8: decode + shift (src/utils.rs:126-376) + radix-C
//                         step from the frame's words staged in shared memory -> y
//   cfft_kernel<M>        M-point Stockham FFT per row, the next row prefetched by
//                         a bulk copy                                         -> Z
//   acc_global_kernel     two-for-one split, band alignment, fringe x ramp rotation and
//                         ACF/XCF accumulation (src/main.rs:2491-2568) per bin, f32 over
//                         each frame group (<= 32 frames), then f64 per-group partials
//                         reduced by reduce_partials_kernel.
//   phased_global_kernel  per-bin phased synthesis (src/main.rs:2222-2365) and the
//                         Hermitian-extended inverse input; rows_fft_complex_kernel<C>
//                         (C <= 4) or dif_kernel + cfft_kernel its FFT; quant_global_kernel
//                         the re-quantised .raw frames (src/utils.rs:378-410).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "decode_tables.cuh"
#include "fxc_device.cuh"
#include "fxc_kernels.h"

namespace fxc {

constexpr int kLargeM = 8192;

// One decoded, shifted sample of a station (0 outside [0, N)).
__device__ __forceinline__ float sample_at(const uint8_t* __restrict__ frame, int bits, int kind,
                                           const uint32_t* lut, const float* lv, int lsb, int m,
                                           int n) {
  if ((unsigned)m >= (unsigned)n) return 0.f;
  const uint32_t bit = (uint32_t)m * (uint32_t)bits;
  const uint32_t w = shuffle_word(reinterpret_cast<const uint32_t*>(frame)[bit >> 5], kind, lut);
  const float v = lv[(w >> (bit & 31u)) & ((1u << bits) - 1u)];
  return (lsb && (m & 1)) ? -v : v;
}

// z[f][n] = x1[n - s1] + i x2[n - s2] (levels scaled by the stations' exact
// powers of two), or, with planar outputs, x1 / x2 unscaled.
__global__ void decode_global_kernel(const LargeParams p, uint64_t f0, uint64_t nb, float2* z,
                                     float* x1o, float* x2o) {
  __shared__ uint32_t lut[2048];
  __shared__ float lv[512];
  for (int i = threadIdx.x; i < 512; i += blockDim.x)
    lv[i] = p.st[i >> 8].levels[i & 255] * p.st[i >> 8].scale;
  for (int s = 0; s < 2; ++s)
    if (p.st[s].shkind == SH_GENERIC)
      for (int i = threadIdx.x; i < 1024; i += blockDim.x) lut[s * 1024 + i] = p.st[s].shlut[i];
  __syncthreads();
  const int n = p.n;
  const uint64_t total = nb * (uint64_t)n;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t fl = idx / (uint64_t)n;
    const int k = (int)(idx - fl * (uint64_t)n);
    const uint64_t f = f0 + fl;
    const FrameInfo& F = p.finfo[f];
    const float a = sample_at(p.st[0].raw + f * p.st[0].bpf, p.st[0].bits, p.st[0].shkind, lut,
                              lv, p.st[0].lsb, k - F.s1, n);
    const float b = sample_at(p.st[1].raw + f * p.st[1].bpf, p.st[1].bits, p.st[1].shkind,
                              lut + 1024, lv + 256, p.st[1].lsb, k - F.s2, n);
    if (z) {
      // station 2 enters odd frames negated (undone after the FFT), so the
      // shared FFT's cross-station rounding leak alternates in sign and
      // cancels over frames instead of biasing the cross-spectrum
      z[idx] = make_float2(a, (f & 1u) ? -b : b);
    } else {
      x1o[f * n + k] = a / p.st[0].scale;
      x2o[f * n + k] = b / p.st[1].scale;
    }
  }
}

// ---------------------------------------------- fused decode + DIF + row FFT
//
// One work item = one row q of one frame: the frame's packed words are staged
// in shared memory by bulk copies (the next item's copies in flight while this
// one computes), thread t decodes its 16 column inputs m = t + 512 r straight
// from the words for every segment c (samples m + M c of both stations, the
// integer shifts and zero fill applied at the sample index), forms the
// radix-C decimation-in-frequency input
//   y_q[m] = W_N^(m q) * sum_c z[m + M c] W_C^(c q),   z = x1 + i x2,
// and runs the M-point Stockham FFT of the row in shared memory; the row's
// spectrum Z[C k + q] goes to y[f][q M + k], the layout acc_global_kernel and
// the phased kernels read.  This replaces a decode + DIF kernel and cfft_kernel (two
// round trips of the complex frame through global memory) when the frame's
// words fit the staging space.

// Shared-memory layout (bytes): level tables (station 1 at 0, station 2 at
// 2048, 2^b f32 each then their negations), rotate amounts, mbarriers, error
// flag, byte LUTs of 4/8-bit generic shuffles, the two padded FFT buffers,
// then the staging slots [FrameInfo (128 B)][station 1 words][station 2 words].
constexpr uint32_t kRwPos = kTabPos, kRwBar = 4352, kRwFlag = 4384, kRwLut = kTabLut;
constexpr uint32_t kRwA = kRwLut + 8192;
constexpr uint32_t kRwBuf = (uint32_t)Geom<kLargeM>::CSTRIDE * (uint32_t)sizeof(float2);
constexpr uint32_t kRwStage0 = kRwA + 2 * kRwBuf;
constexpr uint32_t kRwMaxSmem = 232448;  // 227 KB per CTA on sm_100

__host__ __device__ inline uint32_t rows_stage_stride(uint32_t bpf1, uint32_t bpf2) {
  return (128u + bpf1 + bpf2 + 127u) & ~127u;
}

// Staging slots that fit: 2 (copies overlap the previous item) or 1; 0 = the
// frame does not fit (the two-kernel path runs instead).
__host__ __device__ inline int rows_stages(uint32_t bpf1, uint32_t bpf2) {
  const uint32_t st = rows_stage_stride(bpf1, bpf2);
  if (kRwStage0 + 2 * st <= kRwMaxSmem) return 2;
  if (kRwStage0 + st <= kRwMaxSmem) return 1;
  return 0;
}

// Adds station ST's samples of the C segments to the 16 column inputs: x at
// m0 + 512 r + M c (zero outside the frame) times W_C^(c q) (ST = 1: times
// i W_C^(c q), the imaginary part of z).  The sample's bits are rotated to
// byte-offset bits 2.. of the level table and merged with tbase (which picks
// the station's table and the negated copy for odd samples of LSB input or
// station 2 on odd frames), as in the FFT-8192 kernel.
template <int C, int BITS, bool SPLIT, int ST>
__device__ __forceinline__ void rows_station(const uint32_t* __restrict__ words,
                                             const uint8_t* lvbase, int m0, uint32_t rots,
                                             uint32_t tbase, const float2 (&wq)[C],
                                             float2 (&v)[16]) {
  constexpr int M = kLargeM, N = C * M;
  constexpr int SPW = 32 / BITS;
  constexpr int LOG2_SPW = BITS == 1 ? 5 : (BITS == 2 ? 4 : (BITS == 4 ? 3 : 2));
  constexpr int WSTEP = 512 / SPW, SEGW = M / SPW;
  constexpr uint32_t OMASK = ((1u << BITS) - 1u) << 2;
  const int w0 = m0 >> LOG2_SPW;  // floor division
  const uint32_t r0 = rots & 31u, r1 = (rots >> 8) & 31u;
  auto level = [&](uint32_t w) -> float {
    uint32_t off;
    if constexpr (SPLIT) {
      off = (__funnelshift_r(w, w, r0) & 4u) | tbase;
      off |= __funnelshift_r(w, w, r1) & 8u;
    } else {
      off = (__funnelshift_r(w, w, r0) & OMASK) | tbase;
    }
    return *reinterpret_cast<const float*>(lvbase + off);
  };
  auto add = [&](int r, int c, float x) {
    if constexpr (ST == 0) {
      v[r].x = fmaf(x, wq[c].x, v[r].x);
      v[r].y = fmaf(x, wq[c].y, v[r].y);
    } else {
      v[r].x = fmaf(-x, wq[c].y, v[r].x);
      v[r].y = fmaf(x, wq[c].x, v[r].y);
    }
  };
  if ((unsigned)m0 < 512u) {
    // every sample of this thread lies inside the frame
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int r = 0; r < 16; ++r) add(r, c, level(words[w0 + r * WSTEP + c * SEGW]));
  } else {
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int m = m0 + r * 512 + c * M;
        const bool in = (unsigned)m < (unsigned)N;
        const float x = level(words[in ? w0 + r * WSTEP + c * SEGW : 0]);
        add(r, c, in ? x : 0.0f);
      }
  }
}

template <int C, int ST>
__device__ __forceinline__ void rows_station_any(int bits, bool split, const uint32_t* words,
                                                 const uint8_t* lvbase, int m0, uint32_t rots,
                                                 uint32_t tbase, const float2 (&wq)[C],
                                                 float2 (&v)[16]) {
  switch (bits) {
    case 1: rows_station<C, 1, false, ST>(words, lvbase, m0, rots, tbase, wq, v); break;
    case 2:
      if (split) rows_station<C, 2, true, ST>(words, lvbase, m0, rots, tbase, wq, v);
      else rows_station<C, 2, false, ST>(words, lvbase, m0, rots, tbase, wq, v);
      break;
    case 4: rows_station<C, 4, false, ST>(words, lvbase, m0, rots, tbase, wq, v); break;
    default: rows_station<C, 8, false, ST>(words, lvbase, m0, rots, tbase, wq, v); break;
  }
}

template <int C>
__global__ void __launch_bounds__(512, 1) rows_fft_kernel(const LargeParams p, uint64_t f0,
                                                          uint64_t nb, float2* __restrict__ y) {
  constexpr int M = kLargeM, N = C * M, T = M / 16;
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x;
  uint32_t* pos = reinterpret_cast<uint32_t*>(smem + kRwPos);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kRwBar);
  int* flag = reinterpret_cast<int*>(smem + kRwFlag);
  uint32_t* lut = reinterpret_cast<uint32_t*>(smem + kRwLut);
  float2* bufA = reinterpret_cast<float2*>(smem + kRwA);
  float2* bufB = reinterpret_cast<float2*>(smem + kRwA + kRwBuf);
  uint8_t* stage = smem + kRwStage0;
  const StationParams& s1 = p.st[0];
  const StationParams& s2 = p.st[1];
  const uint32_t bpf1 = s1.bpf, bpf2 = s2.bpf;
  const uint32_t stride = rows_stage_stride(bpf1, bpf2);
  const int stages = rows_stages(bpf1, bpf2);
  // 4- and 8-bit stations with a non-identity shuffle are rewritten in place
  // (byte LUTs); 1- and 2-bit stations are decoded from the raw words
  const bool pre1 = s1.bits > 2 && s1.shkind != SH_IDENTITY;
  const bool pre2 = s2.bits > 2 && s2.shkind != SH_IDENTITY;
  const uint64_t items = nb * (uint64_t)C;

  if (tid == 0) {
    for (int k = 0; k < 2; ++k) mbar_init(&bars[k], 1);
    *flag = 0;
    fence_proxy_async();
  }
  build_decode_tables(s1, s2, pre1, pre2, smem, tid, T);
  const bool sp1 = split_2bit(s1), sp2 = split_2bit(s2);
  Twiddles<M> tw;
  tw.init(tid);

  // item i of this CTA's sequence: batch item blockIdx.x + i * gridDim.x
  auto item_of = [&](uint32_t i) { return (uint64_t)blockIdx.x + (uint64_t)i * gridDim.x; };
  auto issue = [&](uint32_t i) {
    const uint64_t f = f0 + item_of(i) / C;  // sector-local frame
    const int slot = (int)(i % (uint32_t)stages);
    uint8_t* dst = stage + slot * stride;
    mbar_expect_tx(&bars[slot], kFiBytes + bpf1 + bpf2);
    bulk_g2s(dst, p.finfo + f, kFiBytes, &bars[slot]);
    bulk_g2s(dst + 128, s1.raw + f * bpf1, bpf1, &bars[slot]);
    bulk_g2s(dst + 128 + bpf1, s2.raw + f * bpf2, bpf2, &bars[slot]);
  };
  __syncthreads();  // mbarriers and tables
  if (tid == 0) {
    fence_proxy_async();
    for (uint32_t i = 0; i < (uint32_t)stages && item_of(i) < items; ++i) issue(i);
  }
  for (uint32_t i = 0; item_of(i) < items; ++i) {
    const uint64_t it = item_of(i);
    const uint64_t fl = it / C;          // batch-local frame
    const int q = (int)(it % C);         // row
    const int slot = (int)(i % (uint32_t)stages);
    const uint32_t parity = (i / (uint32_t)stages) & 1u;
    if (!mbar_wait(&bars[slot], parity, kWaitPolls)) {
      atomicOr(flag, 1);
      atomicOr(p.err, ERR_WAIT_TIMEOUT);
    }
    uint8_t* st = stage + slot * stride;
    uint32_t* w1 = reinterpret_cast<uint32_t*>(st + 128);
    uint32_t* w2 = reinterpret_cast<uint32_t*>(st + 128 + bpf1);
    __syncthreads();  // every thread past its wait (and the flag visible)
    if (*flag) break;
    if (pre1 || pre2) {
      preshuffle_slot(w1, bpf1 / 4, pre1 ? s1.shkind : SH_IDENTITY, lut, w2, bpf2 / 4,
                      pre2 ? s2.shkind : SH_IDENTITY, lut + 1024, tid, T);
      __syncthreads();
    }
    const FrameInfo* F = reinterpret_cast<const FrameInfo*>(st);
    const uint64_t f = f0 + fl;
    const int odd = (int)(f & 1u);  // station 2 enters odd frames negated
    // radix-C weights W_C^(c q)
    float2 wq[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const int e = (c * q) % C;
      float sn, cs;
      sincospif(-2.0f * (float)e / (float)C, &sn, &cs);
      wq[c] = make_float2(cs, sn);
    }
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = make_float2(0.f, 0.f);
    {
      const int m1 = tid - F->s1, m2 = tid - F->s2;
      const int c1 = m1 & ((32 / s1.bits) - 1), c2 = m2 & ((32 / s2.bits) - 1);
      const uint32_t tb1 = (uint32_t)((m1 & (s1.lsb ? 1 : 0)) << (s1.bits + 2));
      const uint32_t tb2 = 2048u + (uint32_t)((((uint32_t)m2 & (uint32_t)(s2.lsb ? 1 : 0)) ^
                                               (uint32_t)odd) << (s2.bits + 2));
      rows_station_any<C, 0>(s1.bits, sp1, w1, smem, m1, pos[c1], tb1, wq, v);
      rows_station_any<C, 1>(s2.bits, sp2, w2, smem, m2, pos[32 + c2], tb2, wq, v);
    }
    if (q > 0) {
      // W_N^(m q), m = t + 512 r (m q < N)
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = cmul(v[r], p.tw[(tid + 512 * r) * q]);
    }
    __syncthreads();  // the staged words are consumed: refill the slot
    if (tid == 0 && item_of(i + stages) < items) {
      fence_proxy_async();
      issue(i + stages);
    }
    dft16(v);
    float2* dst = bufA + 17 * tid;  // cpad(16 t + r) = 17 t + r
#pragma unroll
    for (int r = 0; r < 16; ++r) dst[r] = v[out_pos<16>(r)];
    const float2* Z = fft_rest<M>(bufA, bufB, tid, tw);
    __syncthreads();
    float4* out = reinterpret_cast<float4*>(y + fl * (uint64_t)N + (uint64_t)q * M);
    const float4* zin = reinterpret_cast<const float4*>(Z);
    for (int k = tid; k < M / 2; k += T) out[k] = zin[k];
    __syncthreads();  // the buffers are free for the next item
  }
  if (tid == 0 && *flag) {
    for (int k = 0; k < stages; ++k) mbar_wait(&bars[k], 0, kWaitPolls);
  }
}

// Decode + shift + radix-C step with the frame's words staged in shared memory
// (the C = 4 and 8 forward path, and frames too large for rows_fft_kernel's
// staging): one frame per CTA iteration, thread t decodes its 16 columns
// m = t + 512 r from the staged words (each sample once), forms the C-point
// DFT of z[m + M c] and writes y[f][q M + m] = W_N^(m q) Z_c->q for every row q,
// the input of cfft_kernel.  The next frame's copies are in flight meanwhile.
constexpr uint32_t kDsStage0 = kRwA;  // tables as rows_fft_kernel, then the staging slots

__host__ __device__ inline int dif_staged_stages(uint32_t bpf1, uint32_t bpf2) {
  const uint32_t st = rows_stage_stride(bpf1, bpf2);
  if (kDsStage0 + 2 * st <= kRwMaxSmem) return 2;
  if (kDsStage0 + st <= kRwMaxSmem) return 1;
  return 0;
}

// One sample of a station (0 outside the frame): m is the sample index, w the
// word index of m (m >> log2(samples per word)), the rotate amounts and table
// base as in rows_station.
__device__ __forceinline__ float staged_sample(const uint32_t* words, const uint8_t* lvbase, int m,
                                               int w, int n, uint32_t rots, uint32_t omask,
                                               uint32_t tbase, bool split) {
  if ((unsigned)m >= (unsigned)n) return 0.0f;
  const uint32_t x = words[w];
  uint32_t off;
  if (split) {
    off = (__funnelshift_r(x, x, rots & 31u) & 4u) | tbase;
    off |= __funnelshift_r(x, x, (rots >> 8) & 31u) & 8u;
  } else {
    off = (__funnelshift_r(x, x, rots & 31u) & omask) | tbase;
  }
  return *reinterpret_cast<const float*>(lvbase + off);
}

template <int C>
__global__ void __launch_bounds__(512, 1) dif_staged_kernel(const LargeParams p, uint64_t f0,
                                                            uint64_t nb, float2* __restrict__ y) {
  constexpr int M = kLargeM, N = C * M, T = 512;
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x;
  uint32_t* pos = reinterpret_cast<uint32_t*>(smem + kRwPos);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kRwBar);
  int* flag = reinterpret_cast<int*>(smem + kRwFlag);
  uint32_t* lut = reinterpret_cast<uint32_t*>(smem + kRwLut);
  uint8_t* stage = smem + kDsStage0;
  const StationParams& s1 = p.st[0];
  const StationParams& s2 = p.st[1];
  const uint32_t bpf1 = s1.bpf, bpf2 = s2.bpf;
  const uint32_t stride = rows_stage_stride(bpf1, bpf2);
  const int stages = dif_staged_stages(bpf1, bpf2);
  const bool pre1 = s1.bits > 2 && s1.shkind != SH_IDENTITY;
  const bool pre2 = s2.bits > 2 && s2.shkind != SH_IDENTITY;

  if (tid == 0) {
    for (int k = 0; k < 2; ++k) mbar_init(&bars[k], 1);
    *flag = 0;
    fence_proxy_async();
  }
  build_decode_tables(s1, s2, pre1, pre2, smem, tid, T);
  const bool sp1 = split_2bit(s1), sp2 = split_2bit(s2);
  const int lg1 = s1.bits == 1 ? 5 : (s1.bits == 2 ? 4 : (s1.bits == 4 ? 3 : 2));
  const int lg2 = s2.bits == 1 ? 5 : (s2.bits == 2 ? 4 : (s2.bits == 4 ? 3 : 2));
  const uint32_t om1 = ((1u << s1.bits) - 1u) << 2, om2 = ((1u << s2.bits) - 1u) << 2;

  auto frame_of = [&](uint32_t i) { return (uint64_t)blockIdx.x + (uint64_t)i * gridDim.x; };
  auto issue = [&](uint32_t i) {
    const uint64_t f = f0 + frame_of(i);
    const int slot = (int)(i % (uint32_t)stages);
    uint8_t* dst = stage + slot * stride;
    mbar_expect_tx(&bars[slot], kFiBytes + bpf1 + bpf2);
    bulk_g2s(dst, p.finfo + f, kFiBytes, &bars[slot]);
    bulk_g2s(dst + 128, s1.raw + f * bpf1, bpf1, &bars[slot]);
    bulk_g2s(dst + 128 + bpf1, s2.raw + f * bpf2, bpf2, &bars[slot]);
  };
  __syncthreads();
  if (tid == 0) {
    fence_proxy_async();
    for (uint32_t i = 0; i < (uint32_t)stages && frame_of(i) < nb; ++i) issue(i);
  }
  for (uint32_t i = 0; frame_of(i) < nb; ++i) {
    const uint64_t fl = frame_of(i);
    const int slot = (int)(i % (uint32_t)stages);
    const uint32_t parity = (i / (uint32_t)stages) & 1u;
    if (!mbar_wait(&bars[slot], parity, kWaitPolls)) {
      atomicOr(flag, 1);
      atomicOr(p.err, ERR_WAIT_TIMEOUT);
    }
    uint8_t* st = stage + slot * stride;
    const uint32_t* w1 = reinterpret_cast<const uint32_t*>(st + 128);
    const uint32_t* w2 = reinterpret_cast<const uint32_t*>(st + 128 + bpf1);
    __syncthreads();
    if (*flag) break;
    if (pre1 || pre2) {
      preshuffle_slot(const_cast<uint32_t*>(w1), bpf1 / 4, pre1 ? s1.shkind : SH_IDENTITY, lut,
                      const_cast<uint32_t*>(w2), bpf2 / 4, pre2 ? s2.shkind : SH_IDENTITY,
                      lut + 1024, tid, T);
      __syncthreads();
    }
    const FrameInfo* F = reinterpret_cast<const FrameInfo*>(st);
    const uint64_t f = f0 + fl;
    const uint32_t odd = (uint32_t)(f & 1u);  // station 2 enters odd frames negated
    const int m1 = tid - F->s1, m2 = tid - F->s2;
    const uint32_t rot1 = pos[m1 & ((32 / s1.bits) - 1)], rot2 = pos[32 + (m2 & ((32 / s2.bits) - 1))];
    const uint32_t tb1 = (uint32_t)((m1 & (s1.lsb ? 1 : 0)) << (s1.bits + 2));
    const uint32_t tb2 = 2048u + (uint32_t)((((uint32_t)m2 & (uint32_t)(s2.lsb ? 1 : 0)) ^ odd)
                                            << (s2.bits + 2));
    const int wb1 = m1 >> lg1, wb2 = m2 >> lg2;  // floor divisions
    float2* yf = y + fl * (uint64_t)N;
#pragma unroll 2
    for (int r = 0; r < 16; ++r) {
      const int m = tid + 512 * r;  // column
      float2 v[16];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int o = 512 * r + M * c;
        const float a = staged_sample(w1, smem, m1 + o, wb1 + (o >> lg1), N, rot1, om1, tb1, sp1);
        const float b = staged_sample(w2, smem, m2 + o, wb2 + (o >> lg2), N, rot2, om2, tb2, sp2);
        v[c] = make_float2(a, b);
      }
      if constexpr (C == 2) {
        dft2<0>(v);
      } else if constexpr (C == 4) {
        dft4<0>(v);
      } else {
        dft8<0>(v);
      }
#pragma unroll
      for (int q = 0; q < C; ++q) {
        float2 val = v[out_pos<C>(q)];
        if (q > 0) val = cmul(val, p.tw[m * q]);  // W_N^(m q), m q < N
        yf[q * M + m] = val;
      }
    }
    __syncthreads();  // the staged words are consumed: refill the slot
    if (tid == 0 && frame_of(i + stages) < nb) {
      fence_proxy_async();
      issue(i + stages);
    }
  }
  if (tid == 0 && *flag) {
    for (int k = 0; k < stages; ++k) mbar_wait(&bars[k], 0, kWaitPolls);
  }
}

// The same fused DIF + row FFT on a complex input already in global memory
// (the phased path's Hermitian-extended spectra): item (frame f, row q) reads
// x[f][m + M c] for its 16 columns and every segment, forms
// y_q[m] = W_N^(m q) sum_c x[m + M c] W_C^(c q) and writes FFT_M(y_q) to
// y[f][q M + k].  Replaces dif_kernel + cfft_kernel (one global round trip).
template <int C>
__global__ void __launch_bounds__(512, 1) rows_fft_complex_kernel(const float2* __restrict__ x,
                                                                  float2* __restrict__ y,
                                                                  uint64_t nb,
                                                                  const float2* __restrict__ twn) {
  constexpr int M = kLargeM, N = C * M, T = M / 16;
  extern __shared__ __align__(128) uint8_t smem[];
  float2* bufA = reinterpret_cast<float2*>(smem);
  float2* bufB = reinterpret_cast<float2*>(smem + kRwBuf);
  const int tid = threadIdx.x;
  Twiddles<M> tw;
  tw.init(tid);
  const uint64_t items = nb * (uint64_t)C;
  for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const uint64_t fl = it / C;
    const int q = (int)(it % C);
    const float2* xf = x + fl * (uint64_t)N;
    float2 wq[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      float sn, cs;
      sincospif(-2.0f * (float)((c * q) % C) / (float)C, &sn, &cs);
      wq[c] = make_float2(cs, sn);
    }
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const float2 z = xf[tid + 512 * r + M * c];
        a.x = fmaf(z.x, wq[c].x, fmaf(-z.y, wq[c].y, a.x));
        a.y = fmaf(z.x, wq[c].y, fmaf(z.y, wq[c].x, a.y));
      }
      v[r] = q > 0 ? cmul(a, twn[(tid + 512 * r) * q]) : a;  // W_N^(m q), m q < N
    }
    dft16(v);
    float2* dst = bufA + 17 * tid;  // cpad(16 t + r) = 17 t + r
#pragma unroll
    for (int r = 0; r < 16; ++r) dst[r] = v[out_pos<16>(r)];
    const float2* Z = fft_rest<M>(bufA, bufB, tid, tw);
    __syncthreads();
    float4* out = reinterpret_cast<float4*>(y + fl * (uint64_t)N + (uint64_t)q * M);
    const float4* zin = reinterpret_cast<const float4*>(Z);
    for (int k = tid; k < M / 2; k += T) out[k] = zin[k];
    __syncthreads();  // the buffers are free for the next item
  }
}

// W_N^j = exp(-2 pi i j / N), j < N, correctly rounded from FP64.
__global__ void twiddle_table_kernel(int n, float2* __restrict__ tw) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double s, c;
  sincospi(-2.0 * (double)j / (double)n, &s, &c);
  tw[j] = make_float2((float)c, (float)s);
}

template <int C>
__global__ void dif_kernel(const float2* __restrict__ z, float2* __restrict__ y, uint64_t nb,
                           const float2* __restrict__ tw) {
  constexpr int M = kLargeM;
  constexpr int N = C * M;
  const uint64_t total = nb * (uint64_t)M;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t f = idx / M;
    const int m = (int)(idx - f * M);
    const float2* zf = z + f * N;
    float2 v[16];
#pragma unroll
    for (int c = 0; c < C; ++c) v[c] = zf[m + M * c];
    if constexpr (C == 2) {
      dft2<0>(v);
    } else if constexpr (C == 4) {
      dft4<0>(v);
    } else {
      dft8<0>(v);
    }
    float2* yf = y + f * N;
#pragma unroll
    for (int q = 0; q < C; ++q) {
      float2 val = v[out_pos<C>(q)];
      if (q > 0) val = cmul(val, tw[m * q]);  // W_N^(m q), m q < N
      yf[q * M + m] = val;
    }
  }
}

// In-place M-point FFT of each row of y (rows of M complex values), natural
// order.  The next row of the CTA is brought into a shared-memory staging
// row by a bulk copy while the current row is transformed.
template <int M>
__global__ void __launch_bounds__(M / 16, 1) cfft_kernel(float2* __restrict__ y, uint64_t rows,
                                                         uint32_t* err) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr int T1 = M / 16;
  constexpr uint32_t kRowBytes = (uint32_t)M * sizeof(float2);
  float2* bufA = reinterpret_cast<float2*>(smem);
  float2* bufB = bufA + Geom<M>::CSTRIDE;
  float2* stg = bufB + Geom<M>::CSTRIDE;  // one row, unpadded
  uint64_t* bar = reinterpret_cast<uint64_t*>(stg + M);
  int* flag = reinterpret_cast<int*>(bar + 1);
  const int t = threadIdx.x;
  Twiddles<M> tw;
  tw.init(t);
  if (t == 0) {
    mbar_init(bar, 1);
    *flag = 0;
    fence_proxy_async();
  }
  __syncthreads();
  auto fetch = [&](uint64_t r) {
    mbar_expect_tx(bar, kRowBytes);
    bulk_g2s(stg, y + r * M, kRowBytes, bar);
  };
  if (t == 0 && blockIdx.x < rows) fetch(blockIdx.x);
  uint32_t n = 0;  // rows consumed
  for (uint64_t r = blockIdx.x; r < rows; r += gridDim.x, ++n) {
    if (!mbar_wait(bar, n & 1u, kWaitPolls)) {
      atomicOr(flag, 1);
      atomicOr(err, ERR_WAIT_TIMEOUT);
    }
    __syncthreads();
    if (*flag) break;
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = stg[t + T1 * k];
    dft16(v);
    float2* dst = bufA + 17 * t;  // cpad(16 t + r) = 17 t + r
#pragma unroll
    for (int k = 0; k < 16; ++k) dst[k] = v[out_pos<16>(k)];
    float2* Z = fft_rest<M>(bufA, bufB, t, tw);
    // fft_rest opened with a barrier: the staging row is consumed
    if (t == 0 && r + gridDim.x < rows) {
      fence_proxy_async();
      fetch(r + gridDim.x);
    }
    __syncthreads();
    float4* row = reinterpret_cast<float4*>(y + r * M);
    const float4* zin = reinterpret_cast<const float4*>(Z);
    for (int i = t; i < M / 2; i += T1) row[i] = zin[i];
    __syncthreads();
  }
  if (t == 0 && *flag) mbar_wait(bar, 0, kWaitPolls);
}

// Per-bin split + accumulation.  Bin g = C*kk + q: q = blockIdx.y, kk from x,
// so a warp reads consecutive columns of one row.  blockIdx.z = frame group.
__global__ void acc_global_kernel(const LargeParams p, const float2* __restrict__ Y, uint64_t f0,
                                  uint64_t nb, int first_batch, double* __restrict__ part) {
  const int C = p.c, M = kLargeM, N = p.n, H = N / 2 + 1;
  const int q = blockIdx.y;
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  const int bin = C * kk + q;
  if (kk >= M || bin > N / 2) return;
  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s, ov = a1e - a1s, sb = a2s - a1s;
  const int a_gs = p.grid == 0 ? a1s : a2s;
  const bool want_acf = (p.products & 1u) != 0, want_xcf = (p.products & 2u) != 0;
  const bool ov_only = (p.products & 16u) != 0;
  auto zi = [&](const float2* Zf, int k) {  // Z[k] of the natural-order spectrum
    k &= (N - 1);
    return Zf[(k % C) * M + k / C];
  };
  // f32 sums over the group's frames (at most 32 per launch), added to the
  // f64 partials once per launch, as the FFT-8192 kernel flushes its registers
  float a[4] = {0.f, 0.f, 0.f, 0.f};
  const uint64_t groups = gridDim.z;
  const uint64_t g0 = (blockIdx.z * nb) / groups, g1 = ((blockIdx.z + 1) * nb) / groups;
  // unrolled: the frames' loads go out together (the loop is latency-bound)
#pragma unroll 4
  for (uint64_t fl = g0; fl < g1; ++fl) {
    const float2* Zf = Y + fl * (uint64_t)N;
    const FrameInfo& F = p.finfo[f0 + fl];
    float sn, cs;  // SFU sin/cos: |angle| <= ~pi (ramp over the band), abs error < 4e-7
    __sincosf(fmaf((float)(bin - a_gs), F.dphi, F.phi0), &sn, &cs);
    const float2 r = cmul(F.fr_mix, make_float2(cs, sn));
    const float sg = ((f0 + fl) & 1u) ? -1.0f : 1.0f;  // station 2 sign of this frame
    const float2 u = zi(Zf, bin), w = zi(Zf, N - bin);
    if (p.grid == 0) {
      const bool inov = bin >= a1s && bin < a1e;
      const float2 p1 = make_float2(u.x + w.x, u.y - w.y);
      if (want_acf && (!ov_only || inov)) a[0] += cnorm2(p1);
      if (inov) {
        const int i2 = bin + sb;
        const float2 c = zi(Zf, i2), d = zi(Zf, N - i2);
        const float2 q2 = make_float2(sg * (c.y + d.y), sg * (d.x - c.x));
        if (want_acf) a[1] += cnorm2(q2);
        if (want_xcf) {
          const float2 x = cmul(cmulc(p1, q2), r);
          a[2] += x.x;
          a[3] += x.y;
        }
      }
    } else {
      const bool inov = bin >= a2s && bin < a2s + ov;
      const float2 p2 = make_float2(sg * (u.y + w.y), sg * (w.x - u.x));
      if (want_acf && (!ov_only || inov)) a[1] += cnorm2(p2);
      if (inov) {
        const int i1 = bin - sb;
        const float2 c = zi(Zf, i1), d = zi(Zf, N - i1);
        const float2 q1 = make_float2(c.x + d.x, c.y - d.y);
        if (want_acf) a[0] += cnorm2(q1);
        if (want_xcf) {
          const float2 x = cmul(cmulc(q1, p2), r);
          a[2] += x.x;
          a[3] += x.y;
        }
      }
    }
  }
  double* pg = part + (size_t)blockIdx.z * 4 * H;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double* d = pg + (size_t)v * H + bin;
    *d = (first_batch ? 0.0 : *d) + (double)a[v];
  }
}

// Spectra of both stations from the natural-order Z (stage entry point).
__global__ void split_global_kernel(const LargeParams p, const float2* __restrict__ Y,
                                    uint64_t f0, uint64_t nb, float2* s1, float2* s2) {
  const int C = p.c, M = kLargeM, N = p.n, H = N / 2 + 1;
  const uint64_t total = nb * (uint64_t)H;
  const float u1 = 0.5f / p.st[0].scale, u2 = 0.5f / p.st[1].scale;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t fl = idx / H;
    const int k = (int)(idx - fl * H);
    const float2* Zf = Y + fl * (uint64_t)N;
    const int kn = (N - k) & (N - 1);
    const float2 a = Zf[(k % C) * M + k / C], b = Zf[(kn % C) * M + kn / C];
    s1[(f0 + fl) * H + k] = make_float2(u1 * (a.x + b.x), u1 * (a.y - b.y));
    const float v2 = ((f0 + fl) & 1u) ? -u2 : u2;  // undo the odd-frame negation
    s2[(f0 + fl) * H + k] = make_float2(v2 * (a.y + b.y), -v2 * (a.x - b.x));
  }
}

// Phased synthesis per bin (src/main.rs:2254-2280) for FFT lengths above
// 8192: each thread owns bin C*kk + q across its frame group; |cb|^2 goes to
// the group's f64 partials and, for the .raw product, the Hermitian extension
// of conj(cb) (cb[0].im = cb[N/2].im = 0) to W in natural order, so that the
// forward FFT of W is N x the inverse real FFT of cb (src/utils.rs:60-66).
__global__ void phased_global_kernel(const LargeParams p, const PhasedParams pp,
                                     const float2* __restrict__ Y, uint64_t f0, uint64_t nb,
                                     int first_batch, double* __restrict__ part,
                                     float2* __restrict__ W) {
  const int C = p.c, M = kLargeM, N = p.n, H = N / 2 + 1;
  const int q = blockIdx.y;
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  const int bin = C * kk + q;
  if (kk >= M || bin > N / 2) return;
  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s, ov = a1e - a1s, sb = a2s - a1s;
  const float u1 = 0.5f / p.st[0].scale, u2 = 0.5f / p.st[1].scale;
  auto zi = [&](const float2* Zf, int k) {
    k &= (N - 1);
    return Zf[(k % C) * M + k / C];
  };
  // f32 sums over the group's frames (at most 32 per launch), added to the
  // f64 partials once per launch
  float acc = 0.f;
  const uint64_t groups = gridDim.z;
  const uint64_t g0 = (blockIdx.z * nb) / groups, g1 = ((blockIdx.z + 1) * nb) / groups;
  for (uint64_t fl = g0; fl < g1; ++fl) {
    const float2* Zf = Y + fl * (uint64_t)N;
    const FrameInfo& F = p.finfo[f0 + fl];
    const float sg = ((f0 + fl) & 1u) ? -1.0f : 1.0f;  // station 2 sign of this frame
    // spectrum of station s at its own bin k: unscaled, rotated by the
    // station's fractional delay, Nyquist imaginary part zeroed, times fr_lo
    auto station_bin = [&](int s, int k) -> float2 {
      const float2 a = zi(Zf, k), b = zi(Zf, N - k);
      float2 v = s == 0 ? make_float2(u1 * (a.x + b.x), u1 * (a.y - b.y))
                        : make_float2(sg * u2 * (a.y + b.y), sg * u2 * (b.x - a.x));
      // SFU sin/cos: |angle| <= pi |frac| fs k / N <= pi / 2, abs error < 4e-7
      // (as the FFT <= 8192 phased kernels)
      float sn, cs;
      __sincosf((float)k * (s == 0 ? F.st1 : F.st2), &sn, &cs);
      v = cmul(v, make_float2(cs, sn));
      if (k == N / 2) v.y = 0.f;
      return cmul(v, s == 0 ? F.fr_lo1 : F.fr_lo2);
    };
    float2 a1 = make_float2(0.f, 0.f), a2 = make_float2(0.f, 0.f);
    if (p.grid == 0) {
      a1 = station_bin(0, bin);
      if (bin >= a1s && bin < a1e) a2 = station_bin(1, bin + sb);
    } else {
      a2 = station_bin(1, bin);
      if (bin >= a2s && bin < a2s + ov) a1 = station_bin(0, bin - sb);
    }
    float2 cb = make_float2(a1.x * pp.w1 + a2.x * pp.w2, a1.y * pp.w1 + a2.y * pp.w2);
    acc += cnorm2(cb);
    if (pp.want_raw) {
      float2* wf = W + fl * (uint64_t)N;
      if (bin == 0 || bin == N / 2) cb.y = 0.f;
      wf[bin] = make_float2(cb.x, -cb.y);
      if (bin != 0 && bin != N / 2) wf[N - bin] = cb;
    }
  }
  double* d = part + (size_t)blockIdx.z * H + bin;
  *d = (first_batch ? 0.0 : *d) + (double)acc;
}

// Re-quantise and pack the phased time series (quantise_frame,
// src/utils.rs:378-410): x[n] = Re(X[n]) / N in the row layout of the
// FFT output, odd samples negated when both inputs are LSB, nearest of
// ant1's levels, codes LSB-first, ant1's shuffle applied per word.
__global__ void quant_global_kernel(const LargeParams p, const PhasedParams pp,
                                    const float2* __restrict__ X, uint64_t f0, uint64_t nb) {
  __shared__ float ql[256];
  __shared__ uint32_t elut[1024];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) ql[i] = i < (int)pp.nqlevels ? pp.qlevels[i] : 0.f;
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) elut[i] = pp.enc_lut[i];
  __syncthreads();
  const int C = p.c, M = kLargeM, N = p.n;
  const uint32_t spw = 32u / pp.bits_out, wpf = (uint32_t)N / spw;
  const uint32_t qmask = (1u << pp.bits_out) - 1u;
  const float inv_n = 1.0f / (float)N;
  const uint64_t total = nb * (uint64_t)wpf;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t fl = idx / wpf;
    const uint32_t w = (uint32_t)(idx - fl * wpf);
    const float2* Xf = X + fl * (uint64_t)N;
    uint32_t word = 0;
    for (uint32_t i = 0; i < spw; ++i) {
      const int n = (int)(w * spw + i);
      float x = Xf[(n % C) * M + n / C].x * inv_n;
      if (pp.out_lsb && (n & 1)) x = -x;
      word |= (nearest_level(x, ql, (int)pp.nqlevels, pp.qmonotonic) & qmask) << (i * pp.bits_out);
    }
    const uint32_t sw = elut[word & 255u] | elut[256 + ((word >> 8) & 255u)] |
                        elut[512 + ((word >> 16) & 255u)] | elut[768 + (word >> 24)];
    reinterpret_cast<uint32_t*>(pp.raw_out + (f0 + fl) * pp.bpf_out)[w] = sw;
  }
}

// ------------------------------------------------------------- launchers

int large_batch_frames(uint32_t n) {
  // two scratch buffers of batch * n complex f32 each, 64 MiB apiece; a batch
  // is split into at most kLargeGroups frame groups of at most 32 frames each
  // (16384: 512 / 16), the f32 run length of acc_global_kernel's sums
  const uint64_t per = (uint64_t)n * sizeof(float2);
  return (int)std::max<uint64_t>(1, (64ull << 20) / per);
}

static int grid_for(uint64_t work, int threads, int sms) {
  const uint64_t g = (work + threads - 1) / threads;
  return (int)(g < (uint64_t)sms * 8 ? (g ? g : 1) : (uint64_t)sms * 8);
}

// DIF over C columns (buf0 -> buf1), then the M-point row FFTs in place on buf1.
static cudaError_t row_ffts(const LargeParams& p, uint64_t nb, float2* buf1, int sms,
                           cudaStream_t s);

static cudaError_t large_fft_core(const LargeParams& p, uint64_t nb, const float2* buf0,
                                  float2* buf1, int sms, cudaStream_t s) {
  const uint64_t work = nb * kLargeM;
  switch (p.c) {
    case 2: dif_kernel<2><<<grid_for(work, 256, sms), 256, 0, s>>>(buf0, buf1, nb, p.tw); break;
    case 4: dif_kernel<4><<<grid_for(work, 256, sms), 256, 0, s>>>(buf0, buf1, nb, p.tw); break;
    case 8: dif_kernel<8><<<grid_for(work, 256, sms), 256, 0, s>>>(buf0, buf1, nb, p.tw); break;
    default: return cudaErrorInvalidValue;
  }
  return row_ffts(p, nb, buf1, sms, s);
}

static cudaError_t row_ffts(const LargeParams& p, uint64_t nb, float2* buf1, int sms,
                           cudaStream_t s) {
  // two padded FFT buffers, the staging row, its mbarrier and the error flag
  const uint32_t smem = 2 * Geom<kLargeM>::CSTRIDE * sizeof(float2) + kLargeM * sizeof(float2) + 16;
  auto kern = cfft_kernel<kLargeM>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const uint64_t rows = nb * (uint64_t)p.c;
  kern<<<(unsigned)std::min<uint64_t>(rows, (uint64_t)sms), kLargeM / 16, smem, s>>>(buf1, rows,
                                                                                     p.err);
  return cudaGetLastError();
}

// The fused kernel decodes every segment of the frame for each of its C rows.
// Measured against dif_staged_kernel + cfft_kernel (device-resident 2-bit
// sectors): C = 2 (FFT 16384, odd band shift) 201 against 166 Gsample/s;
// C = 4 156 against 165; C = 8 95 against 134.  So it serves C = 2.
bool rows_fft_supported(const LargeParams& p) {
  return p.c == 2 && rows_stages(p.st[0].bpf, p.st[1].bpf) > 0;
}

cudaError_t launch_rows_fft(const LargeParams& p, uint64_t f0, uint64_t nb, float2* y, int sms,
                            cudaStream_t s) {
  const int stages = rows_stages(p.st[0].bpf, p.st[1].bpf);
  const uint32_t smem = kRwStage0 + (uint32_t)stages * rows_stage_stride(p.st[0].bpf, p.st[1].bpf);
  const uint64_t items = nb * (uint64_t)p.c;
  const unsigned grid = (unsigned)std::min<uint64_t>(items, (uint64_t)sms);
  cudaError_t e;
  switch (p.c) {
    case 2:
      e = cudaFuncSetAttribute(rows_fft_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kRwMaxSmem);
      if (e == cudaSuccess) rows_fft_kernel<2><<<grid, 512, smem, s>>>(p, f0, nb, y);
      break;
    case 4:
      e = cudaFuncSetAttribute(rows_fft_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kRwMaxSmem);
      if (e == cudaSuccess) rows_fft_kernel<4><<<grid, 512, smem, s>>>(p, f0, nb, y);
      break;
    case 8:
      e = cudaFuncSetAttribute(rows_fft_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kRwMaxSmem);
      if (e == cudaSuccess) rows_fft_kernel<8><<<grid, 512, smem, s>>>(p, f0, nb, y);
      break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// The DIF step and the row FFTs of a complex input in global memory (x -> y).
cudaError_t launch_rows_fft_complex(const LargeParams& p, uint64_t nb, const float2* x, float2* y,
                                    int sms, cudaStream_t s) {
  const uint32_t smem = 2 * kRwBuf;
  const unsigned grid = (unsigned)std::min<uint64_t>(nb * (uint64_t)p.c, (uint64_t)sms);
  cudaError_t e;
  switch (p.c) {
    case 2:
      e = cudaFuncSetAttribute(rows_fft_complex_kernel<2>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) rows_fft_complex_kernel<2><<<grid, 512, smem, s>>>(x, y, nb, p.tw);
      break;
    case 4:
      e = cudaFuncSetAttribute(rows_fft_complex_kernel<4>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) rows_fft_complex_kernel<4><<<grid, 512, smem, s>>>(x, y, nb, p.tw);
      break;
    case 8:
      e = cudaFuncSetAttribute(rows_fft_complex_kernel<8>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) rows_fft_complex_kernel<8><<<grid, 512, smem, s>>>(x, y, nb, p.tw);
      break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_large_fft(const LargeParams& p, uint64_t f0, uint64_t nb, float2* buf0,
                             float2* buf1, int sms, cudaStream_t s) {
  // decode + DIF + row FFTs fused (rows_fft_kernel) when the frame's words
  // fit its staging; else decode + DIF -> buf1, row FFTs in place on buf1
  (void)buf0;
  if (rows_fft_supported(p)) return launch_rows_fft(p, f0, nb, buf1, sms, s);
  const int dstages = dif_staged_stages(p.st[0].bpf, p.st[1].bpf);
  if (dstages > 0) {
    // decode + DIF from staged words, then the row FFTs
    const uint32_t smem = kDsStage0 + (uint32_t)dstages * rows_stage_stride(p.st[0].bpf, p.st[1].bpf);
    const unsigned grid = (unsigned)std::min<uint64_t>(nb, (uint64_t)sms);
    cudaError_t e;
    switch (p.c) {
      case 2:
        e = cudaFuncSetAttribute(dif_staged_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kRwMaxSmem);
        if (e == cudaSuccess) dif_staged_kernel<2><<<grid, 512, smem, s>>>(p, f0, nb, buf1);
        break;
      case 4:
        e = cudaFuncSetAttribute(dif_staged_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kRwMaxSmem);
        if (e == cudaSuccess) dif_staged_kernel<4><<<grid, 512, smem, s>>>(p, f0, nb, buf1);
        break;
      case 8:
        e = cudaFuncSetAttribute(dif_staged_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kRwMaxSmem);
        if (e == cudaSuccess) dif_staged_kernel<8><<<grid, 512, smem, s>>>(p, f0, nb, buf1);
        break;
      default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return row_ffts(p, nb, buf1, sms, s);
  }
  // every frame of FFT <= 65536 at <= 8 bits fits one staging slot
  return cudaErrorInvalidValue;
}

cudaError_t launch_twiddle_table(int n, float2* tw, cudaStream_t s) {
  twiddle_table_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, tw);
  return cudaGetLastError();
}

cudaError_t launch_large_phased(const LargeParams& p, const PhasedParams& pp, float2* buf0,
                                float2* buf1, uint64_t f0, uint64_t nb, int groups,
                                int first_batch, double* part, int sms, cudaStream_t s) {
  // buf1 holds the spectra; W goes to buf0, its FFT back to buf1
  dim3 grid((kLargeM + 255) / 256, p.c, groups);
  phased_global_kernel<<<grid, 256, 0, s>>>(p, pp, buf1, f0, nb, first_batch, part, buf0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !pp.want_raw) return e;
  e = p.c <= 4 ? launch_rows_fft_complex(p, nb, buf0, buf1, sms, s)
               : large_fft_core(p, nb, buf0, buf1, sms, s);
  if (e != cudaSuccess) return e;
  const uint64_t words = nb * (uint64_t)(p.n / (32 / pp.bits_out));
  quant_global_kernel<<<grid_for(words, 256, sms), 256, 0, s>>>(p, pp, buf1, f0, nb);
  return cudaGetLastError();
}

cudaError_t launch_large_acc(const LargeParams& p, const float2* Y, uint64_t f0, uint64_t nb,
                             int groups, int first_batch, double* part, cudaStream_t s) {
  dim3 grid((kLargeM + 255) / 256, p.c, groups);
  acc_global_kernel<<<grid, 256, 0, s>>>(p, Y, f0, nb, first_batch, part);
  return cudaGetLastError();
}

cudaError_t launch_large_decode(const LargeParams& p, uint64_t f0, uint64_t nb, float* x1,
                                float* x2, int sms, cudaStream_t s) {
  decode_global_kernel<<<grid_for(nb * p.n, 256, sms), 256, 0, s>>>(p, f0, nb, nullptr, x1, x2);
  return cudaGetLastError();
}

cudaError_t launch_large_split(const LargeParams& p, const float2* Y, uint64_t f0, uint64_t nb,
                               float2* s1, float2* s2, int sms, cudaStream_t s) {
  split_global_kernel<<<grid_for(nb * (p.n / 2 + 1), 256, sms), 256, 0, s>>>(p, Y, f0, nb, s1,
                                                                              s2);
  return cudaGetLastError();
}

}  // namespace fxc
