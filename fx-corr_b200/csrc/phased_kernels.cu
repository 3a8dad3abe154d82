// phased_kernels.cu — phased-array synthesis for sm_100a (yi-phasedarray,
// src/main.rs:2222-2412).
//
// Per frame pair, after the same staging / decode / shift / shared two-for-one
// FFT front end as the correlation kernel:
//   1. S1, S2 from the shared spectrum, each rotated by its own fractional
//      delay exp(-2 pi i k df frac_i) with the Nyquist imaginary part zeroed
//      (apply_delay_and_rate_regular_bins, src/utils.rs:69-124);
//   2. fringe phasors fr_lo1 / fr_lo2, band alignment onto the output grid
//      and the weighted sum cb = w1 S1 + w2 S2 (src/main.rs:2264-2280);
//   3. |cb|^2 accumulated per bin (f32 registers, f64 flushes);
//   4. for the .raw product: cb[0].im = cb[N/2].im = 0, the inverse real FFT
//      computed as the forward FFT of the Hermitian-extended conj(cb) scaled by
//      1/N (src/utils.rs:60-66), odd samples negated when both inputs are LSB,
//      nearest-level re-quantisation with ant1's levels and packing with ant1's
//      shuffle (quantise_frame, src/utils.rs:378-410).
#include <cuda_runtime.h>
#include <stdint.h>

#include "fxc_device.cuh"
#include "fxc_kernels.h"

namespace fxc {

// Per-CTA state that outlives one sector: the twiddle bases and the number of
// staging iterations consumed so far (it sets the mbarrier slot and phase, so
// a persistent CTA can run spans of several scans back to back).
template <int N>
struct PhasedCta {
  Twiddles<N> tw;
  uint32_t seq;
};

template <int N, int FPC>
__device__ __forceinline__ void phased_cta_init(uint8_t* smem, const SmemLayout& L,
                                                PhasedCta<N>& c) {
  constexpr int T1 = N / 16;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);
  int* flag = reinterpret_cast<int*>(smem + L.off_flag);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
    *flag = 0;
    fence_proxy_async();
  }
  c.tw.init(threadIdx.x % T1);
  c.seq = 0;
}

// Never leave a bulk copy in flight into a finished CTA's shared memory.
__device__ __forceinline__ void phased_cta_drain(uint8_t* smem, const SmemLayout& L) {
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);
  const int* flag = reinterpret_cast<const int*>(smem + L.off_flag);
  if (threadIdx.x == 0 && *flag) {
    for (int s = 0; s < kStages; ++s) mbar_wait(&bars[s], 0, kWaitPolls);
  }
}

// CTA iterations [it0, it1) (FPC frame pairs each) of the sector p: phased
// power per bin into part[H] (f32 registers, f64 flushes) and, with
// p.want_raw, the re-quantised frames at p.raw_out.  Returns false when a
// bounded wait gave up (the CTA must stop).  Compiled once (not inlined) and
// called by both the single-scan and the batched kernel, so that a frame's
// .raw bytes do not depend on which of them computed it: two inlined copies
// may contract or schedule the floating-point operations differently, which
// moves samples that sit on a quantiser decision boundary.
template <int N, int FPC>
__device__ __noinline__ bool phased_span(const PhasedParams& p, uint64_t it0, uint64_t it1,
                                            double* part, uint8_t* smem, const SmemLayout& L,
                                            PhasedCta<N>& c) {
  constexpr int T1 = N / 16;
  constexpr int T = FPC * T1;
  constexpr int BPT = (N / 2) / T;
  static_assert(BPT * T == N / 2 && BPT >= 2, "bins per thread");

  float2* bufA = reinterpret_cast<float2*>(smem + L.off_a);
  float2* bufB = reinterpret_cast<float2*>(smem + L.off_b);
  uint8_t* stage = smem + L.off_stage;
  uint32_t* lut = reinterpret_cast<uint32_t*>(smem + L.off_lut);  // decode LUTs, then encode LUT
  float* lv = reinterpret_cast<float*>(smem + L.off_lv);          // [0,512) decode levels
  FrameInfo* finfo = reinterpret_cast<FrameInfo*>(smem + L.off_fi);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);
  int* flag = reinterpret_cast<int*>(smem + L.off_flag);
  // quantiser tables live in the extra tail of the layout
  float* ql = reinterpret_cast<float*>(smem + L.total);              // 256 levels
  uint32_t* elut = reinterpret_cast<uint32_t*>(smem + L.total + 1024);  // [4][256] encode LUT

  const int tid = threadIdx.x;
  const int g = tid / T1;
  const int t = tid % T1;
  const Twiddles<N>& tw = c.tw;
  const uint32_t seq0 = c.seq;

  const uint32_t bpf1 = p.st[0].bpf, bpf2 = p.st[1].bpf;
  constexpr uint32_t kRaw1 = FPC * kFiBytes;

  auto issue = [&](uint64_t it) {
    const int slot = (int)((seq0 + (uint32_t)(it - it0)) % kStages);
    const uint64_t f0 = it * FPC;
    const uint64_t nvalid = (p.nf - f0) < (uint64_t)FPC ? (p.nf - f0) : (uint64_t)FPC;
    const uint32_t bf = (uint32_t)(nvalid * kFiBytes);
    const uint32_t b1 = (uint32_t)(nvalid * bpf1), b2 = (uint32_t)(nvalid * bpf2);
    uint8_t* dst = stage + slot * L.stage_stride;
    mbar_expect_tx(&bars[slot], bf + b1 + b2);
    bulk_g2s(dst, p.finfo + f0, bf, &bars[slot]);
    bulk_g2s(dst + kRaw1, p.st[0].raw + f0 * bpf1, b1, &bars[slot]);
    bulk_g2s(dst + kRaw1 + FPC * bpf1, p.st[1].raw + f0 * bpf2, b2, &bars[slot]);
  };
  // The previous span, if any, is past its last reads of the staging ring and
  // the tables: the first frames' copies go out, the tables are built while
  // they are in flight.
  __syncthreads();
  if (tid == 0) {
    fence_proxy_async();
    for (uint64_t it = it0; it < it1 && it < it0 + kStages; ++it) issue(it);
  }
  for (int i = tid; i < 512; i += T) lv[i] = p.st[i >> 8].levels[i & 255] * p.st[i >> 8].scale;
  for (int s = 0; s < 2; ++s)
    if (p.st[s].shkind == SH_GENERIC)
      for (int i = tid; i < 1024; i += T) lut[s * 1024 + i] = p.st[s].shlut[i];
  for (int i = tid; i < 256; i += T) ql[i] = i < (int)p.nqlevels ? p.qlevels[i] : 0.f;
  for (int i = tid; i < 1024; i += T) elut[i] = p.enc_lut[i];
  __syncthreads();

  float acc[BPT + 1];
#pragma unroll
  for (int i = 0; i <= BPT; ++i) acc[i] = 0.f;
  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s;
  const int ov = a1e - a1s;
  const int sb = a2s - a1s;
  // undo the two-for-one factor 2 and the exact per-station level scaling
  const float u1 = 0.5f / p.st[0].scale, u2 = 0.5f / p.st[1].scale;
  bool first_flush = true;
  uint32_t since_flush = 0;
  const uint32_t spw = 32u / p.bits_out;           // samples per packed word
  const uint32_t wpf = (uint32_t)N / spw;          // words per output frame
  const uint32_t qmask = (p.bits_out >= 32) ? 0xFFFFFFFFu : ((1u << p.bits_out) - 1u);

  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i <= BPT; ++i) {
      if (i == BPT && tid != 0) continue;
      const int bin = (i < BPT) ? (tid + T * i) : N / 2;
      double* q = part + bin;
      *q = (first_flush ? 0.0 : *q) + (double)acc[i];
      acc[i] = 0.f;
    }
    first_flush = false;
    since_flush = 0;
  };

  bool ok = true;
  for (uint64_t it = it0; it < it1; ++it) {
    const uint32_t q_it = seq0 + (uint32_t)(it - it0);
    const int slot = (int)(q_it % kStages);
    const uint32_t parity = (q_it / kStages) & 1u;
    const uint64_t frame_local = it * FPC + g;
    const bool valid = frame_local < p.nf;

    if (!mbar_wait(&bars[slot], parity, kWaitPolls)) {
      atomicOr(flag, 1);
      atomicOr(p.err, ERR_WAIT_TIMEOUT);
    }
    uint8_t* st = stage + slot * L.stage_stride;
    uint32_t* w1 = reinterpret_cast<uint32_t*>(st + kRaw1);
    uint32_t* w2 = reinterpret_cast<uint32_t*>(st + kRaw1 + FPC * bpf1);
    preshuffle_slot(w1, FPC * bpf1 / 4, p.st[0].shkind, lut, w2, FPC * bpf2 / 4, p.st[1].shkind,
                    lut + 1024, tid, T);
    if (t == 0 && valid) finfo[g] = reinterpret_cast<const FrameInfo*>(st)[g];
    __syncthreads();
    if (*flag) {
      ok = false;
      break;
    }
    const int s1 = valid ? finfo[g].s1 : 0;
    const int s2 = valid ? finfo[g].s2 : 0;
    const PackedStation pa{w1 + g * (bpf1 / 4), lv, (uint32_t)p.st[0].bits,
                           (1u << p.st[0].bits) - 1u, p.st[0].lsb ? 1 : 0, s1};
    const PackedStation pb{w2 + g * (bpf2 / 4), lv + 256, (uint32_t)p.st[1].bits,
                           (1u << p.st[1].bits) - 1u, p.st[1].lsb ? 1 : 0, s2};

    float2* za = bufA + g * Geom<N>::CSTRIDE;
    float2* zb = bufB + g * Geom<N>::CSTRIDE;
    first_pass_packed<N>(pa, pb, za, t);
    float2* Z0 = fft_rest<N>(za, zb, t, tw);
    if (tid == 0 && it + kStages < it1) {
      fence_proxy_async();
      issue(it + kStages);
    }
    const bool fin_b = Z0 != za;
    __syncthreads();

    // ---- per-bin synthesis over every valid frame of the iteration; the
    // inverse-FFT input planes go to the buffer that does not hold Z
#pragma unroll 1
    for (int f = 0; f < FPC; ++f) {
      if (it * FPC + f >= p.nf) break;
      const float2* Z = (fin_b ? bufB : bufA) + f * Geom<N>::CSTRIDE;
      float* y1 = reinterpret_cast<float*>(fin_b ? bufA : bufB) + f * 2 * Geom<N>::FSTRIDE;
      float* y2 = y1 + Geom<N>::FSTRIDE;
      const FrameInfo& F = finfo[f];
      // spectrum of station s at its own bin k: unscaled, rotated by the
      // station's fractional delay, Nyquist imaginary part zeroed, times fr_lo
      auto station_bin = [&](int s, int k) -> float2 {
        const float2 a = Z[k], b = Z[(N - k) & (N - 1)];
        float2 v = s == 0 ? make_float2(u1 * (a.x + b.x), u1 * (a.y - b.y))
                          : make_float2(u2 * (a.y + b.y), u2 * (b.x - a.x));
        float sn, cs;
        __sincosf((float)k * (s == 0 ? F.st1 : F.st2), &sn, &cs);
        v = cmul(v, make_float2(cs, sn));
        if (k == N / 2) v.y = 0.f;
        return cmul(v, s == 0 ? F.fr_lo1 : F.fr_lo2);
      };
      auto bin_cb = [&](int k) -> float2 {
        float2 a1 = make_float2(0.f, 0.f), a2 = make_float2(0.f, 0.f);
        if (p.grid == 0) {
          a1 = station_bin(0, k);
          if (k >= a1s && k < a1e) a2 = station_bin(1, k + sb);
        } else {
          a2 = station_bin(1, k);
          if (k >= a2s && k < a2s + ov) a1 = station_bin(0, k - sb);
        }
        return make_float2(a1.x * p.w1 + a2.x * p.w2, a1.y * p.w1 + a2.y * p.w2);
      };
      auto emit = [&](int k, float2 cb) {
        // Hermitian extension of conj(cb) as planes for the forward FFT
        if (k == 0 || k == N / 2) cb.y = 0.f;
        y1[fpad(k)] = cb.x;
        y2[fpad(k)] = -cb.y;
        if (k != 0 && k != N / 2) {
          y1[fpad(N - k)] = cb.x;
          y2[fpad(N - k)] = cb.y;
        }
      };
#pragma unroll
      for (int i = 0; i < BPT; ++i) {
        const int k = tid + T * i;
        const float2 cb = bin_cb(k);
        acc[i] += cnorm2(cb);
        if (p.want_raw) emit(k, cb);
      }
      if (tid == 0) {
        const float2 cb = bin_cb(N / 2);
        acc[BPT] += cnorm2(cb);
        if (p.want_raw) emit(N / 2, cb);
      }
    }
    if (++since_flush >= p.flush_every) flush();

    if (p.want_raw) {
      __syncthreads();
      // inverse real FFT of frame slot g: forward FFT of conj(C), real part / N
      float* y1 = reinterpret_cast<float*>(fin_b ? bufA : bufB) + g * 2 * Geom<N>::FSTRIDE;
      float* y2 = y1 + Geom<N>::FSTRIDE;
      float2* qa = (fin_b ? bufB : bufA) + g * Geom<N>::CSTRIDE;  // free: Z consumed
      float2* qb = (fin_b ? bufA : bufB) + g * Geom<N>::CSTRIDE;
      first_pass<N>(y1, y2, 0, 0, qa, t);
      float2* Y = fft_rest<N>(qa, qb, t, tw);
      __syncthreads();
      if (valid) {
        const float inv_n = 1.0f / (float)N;
        uint8_t* out = p.raw_out + frame_local * p.bpf_out;
        // Consecutive lanes pack consecutive words, spw samples apart: each
        // lane starts its word at a different sample (rot) so that the 16
        // lanes of a half-warp read 16 different bank pairs of Y at every
        // step instead of one.
        const uint32_t lane = (uint32_t)t & 31u;
        const uint32_t rot = spw >= 16 ? lane : lane / (16u / spw);
        for (uint32_t w = (uint32_t)t; w < wpf; w += T1) {
          uint32_t word = 0;
          for (uint32_t i = 0; i < spw; ++i) {
            const uint32_t ii = (i + rot) & (spw - 1u);
            const uint32_t n = w * spw + ii;
            float x = Y[n].x * inv_n;
            if (p.out_lsb && (n & 1u)) x = -x;
            word |= (nearest_level(x, ql, (int)p.nqlevels, p.qmonotonic) & qmask)
                    << (ii * p.bits_out);
          }
          const uint32_t sw = elut[word & 255u] | elut[256 + ((word >> 8) & 255u)] |
                              elut[512 + ((word >> 16) & 255u)] | elut[768 + (word >> 24)];
          reinterpret_cast<uint32_t*>(out)[w] = sw;
        }
      }
    }
    __syncthreads();
  }
  if (since_flush > 0 || first_flush) flush();
  c.seq = seq0 + (uint32_t)(it1 - it0);
  return ok;
}

template <int N, int FPC>
__global__ void __launch_bounds__(FPC * N / 16, (N >= 8192 ? 1 : 2))
phased_kernel(const __grid_constant__ PhasedParams p) {
  constexpr int H = N / 2 + 1;
  extern __shared__ __align__(128) uint8_t smem[];
  const SmemLayout L = smem_layout<N, FPC>(p.stage_bytes);
  PhasedCta<N> c;
  phased_cta_init<N, FPC>(smem, L, c);
  const uint64_t iters = (p.nf + FPC - 1) / FPC;
  const uint64_t it0 = (blockIdx.x * iters) / gridDim.x;
  const uint64_t it1 = ((blockIdx.x + 1) * iters) / gridDim.x;
  phased_span<N, FPC>(p, it0, it1, p.partials + (size_t)blockIdx.x * H, smem, L, c);
  phased_cta_drain(smem, L);
}

// Batched: a persistent grid takes the items of batch group `grp` by ticket;
// an item is a frame range of one scan's phased sector (its own tables, frame
// records, raw words and .raw output) with its own H partials.  The layout is
// sized for 8-bit stations, so one launch serves every bit depth, and every
// frame is computed exactly as by phased_kernel.
template <int N, int FPC>
__global__ void __launch_bounds__(FPC * N / 16, (N >= 8192 ? 1 : 2))
phased_batch_kernel(const BatchArgs a, int grp) {
  extern __shared__ __align__(128) uint8_t smem[];
  const SmemLayout L = smem_layout<N, FPC>(2u * FPC * N);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(smem + L.off_flag + 4);
  PhasedCta<N> c;
  phased_cta_init<N, FPC>(smem, L, c);
  const uint32_t n_items = a.hdr->nitems[grp];
  const BatchItem* items = a.hdr->items + a.hdr->item0[grp];
  const BatchScan* scans = a.hdr->scans;
  for (;;) {
    if (threadIdx.x == 0) *ticket = atomicAdd(&a.hdr->ticket[grp], 1u);
    __syncthreads();
    const uint32_t k = *ticket;  // phased_span opens with a barrier before the next write
    if (k >= n_items) break;
    const BatchItem w = items[k];
    const uint64_t it0 = w.f0 / FPC, it1 = (w.f1 + FPC - 1) / FPC;
    if (!phased_span<N, FPC>(scans[w.scan].pp, it0, it1, a.partials + w.part, smem, L, c)) break;
  }
  phased_cta_drain(smem, L);
}

// Fixed-order sum of the per-CTA phased partials into acc[4H, 5H).
// (32 bins per block; each of 8 warps sums a contiguous eighth of the slots in
// slot order, the warp sums are added in warp order: deterministic.)
__global__ void __launch_bounds__(256) reduce_phased_kernel(const double* __restrict__ part,
                                                            int nblk, int h,
                                                            double* __restrict__ out) {
  __shared__ double sm[8][32];
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const int k = blockIdx.x * 32 + lane;
  const int b0 = (nblk * grp) / 8, b1 = (nblk * (grp + 1)) / 8;
  double s = 0.0;
  if (k < h)
    for (int b = b0; b < b1; ++b) s += part[(size_t)b * h + k];
  sm[grp][lane] = s;
  __syncthreads();
  if (grp != 0 || k >= h) return;
  double t = 0.0;
#pragma unroll
  for (int g = 0; g < 8; ++g) t += sm[g][lane];
  out[4 * h + k] = t;
}

template <int N, int FPC>
static cudaError_t launch_phased_one(const PhasedParams& p, int grid, cudaStream_t stream) {
  const uint32_t smem = smem_layout<N, FPC>(p.stage_bytes).total + 1024 + 4096;
  auto kern = phased_kernel<N, FPC>;
  // the limit is shared by every host thread: always the largest layout
  // (8-bit stations), never lowered under a concurrent launch
  cudaError_t e = cudaFuncSetAttribute(
      kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
      (int)(smem_layout<N, FPC>(2u * FPC * N).total + 1024 + 4096));
  if (e != cudaSuccess) return e;
  kern<<<grid, FPC * N / 16, smem, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_phased(uint32_t n, const PhasedParams& p, int grid, cudaStream_t s) {
  switch (n) {
    case 1024: return launch_phased_one<1024, 4>(p, grid, s);
    case 2048: return launch_phased_one<2048, 2>(p, grid, s);
    case 4096: return launch_phased_one<4096, 1>(p, grid, s);
    case 8192: return launch_phased_one<8192, 1>(p, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

namespace {
template <int N, int FPC>
uint32_t phased_batch_smem() {
  return smem_layout<N, FPC>(2u * FPC * N).total + 1024 + 4096;
}
}  // namespace

// Batch groups of the phased kernels: FFT 1024 / 2048 / 4096 / 8192 with the
// single-scan kernels' frames per CTA iteration (4 / 2 / 1 / 1); FFT 16384
// is the two-row kernel's group (phased_pair.cu).
cudaError_t phased_batch_prepare(uint32_t n) {
  switch (n) {
    case 16384: return phased_pair_batch_prepare();
    case 1024: return cudaFuncSetAttribute(phased_batch_kernel<1024, 4>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)phased_batch_smem<1024, 4>());
    case 2048: return cudaFuncSetAttribute(phased_batch_kernel<2048, 2>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)phased_batch_smem<2048, 2>());
    case 4096: return cudaFuncSetAttribute(phased_batch_kernel<4096, 1>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)phased_batch_smem<4096, 1>());
    case 8192: return cudaFuncSetAttribute(phased_batch_kernel<8192, 1>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)phased_batch_smem<8192, 1>());
    default: return cudaErrorInvalidValue;
  }
}

int phased_batch_ctas_per_sm(uint32_t n) {
  int nb = 0;
  cudaError_t e = cudaErrorInvalidValue;
  switch (n) {
    case 1024: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, phased_batch_kernel<1024, 4>,
                                                                 256, phased_batch_smem<1024, 4>());
      break;
    case 2048: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, phased_batch_kernel<2048, 2>,
                                                                 256, phased_batch_smem<2048, 2>());
      break;
    case 4096: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, phased_batch_kernel<4096, 1>,
                                                                 256, phased_batch_smem<4096, 1>());
      break;
    case 8192: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, phased_batch_kernel<8192, 1>,
                                                                 512, phased_batch_smem<8192, 1>());
      break;
    case 16384: return phased_pair_batch_ctas_per_sm();
    default: break;
  }
  return e == cudaSuccess ? nb : 0;
}

int phased_frames_per_cta_iter(uint32_t n) { return n == 1024 ? 4 : (n == 2048 ? 2 : 1); }

cudaError_t launch_phased_batch(uint32_t n, const BatchArgs& a, int grp, int grid, cudaStream_t s) {
  switch (n) {
    case 1024: phased_batch_kernel<1024, 4><<<grid, 256, phased_batch_smem<1024, 4>(), s>>>(a, grp); break;
    case 2048: phased_batch_kernel<2048, 2><<<grid, 256, phased_batch_smem<2048, 2>(), s>>>(a, grp); break;
    case 4096: phased_batch_kernel<4096, 1><<<grid, 256, phased_batch_smem<4096, 1>(), s>>>(a, grp); break;
    case 8192: phased_batch_kernel<8192, 1><<<grid, 512, phased_batch_smem<8192, 1>(), s>>>(a, grp); break;
    case 16384: return launch_phased_pair_batch(a, grp, grid, s);
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_reduce_phased(const double* part, int nblk, int h, double* out, cudaStream_t s) {
  reduce_phased_kernel<<<(h + 31) / 32, 256, 0, s>>>(part, nblk, h, out);
  return cudaGetLastError();
}

}  // namespace fxc
