// phased_pair.cu — phased-array synthesis for FFT 16384 (yi-phasedarray,
// src/main.rs:2222-2412), 1- to 8-bit stations: one CTA per frame pair, both
// 8192-point rows of the frame in its shared memory.
//
// Per frame pair (the contract of phased_kernel, whose N <= 8192 frame loop
// holds a frame in one FFT):
//   1. forward: each row of the radix-2 decimation in frequency,
//      y_q[m] = W_N^(m q) (z[m] + (-1)^q z[m + M]), z = x1 + i x2, is decoded
//      straight from the staged words by the FFT-16384 fold kernel's decode
//      (fold_decode.cuh) into its first radix-16 pass; the row FFTs run in
//      shared memory, the trailing radix-2 pass in place, so bin 2 j + q of
//      the frame is Z_q[j];
//   2. per bin: both stations' spectra from the shared FFT (two-for-one),
//      each rotated by its fractional delay with the Nyquist imaginary part
//      zeroed and multiplied by its fringe phasor, band-aligned onto the
//      output grid and summed with the weights (src/main.rs:2264-2280,
//      src/utils.rs:69-124); |cb|^2 accumulates in f32 registers (f64
//      flushes every flush_every frames);
//   3. for the .raw product: cb[0].im = cb[N/2].im = 0, the inverse real FFT
//      as the forward FFT of the Hermitian-extended conj(cb) scaled by 1/N
//      (src/utils.rs:60-66) through the same two-row decomposition (x[m] and
//      x[m + M] gathered from cb), odd samples negated when both inputs are
//      LSB, nearest-level re-quantisation with ant1's levels and packing with
//      ant1's shuffle (src/utils.rs:378-410) of whole words from both rows.
// Three padded row buffers.  With 1- and 2-bit stations a staging slot of its
// own follows them and the next frame's words are copied while the frame is
// computed; 4- and 8-bit stations (twice or four times the words) stage into
// the third row buffer once the frame is done with it (during the
// re-quantiser, or after the frame when no .raw is written).
#include <cuda_runtime.h>
#include <stdint.h>

#include "decode_tables.cuh"
#include "fold_decode.cuh"
#include "row_fft.cuh"
#include "fxc_device.cuh"
#include "fxc_kernels.h"

namespace fxc {
namespace {

constexpr int kM = fold::kN;   // row length
constexpr int kT = kM / 16;    // threads per CTA
constexpr int kN2 = 2 * kM;    // frame length
constexpr int kH2 = kN2 / 2 + 1;
constexpr int kJ = kM / 2 / kT;  // bin pairs (rows 0 and 1) per thread

// Shared memory (bytes): decode tables [0, 4608) (levels, rotate amounts); the
// gap [4352, 4608) holds the frame record, the staging mbarrier, the error
// flag and the batch ticket; then the three row buffers.  Narrow stations
// (1- and 2-bit, output <= 2 bits): need no byte LUTs, so [4608, 12800) holds
// ant1's output encode LUT, the output levels sit in the gap, and one staging
// slot [FrameInfo (128 B)][station 1][station 2] follows the buffers.  Wide
// stations: [4608, 12800) holds the byte LUTs of 4- and 8-bit generic
// shuffles, the encode LUT and up to 256 output levels follow the buffers, and
// the staging slot is a row buffer.
constexpr uint32_t kPpFi = 4352, kPpBar = 4400, kPpFlag = 4408, kPpTicket = 4412;
constexpr uint32_t kPpQl = 4416;  // 16 levels max
constexpr uint32_t kPpEnc = kTabLut;  // [4][256] u32
constexpr uint32_t kPpBuf = (uint32_t)Geom<kM>::CSTRIDE * (uint32_t)sizeof(float2);
constexpr uint32_t kPpB0 = kTabEnd, kPpB1 = kPpB0 + kPpBuf, kPpB2 = kPpB1 + kPpBuf;
constexpr uint32_t kPpStage = kPpB2 + kPpBuf;
constexpr uint32_t kPpMaxSmem = 232448;  // 227 KB per CTA on sm_100
static_assert(kPpFi + kFiBytes <= kPpBar && kPpQl + 16 * 4 <= kTabLut, "records fit the gap");
static_assert(kPpStage % 128 == 0, "alignment");

__host__ __device__ constexpr uint32_t pp_smem_bytes(uint32_t bpf1, uint32_t bpf2) {
  return kPpStage + ((128u + bpf1 + bpf2 + 127u) & ~127u);
}
static_assert(pp_smem_bytes(kN2 / 4, kN2 / 4) <= kPpMaxSmem, "2-bit stations fit");
constexpr uint32_t kPpWideEnc = kPpStage, kPpWideQl = kPpStage + 4096;
constexpr uint32_t kPpWideSmem = kPpWideQl + 256 * 4;
static_assert(kPpWideSmem <= pp_smem_bytes(kN2 / 4, kN2 / 4), "one batch layout serves both");
static_assert(128u + 2u * kN2 <= kPpBuf, "8-bit stations' words fit a row buffer");

// Narrow stations take the separate staging slot (and the encode LUT and
// output levels at their narrow places); any wider station or output selects
// the wide layout.
__host__ __device__ inline bool pp_wide(uint32_t bits1, uint32_t bits2, uint32_t bits_out) {
  return bits1 > 2 || bits2 > 2 || bits_out > 2;
}

using rows::first_pass_regs;
using rows::row1_twiddle;
using rows::row_radix2;
using rows::fold_lower;
using rows::fold_mirror;
using rows::fold_twiddles;

// Per-CTA state that does not depend on the scan: the twiddle chains and
// bases, and the staging mbarrier's next phase (a persistent CTA runs spans
// of several scans back to back on one mbarrier).
struct PpCta {
  Twiddles<kM> tw;
  float2 wb1, dtw0, dtw1;
  uint32_t phase;
  bool stopped;
};

__device__ __forceinline__ void pp_cta_init(uint8_t* smem, PpCta& c) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(reinterpret_cast<uint64_t*>(smem + kPpBar), 1);
    *reinterpret_cast<int*>(smem + kPpFlag) = 0;
    fence_proxy_async();
  }
  c.tw.init(tid);
  c.wb1 = rows::fold_base1(tid);  // W_M^(t+1)
  // row 1's DIF twiddle bases W_N^t, W_N^(t + T), correctly rounded from FP64
  double sn, cs;
  sincospi(-2.0 * (double)tid / (double)kN2, &sn, &cs);
  c.dtw0 = make_float2((float)cs, (float)sn);
  sincospi(-2.0 * (double)(tid + kT) / (double)kN2, &sn, &cs);
  c.dtw1 = make_float2((float)cs, (float)sn);
  c.phase = 0;
  c.stopped = false;
}

// Never leave a bulk copy in flight into a finished CTA's shared memory: after
// a wait gave up, wait (bounded) once more for the phase that did not complete.
__device__ __forceinline__ void pp_cta_drain(uint8_t* smem, const PpCta& c) {
  if (c.stopped && threadIdx.x == 0)
    mbar_wait(reinterpret_cast<uint64_t*>(smem + kPpBar), c.phase ^ 1u, kWaitPolls);
}

// Frame pairs [it0, it1) of the sector described by p, phased power summed
// into the f64 partials at part ([H]) and .raw frames written when asked.
// Opens with a CTA barrier (the previous span, if any, is past its last use
// of the tables, the buffers and the staging slot).  Returns false when a
// bounded wait gave up (the CTA must stop).
//
// Buffers P, Q, S: row 0 forward into P, row 1 into Q, the secondary
// station's spectrum by bin into S, cb into P; the inverse row 0 into Q, row
// 1 into S (into P, in place of cb, when WIDE), the scratch of each FFT a free
// buffer.  WIDE: the frame's words arrive in S, the next frame's go there once
// the inverse is done with it.
template <bool WIDE>
__device__ __forceinline__ bool pp_span(const PhasedParams& p, uint64_t it0, uint64_t it1,
                                        double* part, uint8_t* smem, PpCta& c) {
  const int tid = threadIdx.x;
  FrameInfo* finfo = reinterpret_cast<FrameInfo*>(smem + kPpFi);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kPpBar);
  int* flag = reinterpret_cast<int*>(smem + kPpFlag);
  float* ql = reinterpret_cast<float*>(smem + (WIDE ? kPpWideQl : kPpQl));
  uint32_t* elut = reinterpret_cast<uint32_t*>(smem + (WIDE ? kPpWideEnc : kPpEnc));
  const uint32_t* lut = reinterpret_cast<const uint32_t*>(smem + kTabLut);
  const uint32_t* pos = reinterpret_cast<const uint32_t*>(smem + kTabPos);
  float2* P = reinterpret_cast<float2*>(smem + kPpB0);
  float2* Q = reinterpret_cast<float2*>(smem + kPpB1);
  float2* S = reinterpret_cast<float2*>(smem + kPpB2);

  const StationParams& s1 = p.st[0];
  const StationParams& s2 = p.st[1];
  const uint32_t bpf1 = s1.bpf, bpf2 = s2.bpf;
  // 4- and 8-bit stations with a non-identity shuffle: words rewritten in place
  const bool pre1 = WIDE && s1.bits > 2 && s1.shkind != SH_IDENTITY;
  const bool pre2 = WIDE && s2.bits > 2 && s2.shkind != SH_IDENTITY;

  auto issue = [&](uint64_t it, uint8_t* stage) {
    mbar_expect_tx(bar, kFiBytes + bpf1 + bpf2);
    bulk_g2s(stage, p.finfo + it, kFiBytes, bar);
    bulk_g2s(stage + 128, s1.raw + it * bpf1, bpf1, bar);
    bulk_g2s(stage + 128 + bpf1, s2.raw + it * bpf2, bpf2, bar);
  };
  uint8_t* stage = WIDE ? reinterpret_cast<uint8_t*>(S) : smem + kPpStage;
  __syncthreads();
  if (tid == 0 && it0 < it1) {
    fence_proxy_async();
    issue(it0, stage);
  }
  build_decode_tables(s1, s2, pre1, pre2, smem, tid, kT);
  const int nql = WIDE ? 256 : 16;
  for (int i = tid; i < nql; i += kT) ql[i] = i < (int)p.nqlevels ? p.qlevels[i] : 0.f;
  for (int i = tid; i < 1024; i += kT) elut[i] = p.enc_lut[i];
  const bool split1 = split_2bit(s1), split2 = split_2bit(s2);
  const Twiddles<kM>& tw = c.tw;
  const float2 wb1 = c.wb1, dtw0 = c.dtw0, dtw1 = c.dtw1;
  __syncthreads();

  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s;
  const int ov = a1e - a1s, sb = a2s - a1s;
  const bool g0 = p.grid == 0;
  // output bin b: primary (on the output grid) at b, secondary at b + qoff
  const int ovs = g0 ? a1s : a2s;
  const int qoff = g0 ? sb : -sb;
  // undo the two-for-one factor 2 and the exact per-station level scaling
  const float u1 = 0.5f / s1.scale, u2 = 0.5f / s2.scale;
  const int lsb1 = s1.lsb ? 1 : 0, lsb2 = s2.lsb ? 1 : 0;
  const bool half = tid == 0;  // bin N/2
  const uint32_t spw = 32u / p.bits_out;
  const uint32_t wpf = (uint32_t)kN2 / spw;
  const uint32_t qmask = (1u << p.bits_out) - 1u;
  const float inv_n = 1.0f / (float)kN2;

  // acc[2 i + q]: bin 2 (t + T i) + q; acc[2 kJ]: bin N/2
  float acc[2 * kJ + 1];
#pragma unroll
  for (int i = 0; i <= 2 * kJ; ++i) acc[i] = 0.f;
  bool first_flush = true;
  uint32_t since_flush = 0;
  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i <= 2 * kJ; ++i) {
      if (i == 2 * kJ && !half) continue;
      const int bin = i == 2 * kJ ? kN2 / 2 : 2 * (tid + kT * (i >> 1)) + (i & 1);
      double* d = part + bin;
      *d = (first_flush ? 0.0 : *d) + (double)acc[i];
      acc[i] = 0.f;
    }
    first_flush = false;
    since_flush = 0;
  };

  uint32_t phase = c.phase;
  bool ok = true;
  for (uint64_t it = it0; it < it1; ++it) {
    if (!mbar_wait(bar, phase, kWaitPolls)) {
      atomicOr(flag, 1);
      atomicOr(p.err, ERR_WAIT_TIMEOUT);
    }
    phase ^= 1u;
    __syncthreads();  // every thread past its wait, the flag visible
    if (*flag) {
      ok = false;
      break;
    }
    uint32_t* w1 = reinterpret_cast<uint32_t*>(stage + 128);
    uint32_t* w2 = reinterpret_cast<uint32_t*>(stage + 128 + bpf1);
    const FrameInfo* fs = reinterpret_cast<const FrameInfo*>(stage);
    const int sh1 = fs->s1, sh2 = fs->s2;
    if (tid == 0) *finfo = *fs;  // before the slot is refilled or reused
    if (pre1 || pre2) {
      preshuffle_slot(w1, bpf1 / 4, pre1 ? s1.shkind : SH_IDENTITY, lut, w2, bpf2 / 4,
                      pre2 ? s2.shkind : SH_IDENTITY, lut + 1024, tid, kT);
      __syncthreads();
    }
    const float sg = (it & 1u) ? -1.0f : 1.0f;  // station 2 enters odd frames negated

    // ---- 1. forward: rows 0 and 1 of the radix-2 DIF, decoded into their first pass
    {
      const int m1 = tid - sh1, m2 = tid - sh2;
      const int c1 = m1 & ((32 / s1.bits) - 1), c2 = m2 & ((32 / s2.bits) - 1);
      const uint32_t tb1 = (uint32_t)((m1 & lsb1) << (s1.bits + 2));
      const uint32_t tb2 = 2048u + (uint32_t)((((uint32_t)m2 & (uint32_t)lsb2) ^ (uint32_t)(it & 1u))
                                              << (s2.bits + 2));
      for (int q = 0; q < 2; ++q) {
        float2 v[16];
        fold::fold_station<false, 2>(s1.bits, split1, w1, smem, sh1, pos[c1], tb1, v, tid, q == 1);
        fold::fold_station<true, 2>(s2.bits, split2, w2, smem, sh2, pos[32 + c2], tb2, v, tid,
                                    q == 1);
        if (q == 1) row1_twiddle(v, dtw0, dtw1);
        // WIDE: row 0's FFT took Q as its scratch (S holds the words)
        if (WIDE && q == 1) __syncthreads();
        first_pass_regs(v, q == 0 ? P : Q, tid);
        if (q == 0) fft_rest<kM, true>(P, WIDE ? Q : S, tid, tw);  // row 0's spectrum in P
      }
    }
    fft_rest<kM, true>(Q, S, tid, tw);  // row 1's spectrum in Q
    // the staged words are consumed (fft_rest opened with a barrier): refill
    if (!WIDE && tid == 0 && it + 1 < it1) {
      fence_proxy_async();
      issue(it + 1, stage);
    }
    __syncthreads();

    // ---- 2. per bin: both stations rotated; the secondary one into S by bin
    const FrameInfo& F = *finfo;
    auto station = [&](float2 u, float2 w, int k, int s) -> float2 {
      // spectrum of station s at its own bin k: unscaled, rotated by the
      // station's fractional delay, Nyquist imaginary part zeroed, times fr_lo
      float2 v = s == 0 ? make_float2(u1 * (u.x + w.x), u1 * (u.y - w.y))
                        : make_float2(sg * u2 * (u.y + w.y), sg * u2 * (w.x - u.x));
      float sn, cs;
      __sincosf((float)k * (s == 0 ? F.st1 : F.st2), &sn, &cs);
      v = cmul(v, make_float2(cs, sn));
      if (k == kN2 / 2) v.y = 0.f;
      return cmul(v, s == 0 ? F.fr_lo1 : F.fr_lo2);
    };
    const int sp = g0 ? 0 : 1;  // the station on the output grid
    float2 prim[2 * kJ + 1];
#pragma unroll
    for (int i2 = 0; i2 < kJ; ++i2) {
      const int j = tid + kT * i2;
      float2 wj, wj1;
      fold_twiddles(tw, wb1, i2, wj, wj1);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        // the rows' trailing radix-2 pass folded in: Z_q[j] and Z[N - k],
        // which is row 1's index M - 1 - j or row 0's index M - j
        const int k = 2 * j + q;
        const float2* Y = q ? Q : P;
        const float2 u = fold_lower(Y, j, wj);
        const float2 w = fold_mirror(Y, j, q == 0, wj, wj1);
        prim[2 * i2 + q] = station(u, w, k, sp);
        S[k] = station(u, w, k, 1 - sp);
      }
    }
    prim[2 * kJ] = make_float2(0.f, 0.f);
    if (half) {  // Z[N/2] = row 0's index M/2 (Y[0] - Y[M/2]) pairs with itself
      const float2 u = csub(P[0], P[kM / 2]);
      prim[2 * kJ] = station(u, u, kN2 / 2, sp);
      S[kN2 / 2] = station(u, u, kN2 / 2, 1 - sp);
    }
    __syncthreads();
    // ---- band alignment and the weighted sum; cb by bin into P
    auto combine = [&](int b, float2 pv) -> float2 {
      float2 sv = make_float2(0.f, 0.f);
      if ((unsigned)(b - ovs) < (unsigned)ov) sv = S[b + qoff];
      // cb = w1 a1 + w2 a2 with a1 / a2 the station-1 / station-2 terms
      const float2 a1 = g0 ? pv : sv, a2 = g0 ? sv : pv;
      return make_float2(a1.x * p.w1 + a2.x * p.w2, a1.y * p.w1 + a2.y * p.w2);
    };
#pragma unroll
    for (int i = 0; i < 2 * kJ; ++i) {
      const int b = 2 * (tid + kT * (i >> 1)) + (i & 1);
      float2 cb = combine(b, prim[i]);
      acc[i] += cnorm2(cb);
      if (b == 0) cb.y = 0.f;
      P[b] = cb;
    }
    if (half) {
      float2 cb = combine(kN2 / 2, prim[2 * kJ]);
      acc[2 * kJ] += cnorm2(cb);
      cb.y = 0.f;
      P[kN2 / 2] = cb;
    }
    if (++since_flush >= p.flush_every) flush();

    if (p.want_raw) {
      __syncthreads();
      // ---- 3. inverse: x[n] = conj(cb[n]) (n <= N/2), cb[N - n] (n > N/2);
      // rows x[m] +- x[m + M] = conj(cb[m]) +- cb[M - m], m = t + T r
      for (int q = 0; q < 2; ++q) {
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int m = tid + kT * r;
          const float2 lo = P[m], hi = P[kM - m];
          v[r] = q == 0 ? make_float2(lo.x + hi.x, hi.y - lo.y) : make_float2(lo.x - hi.x, -lo.y - hi.y);
        }
        if (q == 1) row1_twiddle(v, dtw0, dtw1);
        if (q == 0) {
          first_pass_regs(v, Q, tid);
          fft_rest<kM, true>(Q, S, tid, tw);  // X[2 k] (pre radix-2) in Q
          __syncthreads();
          row_radix2(Q, tid, tw);
        } else if (!WIDE) {
          first_pass_regs(v, S, tid);
          fft_rest<kM, true>(S, P, tid, tw);  // X[2 k + 1] in S (cb consumed)
          __syncthreads();
          row_radix2(S, tid, tw);
        } else {
          __syncthreads();  // every thread has read its cb values
          first_pass_regs(v, P, tid);
          fft_rest<kM, true>(P, S, tid, tw);  // X[2 k + 1] in P
          __syncthreads();
          // S is free until the next frame's decode: its words go there
          if (tid == 0 && it + 1 < it1) {
            fence_proxy_async();
            issue(it + 1, stage);
          }
          row_radix2(P, tid, tw);
        }
      }
      __syncthreads();
      // ---- re-quantise and pack: sample n is row n & 1, index n >> 1.  Each
      // lane starts its word at a different sample so that a warp's loads
      // spread over the banks.
      uint8_t* out = p.raw_out + it * p.bpf_out;
      const uint32_t lane = (uint32_t)tid & 31u;
      const uint32_t rot = spw >= 16 ? lane : lane / (16u / spw);
      for (uint32_t wdx = (uint32_t)tid; wdx < wpf; wdx += kT) {
        uint32_t word = 0;
        for (uint32_t i = 0; i < spw; ++i) {
          const uint32_t ii = (i + rot) & (spw - 1u);
          const uint32_t n = wdx * spw + ii;
          float x = ((n & 1u) ? (WIDE ? P : S) : Q)[n >> 1].x * inv_n;
          if (p.out_lsb && (n & 1u)) x = -x;
          word |= (nearest_level(x, ql, (int)p.nqlevels, p.qmonotonic) & qmask) << (ii * p.bits_out);
        }
        reinterpret_cast<uint32_t*>(out)[wdx] =
            elut[word & 255u] | elut[256 + ((word >> 8) & 255u)] |
            elut[512 + ((word >> 16) & 255u)] | elut[768 + (word >> 24)];
      }
    }
    __syncthreads();  // the buffers are free for the next frame
    if (WIDE && !p.want_raw && tid == 0 && it + 1 < it1) {
      fence_proxy_async();
      issue(it + 1, stage);
    }
  }
  if (since_flush > 0 || first_flush) flush();
  c.phase = phase;
  c.stopped = !ok;
  return ok;
}

template <bool WIDE>
__global__ void __launch_bounds__(kT, 1) phased_pair_kernel(const __grid_constant__ PhasedParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  PpCta c;
  pp_cta_init(smem, c);
  const uint64_t it0 = ((uint64_t)blockIdx.x * p.nf) / gridDim.x;
  const uint64_t it1 = ((uint64_t)(blockIdx.x + 1) * p.nf) / gridDim.x;
  pp_span<WIDE>(p, it0, it1, p.partials + (size_t)blockIdx.x * kH2, smem, c);
  pp_cta_drain(smem, c);
}

// Batched: a persistent grid takes the items of batch group `grp` by ticket;
// an item is a frame range of one scan's phased FFT-16384 sector (its own
// tables, frame records, raw words and .raw output) with its own H partials.
// Shared memory is sized for the larger (narrow) layout, so one launch serves
// every bit depth, and every frame is computed exactly as by phased_pair_kernel.
__global__ void __launch_bounds__(kT, 1) phased_pair_batch_kernel(const BatchArgs a, int grp) {
  extern __shared__ __align__(128) uint8_t smem[];
  uint32_t* ticket = reinterpret_cast<uint32_t*>(smem + kPpTicket);
  PpCta c;
  pp_cta_init(smem, c);
  const uint32_t n_items = a.hdr->nitems[grp];
  const BatchItem* items = a.hdr->items + a.hdr->item0[grp];
  const BatchScan* scans = a.hdr->scans;
  for (;;) {
    if (threadIdx.x == 0) *ticket = atomicAdd(&a.hdr->ticket[grp], 1u);
    __syncthreads();
    const uint32_t k = *ticket;  // pp_span opens with a barrier before the next write
    if (k >= n_items) break;
    const BatchItem w = items[k];
    const PhasedParams& pp = scans[w.scan].pp;
    const bool ok = pp_wide(pp.st[0].bits, pp.st[1].bits, pp.bits_out)
                        ? pp_span<true>(pp, w.f0, w.f1, a.partials + w.part, smem, c)
                        : pp_span<false>(pp, w.f0, w.f1, a.partials + w.part, smem, c);
    if (!ok) break;
  }
  pp_cta_drain(smem, c);
}

}  // namespace

bool phased_pair_supported(uint32_t n, const PhasedParams& p) {
  return n == (uint32_t)kN2 && p.nqlevels <= 256;
}

int phased_pair_grid(int sms, uint64_t nf) {
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(nf, (uint64_t)sms));
}

cudaError_t launch_phased_pair(const PhasedParams& p, int grid, cudaStream_t s) {
  const bool wide = pp_wide(p.st[0].bits, p.st[1].bits, p.bits_out);
  auto* kern = wide ? phased_pair_kernel<true> : phased_pair_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kPpMaxSmem);
  if (e != cudaSuccess) return e;
  kern<<<grid, kT, wide ? kPpWideSmem : pp_smem_bytes(p.st[0].bpf, p.st[1].bpf), s>>>(p);
  return cudaGetLastError();
}

// The batch group's kernel, its shared memory sized for the narrow layout with
// 2-bit stations (the larger of the two layouts).
cudaError_t phased_pair_batch_prepare() {
  return cudaFuncSetAttribute(phased_pair_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)pp_smem_bytes(kN2 / 4, kN2 / 4));
}

int phased_pair_batch_ctas_per_sm() {
  int nb = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &nb, phased_pair_batch_kernel, kT, pp_smem_bytes(kN2 / 4, kN2 / 4));
  return e == cudaSuccess ? nb : 0;
}

cudaError_t launch_phased_pair_batch(const BatchArgs& a, int grp, int grid, cudaStream_t s) {
  phased_pair_batch_kernel<<<grid, kT, pp_smem_bytes(kN2 / 4, kN2 / 4), s>>>(a, grp);
  return cudaGetLastError();
}

}  // namespace fxc
