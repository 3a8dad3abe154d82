// corr_fold.cu — the FFT-8192 correlation kernel (the full-rate path).
//
// Same contract as corr_kernel<8192, 1, MODE_CORR> (src/main.rs:2491-2568
// per frame pair, partials reduced by reduce_partials_kernel), arranged to
// spend as few shared-memory wavefronts and barriers per frame pair as the
// data flow allows:
//   * decode straight from the staged .raw words: each thread's 16 samples of
//     a station sit at one bit position of 16 words (the frame stride N/16 is
//     a whole number of words), so a sample costs a word load, a rotate and a
//     masked merge into a byte offset of the level table.  A shuffle that
//     splits a 2-bit sample's bits takes two rotates; 1- and 2-bit shuffles
//     never rewrite the staged words.  The LSB flip (odd samples negated,
//     src/utils.rs:196-197) is a per-thread constant because N/16 is even: it
//     selects a negated copy of the level table;
//   * the station whose bin grid the products are indexed on (the primary:
//     station 1 for grid 0, station 2 for grid 1) is the real part of the
//     shared complex FFT, so the accumulation is free of grid selects;
//   * the trailing radix-2 pass is folded into the accumulation: a thread
//     reads Y[j], Y[j + N/2], Y[N/2 - j], Y[N - j] of the last radix-16 pass
//     and forms Z at j, N/2 - j, N/2 + j, N - j, i.e. both stations' spectra
//     at the bin pair (j, N/2 - j); the secondary spectrum goes through the
//     free ping-pong buffer to the thread that owns the band-shifted bin;
//   * four barriers per frame pair: after the first pass, after each
//     radix-16 pass, and between the two halves of the accumulation.  The
//     frame record is double-buffered so no barrier closes an iteration.
#include <cuda_runtime.h>
#include <stdint.h>

#include "decode_tables.cuh"
#include "fold_decode.cuh"
#include "fxc_device.cuh"
#include "fxc_kernels.h"

namespace fxc {
namespace {

constexpr int kN = 8192;
constexpr int kT = kN / 16;          // threads per CTA, one frame pair per iteration
constexpr int kH = kN / 2 + 1;
constexpr int kUnits = kN / 4 / kT;  // bin pairs per thread
static_assert(kUnits == 4, "the twiddle switch below covers W_16^0..3");
constexpr int kSlots = 2 * kUnits + 1;  // accumulator rows (bin N/4 by thread 0)

// Shared memory: level tables first, at a fixed address, so that the decode's
// table loads take an immediate base.
//   [0, 4096)      levels: primary at 0, secondary at 2048 (2^b f32 each, then their negations)
//   [4096, 4352)   rotate amounts: [2 stations][32 sample slots] u32
//   [4352, 4448)   frame records, double-buffered
//   [4448, 4464)   mbarriers; [4464, 4480) error flag
//   [4608, 12800)  byte LUTs of 4- and 8-bit generic shuffles
//   then the two ping-pong buffers and the staging slots
struct FoldLayout {
  uint32_t off_a, off_b, off_stage, stage_stride, total;
};
constexpr uint32_t kOffPos = kTabPos, kOffFi = 4352, kOffBar = 4448, kOffFlag = 4464, kOffLut = kTabLut;
constexpr uint32_t kOffA = kOffLut + 8192;

__host__ __device__ inline FoldLayout fold_layout(uint32_t raw_bytes) {
  FoldLayout L;
  L.off_a = kOffA;
  L.off_b = L.off_a + Geom<kN>::CSTRIDE * (uint32_t)sizeof(float2);
  L.off_stage = L.off_b + Geom<kN>::CSTRIDE * (uint32_t)sizeof(float2);
  L.stage_stride = (kFiBytes + raw_bytes + 127u) & ~127u;
  L.total = L.off_stage + kStages * L.stage_stride;
  return L;
}
static_assert(kOffA % 128 == 0 && kOffFi % 16 == 0 && kOffBar % 8 == 0, "alignment");

using fold::fold_inputs;
using fold::fold_station;

// The scan's decode tables (primary station first, decode_tables.cuh).
__device__ __forceinline__ void fold_build_tables(const StationParams& sp, const StationParams& ss,
                                                  bool preP, bool preS, uint8_t* smem, int tid) {
  build_decode_tables(sp, ss, preP, preS, smem, tid, kT);
}

__device__ __forceinline__ bool fold_split2(const StationParams& q) { return split_2bit(q); }

// Per-CTA state of the fold kernels that does not depend on the scan: the
// twiddle power chains, the two-row DIF twiddle bases, and the number of
// staging iterations consumed so far (it sets the mbarrier slot and phase, so
// a persistent CTA can run spans of several scans back to back).
template <int ROWS>
struct FoldCta {
  Twiddles<kN> tw;
  float2 dtw0, dtw1, wb1;
  uint32_t seq;
  uint32_t polls;  // bounded-wait limit of the last span (the drain uses it)
};

template <int ROWS>
__device__ __forceinline__ void fold_cta_init(uint8_t* smem, FoldCta<ROWS>& c) {
  const int tid = threadIdx.x;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
  int* flag = reinterpret_cast<int*>(smem + kOffFlag);
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
    *flag = 0;
    fence_proxy_async();
  }
  c.tw.init(tid);
  // ROWS = 2: row-1 DIF twiddle bases W_NF^t, W_NF^(t+512) (= W^t W_32) and
  // the row-1 fold's W_M^(t+1); all correctly rounded from FP64
  c.dtw0 = make_float2(1.f, 0.f);
  c.dtw1 = c.dtw0;
  c.wb1 = c.dtw0;
  if constexpr (ROWS == 2) {
    constexpr int NF = 2 * kN;
    double sn, cs;
    sincospi(-2.0 * (double)tid / (double)NF, &sn, &cs);
    c.dtw0 = make_float2((float)cs, (float)sn);
    sincospi(-2.0 * (double)(tid + NF / 32) / (double)NF, &sn, &cs);
    c.dtw1 = make_float2((float)cs, (float)sn);
    sincospi(-2.0 * (double)(tid + 1) / (double)kN, &sn, &cs);
    c.wb1 = make_float2((float)cs, (float)sn);
  }
  c.seq = 0;
  c.polls = kWaitPolls;
}

// Never leave a bulk copy in flight into a finished CTA's shared memory.
template <int ROWS>
__device__ __forceinline__ void fold_cta_drain(uint8_t* smem, const FoldCta<ROWS>& c) {
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
  const int* flag = reinterpret_cast<const int*>(smem + kOffFlag);
  if (threadIdx.x == 0 && *flag) {
    for (int s = 0; s < kStages; ++s) mbar_wait(&bars[s], 0, c.polls);
  }
}

// Frame pairs [it0, it1) of the sector described by p (ROWS = 1: FFT 8192;
// ROWS = 2: FFT 16384 as two 8192-point rows, the radix-2 DIF step fused into
// the decode, `row` 0 the even bins and 1 the odd bins), accumulated into the
// f64 partials at part ([4][NF/2 + 1]; each row writes only its own bins).
// Returns false when a bounded wait gave up (the CTA must stop).
template <int ROWS>
__device__ __forceinline__ bool fold_span(const CorrParams& p, int row, uint64_t it0, uint64_t it1,
                                          double* part, uint8_t* smem, const FoldLayout& L,
                                          FoldCta<ROWS>& c) {
  constexpr int NF = kN * ROWS;       // frame FFT length
  constexpr int HF = NF / 2 + 1;      // bins
  static_assert(ROWS == 1 || ROWS == 2, "one or two rows");
  float* lv = reinterpret_cast<float*>(smem);
  uint32_t* pos = reinterpret_cast<uint32_t*>(smem + kOffPos);
  FrameInfo* finfo = reinterpret_cast<FrameInfo*>(smem + kOffFi);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kOffBar);
  int* flag = reinterpret_cast<int*>(smem + kOffFlag);
  uint32_t* lut = reinterpret_cast<uint32_t*>(smem + kOffLut);
  float2* bufA = reinterpret_cast<float2*>(smem + L.off_a);
  float2* bufB = reinterpret_cast<float2*>(smem + L.off_b);
  uint8_t* stage = smem + L.off_stage;
  const int tid = threadIdx.x;
  const Twiddles<kN>& tw = c.tw;
  const uint32_t seq0 = c.seq;

  // primary station (real part of the FFT, products indexed on its bins) first
  const bool g0 = p.grid == 0;
  const StationParams& sp = p.st[g0 ? 0 : 1];
  const StationParams& ss = p.st[g0 ? 1 : 0];
  const int bitsP = sp.bits, bitsS = ss.bits;
  // 4- and 8-bit stations with a non-identity shuffle are rewritten in place
  // (byte LUTs); 1- and 2-bit stations are decoded from the raw words
  const bool preP = bitsP > 2 && sp.shkind != SH_IDENTITY;
  const bool preS = bitsS > 2 && ss.shkind != SH_IDENTITY;

  const uint32_t bpfP = sp.bpf, bpfS = ss.bpf;
  const uint8_t* rawP = sp.raw;
  const uint8_t* rawS = ss.raw;
  const FrameInfo* gfi = p.finfo;
  const uint32_t polls = p.wait_polls ? p.wait_polls : kWaitPolls;
  const bool withhold = (p.debug_flags & DBG_WITHHOLD_COPIES) != 0;
  c.polls = polls;

  // slot: [FrameInfo][primary frame][secondary frame]
  auto issue = [&](uint64_t it) {
    const int slot = (int)((seq0 + (uint32_t)(it - it0)) % kStages);
    uint8_t* dst = stage + slot * L.stage_stride;
    mbar_expect_tx(&bars[slot], kFiBytes + bpfP + bpfS);
    if (withhold) return;  // failure injection: the wait below runs out
    bulk_g2s(dst, gfi + it, kFiBytes, &bars[slot]);
    bulk_g2s(dst + kFiBytes, rawP + it * bpfP, bpfP, &bars[slot]);
    bulk_g2s(dst + kFiBytes + bpfP, rawS + it * bpfS, bpfS, &bars[slot]);
  };
  // The previous span, if any, is past its last decode and its last frame's
  // barriers: the staging ring and the tables are free.  The first frames'
  // copies go out first, the tables are built while they are in flight.
  __syncthreads();
  if (tid == 0) {
    fence_proxy_async();
    for (uint64_t it = it0; it < it1 && it < it0 + kStages; ++it) issue(it);
  }
  // ---- constant tables of this scan
  fold_build_tables(sp, ss, preP, preS, smem, tid);
  const bool splitP = fold_split2(sp), splitS = fold_split2(ss);
  const float2 dtw0 = c.dtw0, dtw1 = c.dtw1, wb1 = c.wb1;
  __syncthreads();

  // acc[2i]: bin tid + T i, acc[2i+1]: bin N/2 - tid - T i, acc[2 kUnits]: bin N/4 (tid 0).
  // Columns: primary ACF, secondary ACF (at the primary bin), XCF re, im.
  float acc[kSlots][4];
#pragma unroll
  for (int i = 0; i < kSlots; ++i)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[i][v] = 0.f;
  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s;
  const int ov = a1e - a1s;
  const int sb = a2s - a1s;
  const int ovs = g0 ? a1s : a2s;   // overlap on the primary grid: [ovs, ovs + ov)
  const int qoff = g0 ? sb : -sb;   // secondary bin = primary bin + qoff
  const bool want_acf = (p.products & 1u) != 0;
  const bool want_xcf = (p.products & 2u) != 0;
  const bool ov_only = (p.products & 16u) != 0;
  const float xconj = g0 ? 1.0f : -1.0f;  // XCF = S1 conj(S2): conj(P conj(S)) for grid 1
  const int lsbP = sp.lsb ? 1 : 0, lsbS = ss.lsb ? 1 : 0;
  const uint32_t flush_every = p.flush_every;
  uint32_t* err = p.err;
  bool first_flush = true;
  uint32_t since_flush = 0;
  const int colP = g0 ? 0 : 1, colS = g0 ? 1 : 0;  // output columns of the two ACFs

  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i < kSlots; ++i) {
      if (i == kSlots - 1 && tid != 0) continue;
      if (ROWS == 2 && row == 1 && i == kSlots - 1) continue;  // bin N/4 is even
      const int j = tid + kT * (i >> 1);
      const int bin = ROWS == 1 ? ((i == kSlots - 1) ? kN / 4 : ((i & 1) ? kN / 2 - j : j))
                                : ((i == kSlots - 1) ? NF / 4
                                   : ((i & 1) ? NF / 2 - 2 * j - row : 2 * j + row));
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int col = v == 0 ? colP : (v == 1 ? colS : v);
        double* q = part + (size_t)col * HF + bin;
        *q = (first_flush ? 0.0 : *q) + (double)acc[i][v];
        acc[i][v] = 0.f;
      }
    }
    first_flush = false;
    since_flush = 0;
  };

  bool ok = true;
  for (uint64_t it = it0; it < it1; ++it) {
    const uint32_t q_it = seq0 + (uint32_t)(it - it0);
    const int slot = (int)(q_it % kStages);
    const uint32_t parity = (q_it / kStages) & 1u;
    const int fb = (int)(q_it & 1u);
    if (!mbar_wait(&bars[slot], parity, polls)) {
      atomicOr(flag, 1);
      atomicOr(err, ERR_WAIT_TIMEOUT);
    }
    uint8_t* st = stage + slot * L.stage_stride;
    uint32_t* wP = reinterpret_cast<uint32_t*>(st + kFiBytes);
    uint32_t* wS = reinterpret_cast<uint32_t*>(st + kFiBytes + bpfP);
    const FrameInfo* fs = reinterpret_cast<const FrameInfo*>(st);
    const int sP = g0 ? fs->s1 : fs->s2;
    const int sS = g0 ? fs->s2 : fs->s1;
    if (tid == 0) finfo[fb] = *fs;
    if (preP || preS) {  // CTA-uniform
      preshuffle_slot(wP, bpfP / 4, preP ? sp.shkind : SH_IDENTITY, lut, wS, bpfS / 4,
                      preS ? ss.shkind : SH_IDENTITY, lut + 1024, tid, kT);
      __syncthreads();
    }

    // ---- decode + first radix-16 pass into bufA
    {
      float2 v[16];
      const int mP = tid - sP, mS = tid - sS;
      const int cP = mP & ((32 / bitsP) - 1), cS = mS & ((32 / bitsS) - 1);
      const uint32_t tbP = (uint32_t)((mP & lsbP) << (bitsP + 2));
      // the secondary station enters odd frames negated (see sgn below)
      const uint32_t tbS = 2048u + (uint32_t)((((uint32_t)mS & (uint32_t)lsbS) ^ (uint32_t)(it & 1u))
                                              << (bitsS + 2));
      fold_station<false, ROWS>(bitsP, splitP, wP, smem, sP, pos[cP], tbP, v, tid, row == 1);
      fold_station<true, ROWS>(bitsS, splitS, wS, smem, sS, pos[32 + cS], tbS, v, tid, row == 1);
      if (ROWS == 2 && row == 1) {
        // DIF twiddle W_NF^m, m = t + 512 r = W^t W_32^r: even r from
        // b0 = W^t, odd r from b1 = W^t W_32, times W_16^(r/2)
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          float2 w;
          switch (r >> 1) {  // compile-time after unrolling
            case 0: w = (r & 1) ? dtw1 : dtw0; break;
            case 1: w = mul_w16<1>((r & 1) ? dtw1 : dtw0); break;
            case 2: w = mul_w16<2>((r & 1) ? dtw1 : dtw0); break;
            case 3: w = mul_w16<3>((r & 1) ? dtw1 : dtw0); break;
            case 4: w = mul_w16<4>((r & 1) ? dtw1 : dtw0); break;
            case 5: w = mul_w16<5>((r & 1) ? dtw1 : dtw0); break;
            case 6: w = mul_w16<6>((r & 1) ? dtw1 : dtw0); break;
            default: w = mul_w16<7>((r & 1) ? dtw1 : dtw0); break;
          }
          v[r] = cmul(v[r], w);
        }
      }
      dft16(v);
      float2* dst = bufA + 17 * tid;  // cpad(16 t + r) = 17 t + r
#pragma unroll
      for (int r = 0; r < 16; ++r) dst[r] = v[out_pos<16>(r)];
    }
    const float2* Y = fft_rest<kN, true>(bufA, bufB, tid, tw);
    // fft_rest opened with a barrier after the first pass: the staging slot
    // is consumed, refill it with iteration it + kStages.  Not after a wait
    // gave up (every thread's timeout was flagged before that barrier): the
    // slot's phase never completed, and the CTA stops below.
    if (tid == 0 && it + kStages < it1 && !*flag) {
      fence_proxy_async();
      issue(it + kStages);
    }
    float2* Q = (Y == bufA) ? bufB : bufA;  // free buffer: secondary spectrum by bin
    __syncthreads();
    if (*flag) {  // no thread writes the flag before the next barrier
      ok = false;
      break;
    }

    // ---- trailing radix-2 pass + two-for-one split (x2) at the bin pairs
    const FrameInfo& F = finfo[fb];
    float sn, cs;
    const int a_gs = ovs;
    const float2 mix = F.fr_mix;
    // bins of unit i: up = ROWS * j + row, down = NF/2 - ROWS * j - row, j = tid + T i
    const int bup0 = ROWS * tid + row, bdn0 = NF / 2 - ROWS * tid - row;
    __sincosf(fmaf((float)(bup0 - a_gs), F.dphi, F.phi0), &sn, &cs);
    float2 rup = cmul(mix, make_float2(cs, sn));
    __sincosf(fmaf((float)(bdn0 - a_gs), F.dphi, F.phi0), &sn, &cs);
    float2 rdn = cmul(mix, make_float2(cs, sn));
    __sincosf((float)(ROWS * kT) * F.dphi, &sn, &cs);
    const float2 rstep = make_float2(cs, sn);
    const bool quarter = tid == 0 && (ROWS == 1 || row == 0);  // bin NF/4 (even)
    float2 rq = make_float2(0.f, 0.f);
    if (quarter) {
      __sincosf(fmaf((float)(NF / 4 - a_gs), F.dphi, F.phi0), &sn, &cs);
      rq = cmul(mix, make_float2(cs, sn));
    }

    // Rounding in the shared complex FFT leaks a fixed fraction (~1e-6) of
    // each station's spectrum into the other's; summed over frames that
    // would bias the cross-spectrum by ~1e-6 of the auto-spectra, i.e. by
    // 1e-6/rho of a weakly correlated XCF.  Negating the secondary station's
    // input on odd frames (undone exactly here) alternates the sign of that
    // leak, so it cancels in the sum instead of accumulating.
    const float sgn = (it & 1u) ? -1.0f : 1.0f;
    float2 prim[2 * kUnits];
#pragma unroll
    for (int i = 0; i < kUnits; ++i) {
      const int j = tid + kT * i;
      float2 wj;  // W_N^j = W_N^tid W_16^i
      switch (i) {  // compile-time after unrolling
        case 0: wj = tw.w[Geom<kN>::P16]; break;
        case 1: wj = mul_w16<1>(tw.w[Geom<kN>::P16]); break;
        case 2: wj = mul_w16<2>(tw.w[Geom<kN>::P16]); break;
        default: wj = mul_w16<3>(tw.w[Geom<kN>::P16]); break;
      }
      // row-local columns: Z[j], Z[j + M/2] from Y[j], Y[j + M/2]; the mirror
      // pair from Y[c0], Y[c0 + M/2] with c0 = M/2 - j (one row: mirror of
      // column j is M - j) or M/2 - 1 - j (odd row: mirror is M - 1 - j)
      const int c0 = (ROWS == 2 && row == 1) ? kN / 2 - 1 - j : kN / 2 - j;
      const float2 a = Y[j], b = Y[j + kN / 2], cc = Y[c0], d = Y[(c0 + kN / 2) & (kN - 1)];
      // W_M^c0 = -conj(W_M^(M/2 - c0)): W^j for the even mirror, W^(j+1) for the odd one
      float2 wm = wj;
      if (ROWS == 2 && row == 1) {
        switch (i) {
          case 0: wm = wb1; break;
          case 1: wm = mul_w16<1>(wb1); break;
          case 2: wm = mul_w16<2>(wb1); break;
          default: wm = mul_w16<3>(wb1); break;
        }
      }
      const float2 wb = cmul(wj, b), wd = cmulc(d, wm);  // W^j b, conj(W^(M/2-c0)) d
      const float2 zj = cadd(a, wb), zjh = csub(a, wb);  // Z[j], Z[j + M/2]
      const float2 zmn = cadd(cc, wd);                   // Z[c0 + M/2] (mirror of j)
      // Z[c0]; for an even row and j = 0 that is Z[M/2] = Y[0] - Y[M/2]
      const float2 zm = ((ROWS == 1 || row == 0) && j == 0) ? zjh : csub(cc, wd);
      // primary = real part: P[k] = (Z[k] + conj Z[N-k]), S[k] = -i (Z[k] - conj Z[N-k])
      const int bu = ROWS * j + row, bd = NF / 2 - ROWS * j - row;  // global bins
      prim[2 * i] = make_float2(zj.x + zmn.x, zj.y - zmn.y);
      Q[bu] = make_float2(sgn * (zj.y + zmn.y), sgn * (zmn.x - zj.x));
      prim[2 * i + 1] = make_float2(zm.x + zjh.x, zm.y - zjh.y);
      Q[bd] = make_float2(sgn * (zm.y + zjh.y), sgn * (zjh.x - zm.x));
    }
    float2 prim_q = make_float2(0.f, 0.f);
    if (quarter) {  // column M/4: Z[M/4] = Y[M/4] - i Y[3M/4], Z[3M/4] = Y[M/4] + i Y[3M/4]
      const float2 a = Y[kN / 4], b = Y[3 * kN / 4];
      const float2 zq = make_float2(a.x + b.y, a.y - b.x), zq3 = make_float2(a.x - b.y, a.y + b.x);
      prim_q = make_float2(zq.x + zq3.x, zq.y - zq3.y);
      Q[NF / 4] = make_float2(sgn * (zq.y + zq3.y), sgn * (zq3.x - zq.x));
    }
    __syncthreads();

    // ---- accumulation (constant indices into acc[][]: a runtime index
    // would move it to local memory)
    auto bin_acc = [&](int bin, float2 pv, float2 r, float* a) {
      const bool inov = (unsigned)(bin - ovs) < (unsigned)ov;
      const float2 q = Q[inov ? bin + qoff : bin];
      if (want_acf && (!ov_only || inov)) a[0] = fmaf(pv.x, pv.x, fmaf(pv.y, pv.y, a[0]));
      if (inov) {
        if (want_acf) a[1] = fmaf(q.x, q.x, fmaf(q.y, q.y, a[1]));
        if (want_xcf) {
          float2 x = cmulc(pv, q);
          x.y *= xconj;
          a[2] = fmaf(x.x, r.x, fmaf(-x.y, r.y, a[2]));
          a[3] = fmaf(x.x, r.y, fmaf(x.y, r.x, a[3]));
        }
      }
    };
#pragma unroll
    for (int i = 0; i < kUnits; ++i) {
      const int j = tid + kT * i;
      bin_acc(ROWS * j + row, prim[2 * i], rup, acc[2 * i]);
      bin_acc(NF / 2 - ROWS * j - row, prim[2 * i + 1], rdn, acc[2 * i + 1]);
      rup = cmul(rup, rstep);
      rdn = cmulc(rdn, rstep);
    }
    if (quarter) bin_acc(NF / 4, prim_q, rq, acc[kSlots - 1]);
    if (++since_flush >= flush_every) flush();
  }
  if (since_flush > 0 || first_flush) flush();
  c.seq = seq0 + (uint32_t)(it1 - it0);
  return ok;
}

}  // namespace

// ROWS = 1: FFT 8192.  ROWS = 2: FFT 16384 as two 8192-point rows; one launch
// per row, `row` = 0 handles the even bins, 1 the odd bins, both accumulate
// into the same per-CTA partials.
template <int ROWS>
__global__ void __launch_bounds__(kT, 1) corr_fold_kernel(const CorrParams p, int row) {
  constexpr int HF = kN * ROWS / 2 + 1;
  extern __shared__ __align__(128) uint8_t smem[];
  const FoldLayout L = fold_layout(p.stage_bytes);
  FoldCta<ROWS> c;
  fold_cta_init<ROWS>(smem, c);
  const uint64_t iters = p.nf;
  const uint64_t it0 = (blockIdx.x * iters) / gridDim.x;
  const uint64_t it1 = ((blockIdx.x + 1) * iters) / gridDim.x;
  fold_span<ROWS>(p, row, it0, it1, p.partials + (size_t)blockIdx.x * 4 * HF, smem, L, c);
  fold_cta_drain(smem, c);
}

// Batched: a persistent grid takes the items of batch group `grp` by ticket;
// every item is a frame range of one scan's sector (its own tables, frame
// records and raw words) with its own partials.  The layout is sized for the
// largest stage (8-bit stations), so one launch serves every bit depth.
template <int ROWS>
__global__ void __launch_bounds__(kT, 1) corr_fold_batch_kernel(const BatchArgs a, int grp) {
  extern __shared__ __align__(128) uint8_t smem[];
  const FoldLayout L = fold_layout(2u * (uint32_t)(kN * ROWS));
  uint32_t* ticket = reinterpret_cast<uint32_t*>(smem + kOffFlag + 4);
  FoldCta<ROWS> c;
  fold_cta_init<ROWS>(smem, c);
  const uint32_t n_items = a.hdr->nitems[grp];
  const BatchItem* items = a.hdr->items + a.hdr->item0[grp];
  const BatchScan* scans = a.hdr->scans;
  for (;;) {
    if (threadIdx.x == 0) *ticket = atomicAdd(&a.hdr->ticket[grp], 1u);
    __syncthreads();
    const uint32_t k = *ticket;  // fold_span opens with a barrier before the next write
    if (k >= n_items) break;
    const BatchItem w = items[k];
    if (!fold_span<ROWS>(scans[w.scan].p, (int)w.row, w.f0, w.f1, a.partials + w.part, smem, L,
                         c))
      break;
  }
  fold_cta_drain(smem, c);
}

// The decode + integer shift of the FFT-8192 correlation kernel on its own
// (the stage entry point fxc_decode_device): every frame's words go through
// the same tables and fold_inputs path as in fold_span, and the 16 inputs a
// thread would feed its first radix-16 pass, x[t + 512 r - shift], are
// written out (level scale undone exactly) instead of transformed.
__global__ void __launch_bounds__(kT) fold_decode_kernel(const CorrParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x;
  const bool g0 = p.grid == 0;
  const StationParams& sp = p.st[g0 ? 0 : 1];
  const StationParams& ss = p.st[g0 ? 1 : 0];
  const bool preP = sp.bits > 2 && sp.shkind != SH_IDENTITY;
  const bool preS = ss.bits > 2 && ss.shkind != SH_IDENTITY;
  uint32_t* pos = reinterpret_cast<uint32_t*>(smem + kOffPos);
  uint32_t* lut = reinterpret_cast<uint32_t*>(smem + kOffLut);
  uint32_t* wP = reinterpret_cast<uint32_t*>(smem + kOffA);
  uint32_t* wS = wP + sp.bpf / 4;
  fold_build_tables(sp, ss, preP, preS, smem, tid);
  const bool splitP = fold_split2(sp), splitS = fold_split2(ss);
  const int lsbP = sp.lsb ? 1 : 0, lsbS = ss.lsb ? 1 : 0;
  const int bitsP = sp.bits, bitsS = ss.bits;
  float* outP = g0 ? p.out_a : p.out_b;
  float* outS = g0 ? p.out_b : p.out_a;
  const float uP = 1.0f / sp.scale, uS = 1.0f / ss.scale;  // powers of two: exact
  for (uint64_t f = blockIdx.x; f < p.nf; f += gridDim.x) {
    __syncthreads();  // tables built / previous frame's words consumed
    const uint4* gP = reinterpret_cast<const uint4*>(sp.raw + f * sp.bpf);
    const uint4* gS = reinterpret_cast<const uint4*>(ss.raw + f * ss.bpf);
    for (uint32_t i = tid; i < sp.bpf / 16; i += kT) reinterpret_cast<uint4*>(wP)[i] = gP[i];
    for (uint32_t i = tid; i < ss.bpf / 16; i += kT) reinterpret_cast<uint4*>(wS)[i] = gS[i];
    __syncthreads();
    if (preP || preS) {
      preshuffle_slot(wP, sp.bpf / 4, preP ? sp.shkind : SH_IDENTITY, lut, wS, ss.bpf / 4,
                      preS ? ss.shkind : SH_IDENTITY, lut + 1024, tid, kT);
      __syncthreads();
    }
    const FrameInfo fi = p.finfo[f];
    const int sP = g0 ? fi.s1 : fi.s2, sS = g0 ? fi.s2 : fi.s1;
    const int mP = tid - sP, mS = tid - sS;
    const int cP = mP & ((32 / bitsP) - 1), cS = mS & ((32 / bitsS) - 1);
    const uint32_t tbP = (uint32_t)((mP & lsbP) << (bitsP + 2));
    const uint32_t tbS = 2048u + (uint32_t)((mS & lsbS) << (bitsS + 2));
    float2 v[16];
    fold_station<false, 1>(bitsP, splitP, wP, smem, sP, pos[cP], tbP, v, tid, false);
    fold_station<true, 1>(bitsS, splitS, wS, smem, sS, pos[32 + cS], tbS, v, tid, false);
    float* oP = outP + f * kN + tid;
    float* oS = outS + f * kN + tid;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      oP[r * kT] = v[r].x * uP;
      oS[r * kT] = v[r].y * uS;
    }
  }
}

cudaError_t launch_fold_decode(const CorrParams& p, int grid, cudaStream_t stream) {
  // tables, then both stations' words of one frame (8-bit stations at most)
  const uint32_t smem = kOffA + 2u * kN;
  fold_decode_kernel<<<grid, kT, smem, stream>>>(p);
  return cudaGetLastError();
}

uint32_t fold_smem_bytes(uint32_t stage_bytes) { return fold_layout(stage_bytes).total; }

// The shared-memory limit of a kernel is a per-function attribute shared by
// every host thread: it is always set to the largest layout (8-bit stations),
// so that a concurrent launch with a larger stage never meets a limit another
// thread has just lowered.
cudaError_t launch_corr_fold(const CorrParams& p, int grid, cudaStream_t stream) {
  const uint32_t smem = fold_smem_bytes(p.stage_bytes);
  cudaError_t e = cudaFuncSetAttribute(corr_fold_kernel<1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fold_smem_bytes(2u * kN));
  if (e != cudaSuccess) return e;
  corr_fold_kernel<1><<<grid, kT, smem, stream>>>(p, 0);
  return cudaGetLastError();
}

bool corr_fold2_supported(const CorrParams& p) {
  // a row holds the bins of one parity: the band shift must keep it
  return ((p.a2s - p.a1s) & 1) == 0 && fold_smem_bytes(p.stage_bytes) <= 232448u;
}

cudaError_t launch_corr_fold2(const CorrParams& p, int grid, cudaStream_t stream) {
  const uint32_t smem = fold_smem_bytes(p.stage_bytes);
  cudaError_t e = cudaFuncSetAttribute(corr_fold_kernel<2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fold_smem_bytes(4u * kN));
  if (e != cudaSuccess) return e;
  for (int row = 0; row < 2; ++row) {
    corr_fold_kernel<2><<<grid, kT, smem, stream>>>(p, row);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

uint32_t fold_batch_smem_bytes(int rows) { return fold_layout(2u * (uint32_t)(kN * rows)).total; }

cudaError_t prepare_fold_batch(int rows) {
  const int smem = (int)fold_batch_smem_bytes(rows);
  return rows == 1 ? cudaFuncSetAttribute(corr_fold_batch_kernel<1>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                   : cudaFuncSetAttribute(corr_fold_batch_kernel<2>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

int fold_batch_ctas_per_sm(int rows) {
  int nb = 0;
  const cudaError_t e =
      rows == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, corr_fold_batch_kernel<1>, kT,
                                                                fold_batch_smem_bytes(1))
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, corr_fold_batch_kernel<2>, kT,
                                                                fold_batch_smem_bytes(2));
  return e == cudaSuccess ? nb : 0;
}

cudaError_t launch_fold_batch(int rows, const BatchArgs& a, int grp, int grid, cudaStream_t s) {
  const uint32_t smem = fold_batch_smem_bytes(rows);
  if (rows == 1) corr_fold_batch_kernel<1><<<grid, kT, smem, s>>>(a, grp);
  else corr_fold_batch_kernel<2><<<grid, kT, smem, s>>>(a, grp);
  return cudaGetLastError();
}

}  // namespace fxc
