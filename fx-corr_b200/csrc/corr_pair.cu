// corr_pair.cu — correlation for FFT 32768 and 65536 (N = C * M, M = 8192,
// C = 4, 8) with 1- and 2-bit stations and a band shift that is a multiple of
// C: one thread-block cluster of C/2 CTAs per frame pair, each CTA owning a
// mirror pair of rows.  FFT 16384 (C = 2) with an odd band shift: a cluster
// of one CTA holding both rows.
//
// Same contract and decomposition as corr_cluster_kernel (src/main.rs:
// 2491-2568 per frame pair; y_q[m] = W_N^(m q) sum_c z[m + M c] W_C^(c q),
// Z[C k + q] = FFT_M(y_q)[k]), but CTA r owns rows A = r and B = C - r (CTA 0:
// rows 0 and C/2), so that
//   * the two-for-one split, which pairs bin C j + q with row C - q, reads
//     both rows from the CTA's own shared memory (no mirror exchange);
//   * the radix-C step's rows that leave the CTA are (C - 2) of C (48 KB per
//     row at C = 8 instead of 56 KB plus the 32 KB mirror half row);
//   * a cluster has C/2 CTAs: 33 clusters of 4 fit the B200 where only 15
//     clusters of 8 do (132 SMs instead of 120), and 148 clusters of one;
//   * the band-shifted secondary spectrum of a bin lies in the same row (the
//     shift is a multiple of C), so it never leaves the CTA; at C = 2 it may
//     lie in the other row, which is in the same CTA: both rows are split
//     before either is accumulated.
// The accumulators of both rows' bins (32 f32 per thread and row) live in
// tensor memory (TMEM, 256 columns of the SM's 512): registers could hold one
// row's, not two, beside the FFT; each row's are loaded and stored once per
// frame with tcgen05.ld / tcgen05.st.  Two cluster barriers per frame: after the radix-C
// rows are stored (B1), and once every CTA has read its row buffers (B0, whose
// wait sits after the next frame's first decode).  The shared-memory layout
// holds three row buffers, which leaves room for 1- and 2-bit stations only.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <type_traits>

#include "cluster_frame.cuh"
#include "decode_tables.cuh"
#include "fxc_device.cuh"
#include "fxc_kernels.h"
#include "tmem.cuh"

namespace fxc {
namespace {

using namespace clu;
constexpr int kJ = kM / 2 / kT;  // bins per thread and row (8)

// Shared memory (bytes): the decode tables [0, kTabEnd) with the frame
// records, the staging mbarrier, the cluster error flag and the TMEM address
// in their gap; then the row buffers XA, XB (written by the cluster's
// decoders; XA is also the FFT scratch and then holds row B's spectrum, XB
// then the secondary spectra of both rows' bins), Y (row A's FFT, then its
// spectrum), and one staging slot [FrameInfo (128 B)][primary regions]
// [secondary regions].
constexpr uint32_t kPrFi = 4352, kPrBar = 4448, kPrFlag = 4456, kPrTmem = 4460;
constexpr uint32_t kPrBuf = (uint32_t)Geom<kM>::CSTRIDE * (uint32_t)sizeof(float2);
constexpr uint32_t kPrXA = kTabEnd, kPrXB = kPrXA + kPrBuf, kPrY = kPrXB + kPrBuf;
constexpr uint32_t kPrStage = kPrY + kPrBuf;
constexpr uint32_t kPrMaxSmem = 232448;  // 227 KB per CTA on sm_100
constexpr uint32_t kTmemCols = 256;      // 16 warps x 64 accumulators, 4 warps per lane quarter
static_assert(kPrFi + 2 * kFiBytes <= kPrBar && kPrTmem + 4 <= kTabLut, "records fit the gap");
static_assert(kPrStage % 128 == 0, "alignment");

__host__ __device__ constexpr uint32_t pr_stage_bytes(int c, int bits_p, int bits_s) {
  return (128u + 4u * (uint32_t)c *
                     (uint32_t)(region_words(2 * kM / c, bits_p) + region_words(2 * kM / c, bits_s)) +
          127u) & ~127u;
}
__host__ __device__ constexpr uint32_t pr_smem_bytes(int c, int bits_p, int bits_s) {
  return kPrStage + pr_stage_bytes(c, bits_p, bits_s);
}
static_assert(pr_smem_bytes(8, 2, 2) <= kPrMaxSmem && pr_smem_bytes(4, 2, 2) <= kPrMaxSmem &&
                  pr_smem_bytes(2, 2, 2) <= kPrMaxSmem,
              "2-bit stations fit");

// Owner CTA of row k (the CTA holding the mirror pair {k, C - k}) and whether
// k is its row A.
template <int C>
__host__ __device__ constexpr int pr_owner(int k) {
  return k == C / 2 ? 0 : (k < C - k ? k : C - k);
}
template <int C>
__host__ __device__ constexpr bool pr_is_a(int k) {
  return k != C / 2 && k <= C - k;
}

template <int C>
__global__ void __cluster_dims__(C / 2, 1, 1) __launch_bounds__(kT, 1)
    corr_pair_kernel(const __grid_constant__ CorrParams p) {
  constexpr int P = C / 2;           // CTAs per cluster
  constexpr int N = C * kM, H = N / 2 + 1;
  constexpr int CW = kM / P;         // columns per CTA
  constexpr int U = CW / kT;         // column groups per thread
  constexpr int UH = 16 / C;         // column groups per decode half
  static_assert(U == 2 * UH, "two decode halves");
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = (int)cl_rank();
  const int rowA = r, rowB = r == 0 ? C / 2 : C - r;
  const uint32_t cid = cl_id(), ncl = cl_count();
  FrameInfo* finfo = reinterpret_cast<FrameInfo*>(smem + kPrFi);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kPrBar);
  int* flag = reinterpret_cast<int*>(smem + kPrFlag);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kPrTmem);
  const uint32_t* pos = reinterpret_cast<const uint32_t*>(smem + kTabPos);
  float2* XA = reinterpret_cast<float2*>(smem + kPrXA);
  float2* XB = reinterpret_cast<float2*>(smem + kPrXB);
  float2* Y = reinterpret_cast<float2*>(smem + kPrY);
  uint8_t* stage = smem + kPrStage;

  const bool g0 = p.grid == 0;
  const StationParams& sp = p.st[g0 ? 0 : 1];
  const StationParams& ss = p.st[g0 ? 1 : 0];
  const int bitsP = sp.bits, bitsS = ss.bits;
  const int lgP = log2_spw(bitsP), lgS = log2_spw(bitsS);
  const int LP = region_words(CW, bitsP), LS = region_words(CW, bitsS);
  const uint32_t polls = p.wait_polls ? p.wait_polls : kWaitPolls;
  const bool withhold = (p.debug_flags & DBG_WITHHOLD_COPIES) != 0;
  const uint64_t it0 = ((uint64_t)cid * p.nf) / ncl, it1 = ((uint64_t)(cid + 1) * p.nf) / ncl;
  double* part = p.partials + (size_t)cid * 4 * H;

  // Frame `it`'s copies into the staging slot, by the lanes of warp 0: lane
  // c < C the primary's region c, lane C + c the secondary's, lane 2C the
  // frame record; each region clamped to the frame's words.
  auto issue = [&](uint64_t it, int shP, int shS) {
    uint32_t bytes = 0;
    const uint8_t* src = nullptr;
    uint8_t* d = nullptr;
    if (lane < 2 * C) {
      const bool sec = lane >= C;
      const int c = sec ? lane - C : lane;
      const int lg = sec ? lgS : lgP, L = sec ? LS : LP;
      const uint32_t bpf = sec ? ss.bpf : sp.bpf;
      const int nw = (int)(bpf >> 2);
      const int a = r * CW - (sec ? shS : shP);
      const int wa = ((a >> lg) & ~3) + c * (kM >> lg);
      const int lo = max(wa, 0), hi = min(wa + L, nw);
      if (hi > lo) {
        bytes = 4u * (uint32_t)(hi - lo);
        src = (sec ? ss.raw : sp.raw) + it * bpf + 4u * (uint32_t)lo;
        d = stage + 128 + (sec ? 4 * C * LP : 0) + 4 * (c * L + lo - wa);
      }
    } else if (lane == 2 * C) {
      bytes = kFiBytes;
      src = reinterpret_cast<const uint8_t*>(p.finfo + it);
      d = stage;
    }
    const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
    if (lane == 0) mbar_expect_tx(bar, total);
    __syncwarp();
    if (bytes && !withhold) bulk_g2s(d, src, bytes, bar);  // withheld: the wait runs out
  };
  auto shifts = [&](uint64_t it, int* shP, int* shS) {
    const FrameInfo* g = p.finfo + it;
    *shP = g0 ? g->s1 : g->s2;
    *shS = g0 ? g->s2 : g->s1;
  };
  auto raise = [&]() {
    *reinterpret_cast<volatile int*>(flag) = 1;
    for (int k = 0; k < P; ++k)
      if (k != r) cl_st_u32(cl_map(flag, (uint32_t)k), 1u);
    atomicOr(p.err, ERR_WAIT_TIMEOUT);
  };

  if (tid == 0) {
    mbar_init(bar, 1);
    *flag = 0;
    fence_proxy_async();
  }
  if (warp == 0) {
    // the accumulators: 256 TMEM columns (this kernel runs one CTA per SM)
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t taddr =
      *tmem_slot + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(64 * (warp >> 2));
  {
    float z[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) z[i] = 0.f;
    tmem_st32(taddr, z);
    tmem_st32(taddr + 32u, z);
  }
  if (tid < 32 && it0 < it1) {
    int a, b;
    shifts(it0, &a, &b);
    issue(it0, a, b);
  }
  build_decode_tables(sp, ss, false, false, smem, tid, kT);
  const bool splitP = split_2bit(sp), splitS = split_2bit(ss);
  Twiddles<kM> tw;
  tw.init(tid);
  // W_M^(t+1): the mirror half's trailing radix-2 twiddle (correctly rounded)
  float2 wb1;
  {
    double sn, cs;
    sincospi(-2.0 * (double)(tid + 1) / (double)kM, &sn, &cs);
    wb1 = make_float2((float)cs, (float)sn);
  }
  // radix-C step twiddle bases W_N^m of the thread's columns m = r CW + t + T u;
  // C = 2 keeps W_N^t and W_N^(t + T) only: W_N^(t + T u) = W_N^(t + T (u mod 2)) W_16^(u / 2)
  constexpr int ND = C == 2 ? 2 : U;
  float2 dbase[ND];
#pragma unroll
  for (int u = 0; u < ND; ++u) {
    double sn, cs;
    sincospi(-2.0 * (double)(r * CW + tid + kT * u) / (double)N, &sn, &cs);
    dbase[u] = make_float2((float)cs, (float)sn);
  }
  auto dtw = [&](int u) -> float2 {  // u is a compile-time constant after unrolling
    if constexpr (C != 2) {
      return dbase[u];
    } else {
      const float2 b = dbase[u & 1];
      switch (u >> 1) {
        case 0: return b;
        case 1: return mul_w16<1>(b);
        case 2: return mul_w16<2>(b);
        case 3: return mul_w16<3>(b);
        case 4: return mul_w16<4>(b);
        case 5: return mul_w16<5>(b);
        case 6: return mul_w16<6>(b);
        default: return mul_w16<7>(b);
      }
    }
  };
  // every CTA of the cluster has started, zeroed its flag and built its
  // tables before any CTA stores into another's shared memory
  cl_sync();
  cl_arrive();  // B0 of the frame before the first

  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s;
  const int ov = a1e - a1s;
  const int sb = a2s - a1s;
  const int ovs = g0 ? a1s : a2s;   // overlap on the primary grid: [ovs, ovs + ov)
  const int qoff = g0 ? sb : -sb;   // secondary bin = primary bin + qoff (a multiple of C if C > 2)
  const int dq = -qoff / C;         // the primary bin of a secondary bin: row index + dq (C > 2)
  const bool want_acf = (p.products & 1u) != 0;
  const bool want_xcf = (p.products & 2u) != 0;
  const bool ov_only = (p.products & 16u) != 0;
  const float xconj = g0 ? 1.0f : -1.0f;  // XCF = S1 conj(S2): conj(P conj(S)) for grid 1
  const int lsbP = sp.lsb ? 1 : 0, lsbS = ss.lsb ? 1 : 0;
  const int colP = g0 ? 0 : 1, colS = g0 ? 1 : 0;  // output columns of the two ACFs
  const bool half = r == 0 && tid == 0;            // bin N/2 (row 0, index M/2)
  const uint32_t flush_every = p.flush_every;
  uint32_t since_flush = 0;
  bool first_flush = true;

  // Accumulators: row A's bins C (t + T i) + A at TMEM columns [4 i + v] of the
  // warp's first 32, row B's at its next 32; bin N/2 (row 0, thread 0) in
  // registers.  v: primary ACF, secondary ACF (at the primary bin), XCF re, im.
  float acc_h[4] = {0.f, 0.f, 0.f, 0.f};

  auto add_part = [&](int bin, int v, float x) {
    const int col = v == 0 ? colP : (v == 1 ? colS : v);
    double* d = part + (size_t)col * H + bin;
    *d = (first_flush ? 0.0 : *d) + (double)x;
  };
  auto bin_acc = [&](int bin, const float2* qp, float2 pv, float2 rt, float* a) {
    const bool inov = (unsigned)(bin - ovs) < (unsigned)ov;
    if (want_acf && (!ov_only || inov)) a[0] = fmaf(pv.x, pv.x, fmaf(pv.y, pv.y, a[0]));
    if (inov) {
      const float2 qv = *qp;
      if (want_acf) a[1] = fmaf(qv.x, qv.x, fmaf(qv.y, qv.y, a[1]));
      if (want_xcf) {
        float2 x = cmulc(pv, qv);
        x.y *= xconj;
        a[2] = fmaf(x.x, rt.x, fmaf(-x.y, rt.y, a[2]));
        a[3] = fmaf(x.x, rt.y, fmaf(x.y, rt.x, a[3]));
      }
    }
  };
  // the secondary spectra: row A's at XB[0 .. M/2], row B's at XB[M/2 + 1 ..]
  float2* QA = XB;
  float2* QB = XB + kM / 2 + 1;

  bool stopped = false;
  uint32_t phase = 0;  // staging slot parity
  for (uint64_t it = it0; it < it1; ++it) {
    const bool got = mbar_wait(bar, phase, polls);
    if (!got) raise();
    phase ^= 1u;
    const uint32_t* wP = reinterpret_cast<const uint32_t*>(stage + 128);
    const uint32_t* wS = wP + C * LP;
    const FrameInfo* fs = reinterpret_cast<const FrameInfo*>(stage);
    // a thread whose wait gave up decodes in-bounds garbage (shift 0); the
    // cluster stops after B1
    const int sP = got ? (g0 ? fs->s1 : fs->s2) : 0;
    const int sS = got ? (g0 ? fs->s2 : fs->s1) : 0;
    const int fb = (int)((it - it0) & 1u);
    if (tid == 0) finfo[fb] = *fs;  // before the refill below overwrites the slot

    // ---- 1. decode, radix-C step; rows to their owners' XA / XB
    {
      const int aP = r * CW - sP, aS = r * CW - sS;
      const int mP = aP + tid, mS = aS + tid;
      const int lwP = (mP >> lgP) - ((aP >> lgP) & ~3), lwS = (mS >> lgS) - ((aS >> lgS) & ~3);
      const bool inP = aP >= 0 && aP + CW <= kM, inS = aS >= 0 && aS + CW <= kM;
      const int cP = mP & ((32 / bitsP) - 1), cS = mS & ((32 / bitsS) - 1);
      const uint32_t tbP = (uint32_t)((mP & lsbP) << (bitsP + 2));
      // the secondary station enters odd frames negated (undone by sgn below)
      const uint32_t tbS = 2048u + (uint32_t)((((uint32_t)mS & (uint32_t)lsbS) ^ (uint32_t)(it & 1u))
                                              << (bitsS + 2));
      auto rows_out = [&](float2 (&v)[16], auto ub) {
        constexpr int ubase = decltype(ub)::value;
#pragma unroll
        for (int u = 0; u < UH; ++u) {
          float2 s[C], z[C];
#pragma unroll
          for (int c = 0; c < C; ++c) s[c] = v[u * C + c];
          dft_c<C>(s);
#pragma unroll
          for (int k = 0; k < C; ++k) z[k] = s[out_pos<C>(k)];
          twiddle<C, 0>(z, dtw(ubase + u));  // z[k] *= W_N^(m k)
          const int col = r * CW + tid + kT * (ubase + u);
#pragma unroll
          for (int k = 0; k < C; ++k) {
            float2* dst = pr_is_a<C>(k) ? XA : XB;
            if (pr_owner<C>(k) == r) dst[col] = z[k];
            else cl_st(cl_map(dst + col, (uint32_t)pr_owner<C>(k)), z[k]);
          }
        }
      };
      float2 v[16];
      cl_station<C, CW, 0, UH, 2, false>(bitsP, splitP, wP, smem, mP, lwP, pos[cP], tbP, inP, v);
      cl_station<C, CW, 0, UH, 2, true>(bitsS, splitS, wS, smem, mS, lwS, pos[32 + cS], tbS, inS, v);
      cl_wait();  // B0: every CTA of the cluster has read its row buffers of the last frame
      rows_out(v, std::integral_constant<int, 0>{});
      cl_station<C, CW, UH, UH, 2, false>(bitsP, splitP, wP, smem, mP, lwP, pos[cP], tbP, inP, v);
      cl_station<C, CW, UH, UH, 2, true>(bitsS, splitS, wS, smem, mS, lwS, pos[32 + cS], tbS, inS,
                                         v);
      rows_out(v, std::integral_constant<int, UH>{});
    }
    cl_arrive();  // B1: the rows are in their owners' buffers
    int nshP = 0, nshS = 0;
    if (tid < 32 && it + 1 < it1) shifts(it + 1, &nshP, &nshS);
    cl_wait();
    if (*reinterpret_cast<volatile int*>(flag)) {  // raised before B1 by any CTA: cluster-uniform
      stopped = true;
      break;
    }
    // every thread of this CTA is past its decode: refill the slot
    if (tid < 32 && it + 1 < it1) {
      fence_proxy_async();
      issue(it + 1, nshP, nshS);
    }

    // ---- 2. row A: XA -> Y (first pass), then Y <-> XA, spectrum in Y
    {
      float2 v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = XA[tid + kT * q];
      dft16(v);
      float2* dst = Y + 17 * tid;  // cpad(16 t + q) = 17 t + q
#pragma unroll
      for (int q = 0; q < 16; ++q) dst[q] = v[out_pos<16>(q)];
    }
    fft_rest<kM, true>(Y, XA, tid, tw);  // result in Y, unpadded
    __syncthreads();
    // ---- row B: XB -> XA (first pass), then XA <-> XB, spectrum in XA
    {
      float2 v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = XB[tid + kT * q];
      dft16(v);
      float2* dst = XA + 17 * tid;
#pragma unroll
      for (int q = 0; q < 16; ++q) dst[q] = v[out_pos<16>(q)];
    }
    fft_rest<kM, true>(XA, XB, tid, tw);  // result in XA, unpadded
    __syncthreads();

    // ---- 3./4. per row: two-for-one split from the CTA's own spectra, the
    // secondary spectra to their primary bins' slots (same row: the band
    // shift is a multiple of C), then the accumulation into TMEM.  Rounding
    // in the shared complex FFT leaks a fixed fraction (~1e-6) of each
    // station's spectrum into the other's; the secondary's odd-frame negation
    // (undone by sgn) makes it alternate in sign and cancel over frames.
    const float sgn = (it & 1u) ? -1.0f : 1.0f;
    const FrameInfo& F = finfo[fb];
    const bool flush_now = ++since_flush >= flush_every;
    float sn, cs;
    __sincosf((float)(C * kT) * F.dphi, &sn, &cs);
    const float2 rstep = make_float2(cs, sn);
    if constexpr (C == 2) {
      // Slot of primary bin kp's secondary spectrum: with both rows in the CTA,
      // bin kp is row kp mod 2 at index kp / 2 (any band shift).
      auto q_slot = [&](int kp) -> float2* {
        return ((kp & 1) ? QB : QA) + (kp >> 1);
      };
      // split: the row's primary spectrum into prim, its secondary spectra into
      // their primary bins' slots.
      // row: 0 = A (spectrum in Y, mirror in XA; row 0 is its own mirror),
      //      1 = B (spectrum in XA, mirror in Y; row C/2 is its own mirror)
      auto split_row = [&](auto rb, float2 (&prim)[kJ], float2& prim_h) {
        constexpr int RB = decltype(rb)::value;
        const int row = RB ? rowB : rowA;
        // the rows' last radix-16 pass outputs (unpadded): Z[j] = Yo[j] + W^j Yo[j + M/2];
        // the mirror row's upper half Z[c + M/2] = Ym[c] - W^c Ym[c + M/2] with
        // W^c = -conj(W^(M/2 - c)), folded here instead of a radix-2 pass in place
        const float2* Yo = RB ? XA : Y;
        const float2* Ym = RB ? (r == 0 ? XA : Y) : (r == 0 ? Y : XA);
        constexpr bool kSelf0Row = RB == 0;  // row 0 (CTA 0's row A) mirrors at M - j
#pragma unroll
        for (int i = 0; i < kJ; ++i) {
          const int j = tid + kT * i;
          float2 wj, wj1;  // W_M^j = W_M^t W_16^i, W_M^(j+1) = W_M^(t+1) W_16^i
          switch (i) {  // compile-time after unrolling
            case 0: wj = tw.w[Geom<kM>::P16]; wj1 = wb1; break;
            case 1: wj = mul_w16<1>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<1>(wb1); break;
            case 2: wj = mul_w16<2>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<2>(wb1); break;
            case 3: wj = mul_w16<3>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<3>(wb1); break;
            case 4: wj = mul_w16<4>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<4>(wb1); break;
            case 5: wj = mul_w16<5>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<5>(wb1); break;
            case 6: wj = mul_w16<6>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<6>(wb1); break;
            default: wj = mul_w16<7>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<7>(wb1); break;
          }
          const float2 u = cadd(Yo[j], cmul(wj, Yo[j + kM / 2]));  // Z[j]
          // Z[N - k], k = C j + row: the mirror row's index M - 1 - j (row 0: M - j)
          const bool self0 = kSelf0Row && r == 0;
          const int c = self0 ? ((kM / 2 - j) & (kM / 2 - 1)) : kM / 2 - 1 - j;
          float2 w = cadd(Ym[c], cmulc(Ym[c + kM / 2], self0 ? wj : wj1));
          if (self0 && j == 0) w = u;  // bin 0 pairs with itself
          prim[i] = make_float2(u.x + w.x, u.y - w.y);
          const int kp = C * j + row - qoff;
          if ((unsigned)(kp - ovs) < (unsigned)ov)
            *q_slot(kp) = make_float2(sgn * (u.y + w.y), sgn * (w.x - u.x));
        }
        if (RB == 0 && half) {  // Z[N/2] = Y[0] - Y[M/2] pairs with itself
          const float2 u = csub(Y[0], Y[kM / 2]);
          prim_h = make_float2(2.f * u.x, 0.f);
          const int kp = N / 2 - qoff;
          if ((unsigned)(kp - ovs) < (unsigned)ov)
            *q_slot(kp) = make_float2(sgn * 2.f * u.y, 0.f);
        }
      };
      // accumulation of a row's bins into TMEM (its secondary spectra in place)
      auto acc_row = [&](auto rb, const float2 (&prim)[kJ], float2 prim_h) {
        constexpr int RB = decltype(rb)::value;
        const int row = RB ? rowB : rowA;
        const float2* Q = RB ? QB : QA;
        // fringe x ramp rotation of the thread's bins of this row
        __sincosf(fmaf((float)(C * tid + row - ovs), F.dphi, F.phi0), &sn, &cs);
        float2 rot = cmul(F.fr_mix, make_float2(cs, sn));
        float2 rhalf = make_float2(0.f, 0.f);
        if (RB == 0 && half) {
          __sincosf(fmaf((float)(N / 2 - ovs), F.dphi, F.phi0), &sn, &cs);
          rhalf = cmul(F.fr_mix, make_float2(cs, sn));
        }
        float t[32];
        tmem_ld32(taddr + (uint32_t)(32 * RB), t);
#pragma unroll
        for (int i = 0; i < kJ; ++i) {
          const int j = tid + kT * i;
          bin_acc(C * j + row, Q + j, prim[i], rot, &t[4 * i]);
          rot = cmul(rot, rstep);
        }
        if (RB == 0 && half) bin_acc(N / 2, Q + kM / 2, prim_h, rhalf, acc_h);
        if (flush_now) {
#pragma unroll
          for (int i = 0; i < kJ; ++i)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              add_part(C * (tid + kT * i) + row, v, t[4 * i + v]);
              t[4 * i + v] = 0.f;
            }
          if (RB == 0 && half)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              add_part(N / 2, v, acc_h[v]);
              acc_h[v] = 0.f;
            }
        }
        tmem_st32(taddr + (uint32_t)(32 * RB), t);
      };
      const std::integral_constant<int, 0> kRowA{};
      const std::integral_constant<int, 1> kRowB{};
      // both rows in this CTA, an odd band shift: each row's secondary
      // spectra land in the other row's slots, so both splits come first.
      // Row A's split reads Y only and row B's XA only: row A's primary
      // spectrum waits in Y while row B is split.
      float2 prim[kJ], prim_h = make_float2(0.f, 0.f), unused = prim_h;
      split_row(kRowA, prim, prim_h);
      __syncthreads();  // every thread has read Y
#pragma unroll
      for (int i = 0; i < kJ; ++i) Y[tid + kT * i] = prim[i];
      split_row(kRowB, prim, unused);
      __syncthreads();  // both rows' secondary spectra are in place
      acc_row(kRowB, prim, unused);
#pragma unroll
      for (int i = 0; i < kJ; ++i) prim[i] = Y[tid + kT * i];
      acc_row(kRowA, prim, prim_h);
    } else {
      // one row at a time (split, then accumulate), so that one row's primary
      // spectrum is live at a time: these kernels run at the register limit.
      // row: 0 = A (spectrum in Y, mirror in XA; row 0 is its own mirror),
      //      1 = B (spectrum in XA, mirror in Y; row C/2 is its own mirror)
      auto row_pass = [&](auto rb) {
        constexpr int RB = decltype(rb)::value;
        const int row = RB ? rowB : rowA;
        // the rows' last radix-16 pass outputs (unpadded): Z[j] = Yo[j] + W^j Yo[j + M/2];
        // the mirror row's upper half Z[c + M/2] = Ym[c] - W^c Ym[c + M/2] with
        // W^c = -conj(W^(M/2 - c)), folded here instead of a radix-2 pass in place
        const float2* Yo = RB ? XA : Y;
        const float2* Ym = RB ? (r == 0 ? XA : Y) : (r == 0 ? Y : XA);
        constexpr bool kSelf0Row = RB == 0;  // row 0 (CTA 0's row A) mirrors at M - j
        float2* Q = RB ? QB : QA;
        float2 prim[kJ];
#pragma unroll
        for (int i = 0; i < kJ; ++i) {
          const int j = tid + kT * i;
          float2 wj, wj1;  // W_M^j = W_M^t W_16^i, W_M^(j+1) = W_M^(t+1) W_16^i
          switch (i) {  // compile-time after unrolling
            case 0: wj = tw.w[Geom<kM>::P16]; wj1 = wb1; break;
            case 1: wj = mul_w16<1>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<1>(wb1); break;
            case 2: wj = mul_w16<2>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<2>(wb1); break;
            case 3: wj = mul_w16<3>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<3>(wb1); break;
            case 4: wj = mul_w16<4>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<4>(wb1); break;
            case 5: wj = mul_w16<5>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<5>(wb1); break;
            case 6: wj = mul_w16<6>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<6>(wb1); break;
            default: wj = mul_w16<7>(tw.w[Geom<kM>::P16]); wj1 = mul_w16<7>(wb1); break;
          }
          const float2 u = cadd(Yo[j], cmul(wj, Yo[j + kM / 2]));  // Z[j]
          // Z[N - k], k = C j + row: the mirror row's index M - 1 - j (row 0: M - j)
          const bool self0 = kSelf0Row && r == 0;
          const int c = self0 ? ((kM / 2 - j) & (kM / 2 - 1)) : kM / 2 - 1 - j;
          float2 w = cadd(Ym[c], cmulc(Ym[c + kM / 2], self0 ? wj : wj1));
          if (self0 && j == 0) w = u;  // bin 0 pairs with itself
          prim[i] = make_float2(u.x + w.x, u.y - w.y);
          const int kp = C * j + row - qoff;
          if ((unsigned)(kp - ovs) < (unsigned)ov)
            Q[j + dq] = make_float2(sgn * (u.y + w.y), sgn * (w.x - u.x));
        }
        float2 prim_h = make_float2(0.f, 0.f);
        if (RB == 0 && half) {  // Z[N/2] = Y[0] - Y[M/2] pairs with itself
          const float2 u = csub(Y[0], Y[kM / 2]);
          prim_h = make_float2(2.f * u.x, 0.f);
          const int kp = N / 2 - qoff;
          if ((unsigned)(kp - ovs) < (unsigned)ov) Q[kM / 2 + dq] = make_float2(sgn * 2.f * u.y, 0.f);
        }
        // fringe x ramp rotation of the thread's bins of this row
        __sincosf(fmaf((float)(C * tid + row - ovs), F.dphi, F.phi0), &sn, &cs);
        float2 rot = cmul(F.fr_mix, make_float2(cs, sn));
        float2 rhalf = make_float2(0.f, 0.f);
        if (RB == 0 && half) {
          __sincosf(fmaf((float)(N / 2 - ovs), F.dphi, F.phi0), &sn, &cs);
          rhalf = cmul(F.fr_mix, make_float2(cs, sn));
        }
        __syncthreads();  // this row's secondary spectra are in place
        float t[32];
        tmem_ld32(taddr + (uint32_t)(32 * RB), t);
#pragma unroll
        for (int i = 0; i < kJ; ++i) {
          const int j = tid + kT * i;
          bin_acc(C * j + row, Q + j, prim[i], rot, &t[4 * i]);
          rot = cmul(rot, rstep);
        }
        if (RB == 0 && half) bin_acc(N / 2, Q + kM / 2, prim_h, rhalf, acc_h);
        if (flush_now) {
#pragma unroll
          for (int i = 0; i < kJ; ++i)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              add_part(C * (tid + kT * i) + row, v, t[4 * i + v]);
              t[4 * i + v] = 0.f;
            }
          if (RB == 0 && half)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
              add_part(N / 2, v, acc_h[v]);
              acc_h[v] = 0.f;
            }
        }
        tmem_st32(taddr + (uint32_t)(32 * RB), t);
      };
      row_pass(std::integral_constant<int, 0>{});
      row_pass(std::integral_constant<int, 1>{});
    }
    if (flush_now) {
      first_flush = false;
      since_flush = 0;
    }
    cl_arrive();  // B0: this CTA's row buffers are read
  }
  if (!stopped) cl_wait();  // the last B0
  // the remaining sums (every bin written at least once)
  if (since_flush > 0 || first_flush) {
#pragma unroll
    for (int rb = 0; rb < 2; ++rb) {
      float t[32];
      tmem_ld32(taddr + (uint32_t)(32 * rb), t);
      const int row = rb ? rowB : rowA;
#pragma unroll
      for (int i = 0; i < kJ; ++i)
#pragma unroll
        for (int v = 0; v < 4; ++v) add_part(C * (tid + kT * i) + row, v, t[4 * i + v]);
    }
    if (half)
#pragma unroll
      for (int v = 0; v < 4; ++v) add_part(N / 2, v, acc_h[v]);
  }
  // no CTA leaves while a peer may still address its shared memory
  cl_sync();
  // after a stop: never leave a bulk copy in flight into this CTA's shared
  // memory (the stopping frame's copies, if its wait gave up)
  if (stopped && tid == 0) mbar_wait(bar, phase ^ 1u, polls);
  // free the tensor memory
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                 "r"(kTmemCols)
                 : "memory");
  }
}

template <int C>
cudaError_t pair_prepare() {
  return cudaFuncSetAttribute(corr_pair_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kPrMaxSmem);
}

template <int C>
int pair_capacity() {
  static std::atomic<int> cached{-1};
  int v = cached.load(std::memory_order_relaxed);
  if (v >= 0) return v;
  if (pair_prepare<C>() != cudaSuccess) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((C / 2) * 64, 1, 1);
  cfg.blockDim = dim3(kT, 1, 1);
  cfg.dynamicSmemBytes = kPrMaxSmem;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, corr_pair_kernel<C>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  cached.store(n, std::memory_order_relaxed);
  return n;
}

}  // namespace

// FFT 32768 / 65536: band shifts that are a multiple of C.  FFT 16384 (C = 2,
// both rows in one CTA): odd band shifts, where the two-row kernel does not
// apply (an even shift keeps each bin's secondary spectrum in its own row).
bool corr_pair_supported(uint32_t n, const CorrParams& p) {
  const int c = n == 16384 ? 2 : (n == 32768 ? 4 : (n == 65536 ? 8 : 0));
  if (c == 0 || p.st[0].bits > 2 || p.st[1].bits > 2) return false;
  if (c == 2 ? ((p.a2s - p.a1s) & 1) == 0 : ((p.a2s - p.a1s) % c) != 0) return false;
  return corr_pair_capacity(n) > 0;
}

int corr_pair_capacity(uint32_t n) {
  return n == 16384 ? pair_capacity<2>()
                    : (n == 32768 ? pair_capacity<4>() : (n == 65536 ? pair_capacity<8>() : 0));
}

int corr_pair_count(uint32_t n, uint64_t nf) {
  const int cap = corr_pair_capacity(n);
  if (cap <= 0) return 0;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(nf, (uint64_t)cap));
}

cudaError_t launch_corr_pair(uint32_t n, const CorrParams& p, int clusters, cudaStream_t s) {
  const int bp = p.st[p.grid == 0 ? 0 : 1].bits, bs = p.st[p.grid == 0 ? 1 : 0].bits;
  cudaError_t e;
  if (n == 16384) {
    if ((e = pair_prepare<2>()) != cudaSuccess) return e;
    corr_pair_kernel<2><<<clusters, kT, pr_smem_bytes(2, bp, bs), s>>>(p);
  } else if (n == 32768) {
    if ((e = pair_prepare<4>()) != cudaSuccess) return e;
    corr_pair_kernel<4><<<2 * clusters, kT, pr_smem_bytes(4, bp, bs), s>>>(p);
  } else if (n == 65536) {
    if ((e = pair_prepare<8>()) != cudaSuccess) return e;
    corr_pair_kernel<8><<<4 * clusters, kT, pr_smem_bytes(8, bp, bs), s>>>(p);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fxc
