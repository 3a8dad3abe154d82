// corr_cluster.cu — correlation for FFT 16384 .. 65536 (N = C * M, M = 8192,
// C in {2, 4, 8}) by one thread-block cluster of C CTAs per frame pair, the
// CTAs exchanging through distributed shared memory.
//
// Same contract as corr_fold_kernel and the four-step path's acc_global_kernel
// (src/main.rs:2491-2568 per frame pair; f64 partials [cluster][4][H] reduced
// by reduce_partials_kernel).  The N-point complex FFT of z = x_p + i x_s (the
// primary station, on whose bins the products are indexed, in the real part
// as in the FFT-8192 kernel) is one radix-C decimation-in-frequency step and C
// FFTs of M points:
//   y_q[m] = W_N^(m q) sum_c z[m + M c] W_C^(c q),   Z[C k + q] = FFT_M(y_q)[k].
// CTA q of a cluster (its rank) owns row q and the bins C j + q, j < M/2
// (row 0 also bin N/2), with their accumulators in registers across frames:
//   1. CTA r decodes the columns m in [r M/C, (r+1) M/C) of all C segments of
//      both stations from its own staged words (bulk copies of the words of
//      those columns only, so every sample is decoded once per cluster), forms
//      the radix-C butterflies and the twiddles W_N^(m q) in registers and
//      stores y_q[m] into CTA q's row buffer;                    cluster barrier
//   2. each CTA runs the M-point FFT of its row in its own shared memory (the
//      radix-16 Stockham passes of the FFT-8192 kernel; the trailing radix-2
//      pass in registers);
//   3. the two-for-one split at bin k = C j + q needs Z[N - k], which lies in
//      row C - q (row q itself for q = 0 and q = C/2) at index M - 1 - j (row
//      0: M - j): every CTA stores the upper half of its row into the mirror
//      row's CTA;                                                 cluster barrier
//   4. the secondary station's spectrum at bin k goes to the CTA that owns the
//      primary bin k - shift (the CTA itself when the band shift is a multiple
//      of C: then a CTA barrier is enough);                        cluster barrier
//   5. ACF / XCF of the CTA's bins into f32 registers, flushed to the
//      cluster's f64 partials every flush_every frames.
// Every CTA of a cluster takes the same frames and the same barriers.  A
// bounded staging wait that gives up raises the error flag of every CTA of the
// cluster before the first barrier, so all of them stop after it together.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "cluster_frame.cuh"
#include "decode_tables.cuh"
#include "fxc_device.cuh"
#include "fxc_kernels.h"

namespace fxc {
namespace {

using clu::kM;
using clu::kT;
using namespace clu;
constexpr int kJ = kM / 2 / kT;    // bins per thread (8)

// Shared memory (bytes): the decode tables [0, kTabEnd) with the frame
// records, mbarriers and the cluster error flag in their gap [4352, 4608);
// then the row buffer X (written by the cluster's decoders, then the second
// FFT pass's output), Y (first and third passes' output, then the secondary
// spectra of the CTA's bins), the mirror half row, and two staging slots
// [FrameInfo (128 B)][primary regions][secondary regions].  Region c of a
// station holds the words of segment c's columns of this CTA.
constexpr uint32_t kClFi = 4352, kClBar = 4448, kClFlag = 4464;
constexpr uint32_t kClBuf = (uint32_t)Geom<kM>::CSTRIDE * (uint32_t)sizeof(float2);
constexpr uint32_t kClX = kTabEnd;
constexpr uint32_t kClY = kClX + kClBuf;
constexpr uint32_t kClMir = kClY + kClBuf;
constexpr uint32_t kClStage0 = kClMir + (kM / 2) * (uint32_t)sizeof(float2);
constexpr uint32_t kClMaxSmem = 232448;  // 227 KB per CTA on sm_100
static_assert(kClFi + 2 * kFiBytes <= kClBar && kClFlag + 4 <= kTabLut, "records fit the gap");
static_assert(kClX % 128 == 0 && kClStage0 % 128 == 0, "alignment");

// Words of one staged region: the CTA's M/C columns of a segment
// (cluster_frame.cuh).
__host__ __device__ constexpr int cl_region_words(int c, int bits) {
  return region_words(kM / c, bits);
}
__host__ __device__ inline uint32_t cl_stage_stride(int c, int bits_p, int bits_s) {
  return (128u + 4u * (uint32_t)c *
                     (uint32_t)(cl_region_words(c, bits_p) + cl_region_words(c, bits_s)) +
          127u) & ~127u;
}
__host__ __device__ inline uint32_t cl_smem_bytes(int c, int bits_p, int bits_s) {
  return kClStage0 + 2u * cl_stage_stride(c, bits_p, bits_s);
}
static_assert(kClStage0 + 2 * ((128 + 4 * 2 * 2 * (kM / 8 + 4) + 127) & ~127) <= kClMaxSmem,
              "8-bit stations fit");

template <int C>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(kT, 1)
    corr_cluster_kernel(const __grid_constant__ CorrParams p) {
  constexpr int N = C * kM, H = N / 2 + 1, U = kM / (C * kT);
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x, lane = tid & 31;
  const int q = (int)cl_rank();
  const uint32_t cid = cl_id(), ncl = cl_count();
  FrameInfo* finfo = reinterpret_cast<FrameInfo*>(smem + kClFi);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kClBar);
  int* flag = reinterpret_cast<int*>(smem + kClFlag);
  const uint32_t* pos = reinterpret_cast<const uint32_t*>(smem + kTabPos);
  const uint32_t* lut = reinterpret_cast<const uint32_t*>(smem + kTabLut);
  float2* X = reinterpret_cast<float2*>(smem + kClX);
  float2* Yb = reinterpret_cast<float2*>(smem + kClY);
  const float2* Mir = reinterpret_cast<const float2*>(smem + kClMir);
  uint8_t* stage = smem + kClStage0;

  const bool g0 = p.grid == 0;
  const StationParams& sp = p.st[g0 ? 0 : 1];
  const StationParams& ss = p.st[g0 ? 1 : 0];
  const int bitsP = sp.bits, bitsS = ss.bits;
  const bool preP = bitsP > 2 && sp.shkind != SH_IDENTITY;
  const bool preS = bitsS > 2 && ss.shkind != SH_IDENTITY;
  const int lgP = log2_spw(bitsP), lgS = log2_spw(bitsS);
  const int LP = cl_region_words(C, bitsP), LS = cl_region_words(C, bitsS);
  const uint32_t stride = cl_stage_stride(C, bitsP, bitsS);
  const uint32_t polls = p.wait_polls ? p.wait_polls : kWaitPolls;
  const bool withhold = (p.debug_flags & DBG_WITHHOLD_COPIES) != 0;
  const uint64_t it0 = ((uint64_t)cid * p.nf) / ncl, it1 = ((uint64_t)(cid + 1) * p.nf) / ncl;
  double* part = p.partials + (size_t)cid * 4 * H;

  // Frame `it`'s copies into its slot, by the lanes of warp 0: lane c < C the
  // primary's region c, lane C + c the secondary's, lane 2C the frame record.
  // Each region is clamped to the frame's words (the decode zero-fills the
  // samples outside the frame).
  auto issue = [&](uint64_t it, int shP, int shS) {
    const int slot = (int)((it - it0) & 1u);
    uint8_t* dst = stage + slot * stride;
    uint32_t bytes = 0;
    const uint8_t* src = nullptr;
    uint8_t* d = nullptr;
    if (lane < 2 * C) {
      const bool sec = lane >= C;
      const int c = sec ? lane - C : lane;
      const int lg = sec ? lgS : lgP, L = sec ? LS : LP;
      const uint32_t bpf = sec ? ss.bpf : sp.bpf;
      const int nw = (int)(bpf >> 2);
      const int a = q * (kM / C) - (sec ? shS : shP);
      const int wa = ((a >> lg) & ~3) + c * (kM >> lg);
      const int lo = max(wa, 0), hi = min(wa + L, nw);
      if (hi > lo) {
        bytes = 4u * (uint32_t)(hi - lo);
        src = (sec ? ss.raw : sp.raw) + it * bpf + 4u * (uint32_t)lo;
        d = dst + 128 + (sec ? 4 * C * LP : 0) + 4 * (c * L + lo - wa);
      }
    } else if (lane == 2 * C) {
      bytes = kFiBytes;
      src = reinterpret_cast<const uint8_t*>(p.finfo + it);
      d = dst;
    }
    const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
    if (lane == 0) mbar_expect_tx(&bars[slot], total);
    __syncwarp();
    if (bytes && !withhold) bulk_g2s(d, src, bytes, &bars[slot]);  // withheld: the wait runs out
  };
  auto shifts = [&](uint64_t it, int* shP, int* shS) {
    const FrameInfo* g = p.finfo + it;
    *shP = g0 ? g->s1 : g->s2;
    *shS = g0 ? g->s2 : g->s1;
  };

  if (tid == 0) {
    for (int s = 0; s < 2; ++s) mbar_init(&bars[s], 1);
    *flag = 0;
    fence_proxy_async();
  }
  __syncthreads();
  if (tid < 32) {
    for (uint64_t it = it0; it < it1 && it < it0 + 2; ++it) {
      int a, b;
      shifts(it, &a, &b);
      issue(it, a, b);
    }
  }
  build_decode_tables(sp, ss, preP, preS, smem, tid, kT);
  const bool splitP = split_2bit(sp), splitS = split_2bit(ss);
  Twiddles<kM> tw;
  tw.init(tid);
  // radix-C step twiddle bases W_N^m of the thread's columns m = q M/C + t + T u
  float2 dbase[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    double sn, cs;
    sincospi(-2.0 * (double)(q * (kM / C) + tid + kT * u) / (double)N, &sn, &cs);
    dbase[u] = make_float2((float)cs, (float)sn);
  }
  // every CTA of the cluster has started, zeroed its flag and built its tables
  // before any CTA stores into another's shared memory
  cl_sync();

  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s;
  const int ov = a1e - a1s;
  const int sb = a2s - a1s;
  const int ovs = g0 ? a1s : a2s;   // overlap on the primary grid: [ovs, ovs + ov)
  const int qoff = g0 ? sb : -sb;   // secondary bin = primary bin + qoff
  // the secondary spectrum at this CTA's bin k serves the primary bin k - qoff,
  // owned by CTA tq at index j + dq
  const int tq = (((q - qoff) % C) + C) % C;
  const int dq = (q - qoff - tq) / C;
  const bool qlocal = (qoff % C) == 0;  // the same for every CTA of the cluster
  const int mirror = (C - q) % C;
  const bool want_acf = (p.products & 1u) != 0;
  const bool want_xcf = (p.products & 2u) != 0;
  const bool ov_only = (p.products & 16u) != 0;
  const float xconj = g0 ? 1.0f : -1.0f;  // XCF = S1 conj(S2): conj(P conj(S)) for grid 1
  const int lsbP = sp.lsb ? 1 : 0, lsbS = ss.lsb ? 1 : 0;
  const int colP = g0 ? 0 : 1, colS = g0 ? 1 : 0;  // output columns of the two ACFs
  const bool half = q == 0 && tid == 0;            // bin N/2
  const uint32_t flush_every = p.flush_every;
  uint32_t since_flush = 0;
  bool first_flush = true;

  // acc[i]: bin C (t + T i) + q, acc[kJ]: bin N/2 (row 0, thread 0).
  // Columns: primary ACF, secondary ACF (at the primary bin), XCF re, im.
  float acc[kJ + 1][4];
#pragma unroll
  for (int i = 0; i <= kJ; ++i)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[i][v] = 0.f;

  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i <= kJ; ++i) {
      if (i == kJ && !half) continue;
      const int bin = i == kJ ? N / 2 : C * (tid + kT * i) + q;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int col = v == 0 ? colP : (v == 1 ? colS : v);
        double* d = part + (size_t)col * H + bin;
        *d = (first_flush ? 0.0 : *d) + (double)acc[i][v];
        acc[i][v] = 0.f;
      }
    }
    first_flush = false;
    since_flush = 0;
  };

  uint64_t stop = it1;  // the frame after whose first barrier the cluster stopped
  for (uint64_t it = it0; it < it1; ++it) {
    const uint32_t k_it = (uint32_t)(it - it0);
    const int slot = (int)(k_it & 1u);
    const uint32_t parity = (k_it >> 1) & 1u;
    const int fb = slot;
    // the shifts of frame it + 2, whose copies go out after the first barrier
    int nshP = 0, nshS = 0;
    if (tid < 32 && it + 2 < it1) shifts(it + 2, &nshP, &nshS);
    const bool got = mbar_wait(&bars[slot], parity, polls);
    if (!got) {
      for (int r = 0; r < C; ++r) cl_st_u32(cl_map(flag, (uint32_t)r), 1u);
      atomicOr(p.err, ERR_WAIT_TIMEOUT);
    }
    uint8_t* st = stage + slot * stride;
    uint32_t* wP = reinterpret_cast<uint32_t*>(st + 128);
    uint32_t* wS = wP + C * LP;
    const FrameInfo* fs = reinterpret_cast<const FrameInfo*>(st);
    // a thread whose wait gave up decodes in-bounds garbage (shift 0); the
    // cluster stops after the barrier below
    const int sP = got ? (g0 ? fs->s1 : fs->s2) : 0;
    const int sS = got ? (g0 ? fs->s2 : fs->s1) : 0;
    if (tid == 0) finfo[fb] = *fs;
    if (preP || preS) {  // CTA-uniform
      preshuffle_slot(wP, (uint32_t)(C * LP), preP ? sp.shkind : SH_IDENTITY, lut, wS,
                      (uint32_t)(C * LS), preS ? ss.shkind : SH_IDENTITY, lut + 1024, tid, kT);
      __syncthreads();
    }

    // ---- 1. decode, radix-C step, rows to their CTAs
    {
      float2 v[16];
      const int aP = q * (kM / C) - sP, aS = q * (kM / C) - sS;
      const int mP = aP + tid, mS = aS + tid;
      const int lwP = (mP >> lgP) - ((aP >> lgP) & ~3), lwS = (mS >> lgS) - ((aS >> lgS) & ~3);
      const bool inP = aP >= 0 && aP + kM / C <= kM, inS = aS >= 0 && aS + kM / C <= kM;
      const int cP = mP & ((32 / bitsP) - 1), cS = mS & ((32 / bitsS) - 1);
      const uint32_t tbP = (uint32_t)((mP & lsbP) << (bitsP + 2));
      // the secondary station enters odd frames negated (undone by sgn below)
      const uint32_t tbS = 2048u + (uint32_t)((((uint32_t)mS & (uint32_t)lsbS) ^ (uint32_t)(it & 1u))
                                              << (bitsS + 2));
      cl_station<C, kM / C, 0, U, 8, false>(bitsP, splitP, wP, smem, mP, lwP, pos[cP], tbP, inP, v);
      cl_station<C, kM / C, 0, U, 8, true>(bitsS, splitS, wS, smem, mS, lwS, pos[32 + cS], tbS, inS,
                                           v);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        float2 s[C], z[C];
#pragma unroll
        for (int c = 0; c < C; ++c) s[c] = v[u * C + c];
        dft_c<C>(s);
#pragma unroll
        for (int k = 0; k < C; ++k) z[k] = s[out_pos<C>(k)];
        twiddle<C, 0>(z, dbase[u]);  // z[k] *= W_N^(m k)
        const uint32_t off = (uint32_t)(q * (kM / C) + tid + kT * u) * (uint32_t)sizeof(float2);
#pragma unroll
        for (int k = 0; k < C; ++k) cl_st(cl_map(X, (uint32_t)k) + off, z[k]);
      }
    }
    cl_sync();  // B1: every row complete
    if (*reinterpret_cast<volatile int*>(flag)) {  // set before B1 by any CTA: cluster-uniform
      stop = it;
      break;
    }
    // the slot is consumed by every thread of this CTA: refill it
    if (tid < 32 && it + 2 < it1) {
      fence_proxy_async();  // the slot's generic-proxy reads before the copies' writes
      issue(it + 2, nshP, nshS);
    }

    // ---- 2. the row's FFT: first radix-16 pass from X, then the FFT-8192 passes
    {
      float2 v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = X[tid + kT * r];
      dft16(v);
      float2* dst = Yb + 17 * tid;  // cpad(16 t + r) = 17 t + r
#pragma unroll
      for (int r = 0; r < 16; ++r) dst[r] = v[out_pos<16>(r)];
    }
    const float2* Y = fft_rest<kM, true>(Yb, X, tid, tw);  // Y == Yb, unpadded
    __syncthreads();

    // ---- 3. trailing radix-2: Z[j] kept, Z[j + M/2] to the mirror row's CTA
    float2 zl[kJ];
    float2 zhalf = make_float2(0.f, 0.f);
    {
      const uint32_t maddr = cl_map(Mir, (uint32_t)mirror);
#pragma unroll
      for (int i = 0; i < kJ; ++i) {
        const int j = tid + kT * i;
        float2 wj;  // W_M^j = W_M^t W_16^i
        switch (i) {  // compile-time after unrolling
          case 0: wj = tw.w[Geom<kM>::P16]; break;
          case 1: wj = mul_w16<1>(tw.w[Geom<kM>::P16]); break;
          case 2: wj = mul_w16<2>(tw.w[Geom<kM>::P16]); break;
          case 3: wj = mul_w16<3>(tw.w[Geom<kM>::P16]); break;
          case 4: wj = mul_w16<4>(tw.w[Geom<kM>::P16]); break;
          case 5: wj = mul_w16<5>(tw.w[Geom<kM>::P16]); break;
          case 6: wj = mul_w16<6>(tw.w[Geom<kM>::P16]); break;
          default: wj = mul_w16<7>(tw.w[Geom<kM>::P16]); break;
        }
        const float2 a = Y[j], wb = cmul(wj, Y[j + kM / 2]);
        zl[i] = cadd(a, wb);
        const float2 zu = csub(a, wb);
        cl_st(maddr + (uint32_t)j * (uint32_t)sizeof(float2), zu);
        if (i == 0) zhalf = zu;  // Z[M/2]: bin N/2 of row 0
      }
    }
    cl_arrive();  // B2
    // fringe x ramp rotation of the thread's bins (while the barrier completes)
    const FrameInfo& F = finfo[fb];
    float sn, cs;
    __sincosf(fmaf((float)(C * tid + q - ovs), F.dphi, F.phi0), &sn, &cs);
    float2 rot = cmul(F.fr_mix, make_float2(cs, sn));
    __sincosf((float)(C * kT) * F.dphi, &sn, &cs);
    const float2 rstep = make_float2(cs, sn);
    float2 rhalf = make_float2(0.f, 0.f);
    if (half) {
      __sincosf(fmaf((float)(N / 2 - ovs), F.dphi, F.phi0), &sn, &cs);
      rhalf = cmul(F.fr_mix, make_float2(cs, sn));
    }
    const float sgn = (it & 1u) ? -1.0f : 1.0f;
    cl_wait();

    // ---- 4. two-for-one split; secondary spectra to the primary bins' CTA
    // Rounding in the shared complex FFT leaks a fixed fraction (~1e-6) of
    // each station's spectrum into the other's; the secondary's odd-frame
    // negation (undone by sgn) makes that leak alternate in sign and cancel.
    float2 prim[kJ];
    float2 prim_h = make_float2(0.f, 0.f);
    {
      const uint32_t qaddr = cl_map(Yb, (uint32_t)tq);
#pragma unroll
      for (int i = 0; i < kJ; ++i) {
        const int j = tid + kT * i;
        const int mi = q == 0 ? ((kM / 2 - j) & (kM / 2 - 1)) : kM / 2 - 1 - j;
        float2 w = Mir[mi];  // Z[N - k]
        if (q == 0 && j == 0) w = zl[0];  // bin 0 pairs with itself
        const float2 u = zl[i];
        // primary = real part: P[k] = Z[k] + conj Z[N-k], S[k] = -i (Z[k] - conj Z[N-k])
        prim[i] = make_float2(u.x + w.x, u.y - w.y);
        const int kp = C * j + q - qoff;
        if ((unsigned)(kp - ovs) < (unsigned)ov) {
          const float2 sv = make_float2(sgn * (u.y + w.y), sgn * (w.x - u.x));
          if (qlocal) Yb[j + dq] = sv;
          else cl_st(qaddr + (uint32_t)(j + dq) * (uint32_t)sizeof(float2), sv);
        }
      }
      if (half) {  // Z[N/2] pairs with itself
        prim_h = make_float2(2.f * zhalf.x, 0.f);
        const int kp = N / 2 - qoff;
        if ((unsigned)(kp - ovs) < (unsigned)ov) {
          const float2 sv = make_float2(sgn * 2.f * zhalf.y, 0.f);
          if (qlocal) Yb[kM / 2 + dq] = sv;
          else cl_st(qaddr + (uint32_t)(kM / 2 + dq) * (uint32_t)sizeof(float2), sv);
        }
      }
    }
    if (qlocal) __syncthreads();
    else cl_sync();  // B3

    // ---- 5. accumulation (constant indices into acc[][])
    auto bin_acc = [&](int bin, int j, float2 pv, float2 r, float* a) {
      const bool inov = (unsigned)(bin - ovs) < (unsigned)ov;
      if (want_acf && (!ov_only || inov)) a[0] = fmaf(pv.x, pv.x, fmaf(pv.y, pv.y, a[0]));
      if (inov) {
        const float2 qv = Yb[j];
        if (want_acf) a[1] = fmaf(qv.x, qv.x, fmaf(qv.y, qv.y, a[1]));
        if (want_xcf) {
          float2 x = cmulc(pv, qv);
          x.y *= xconj;
          a[2] = fmaf(x.x, r.x, fmaf(-x.y, r.y, a[2]));
          a[3] = fmaf(x.x, r.y, fmaf(x.y, r.x, a[3]));
        }
      }
    };
#pragma unroll
    for (int i = 0; i < kJ; ++i) {
      const int j = tid + kT * i;
      bin_acc(C * j + q, j, prim[i], rot, acc[i]);
      rot = cmul(rot, rstep);
    }
    if (half) bin_acc(N / 2, kM / 2, prim_h, rhalf, acc[kJ]);
    if (++since_flush >= flush_every) flush();
  }
  if (since_flush > 0 || first_flush) flush();
  // no CTA leaves while a peer may still address its shared memory
  cl_sync();
  // after a stop: never leave a bulk copy in flight into this CTA's shared
  // memory (frame `stop` and the next one may have copies outstanding)
  if (stop < it1 && tid == 0) {
    for (uint64_t it = stop; it < it1 && it < stop + 2; ++it) {
      const uint32_t k_it = (uint32_t)(it - it0);
      mbar_wait(&bars[k_it & 1u], (k_it >> 1) & 1u, polls);
    }
  }
}

template <int C>
cudaError_t cluster_prepare() {
  return cudaFuncSetAttribute(corr_cluster_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)cl_smem_bytes(C, 8, 8));
}

// Clusters of C CTAs that fit the GPU at once with the largest layout (cached:
// the value depends only on the kernel and the device type).
template <int C>
int cluster_capacity() {
  static std::atomic<int> cached{-1};
  int v = cached.load(std::memory_order_relaxed);
  if (v >= 0) return v;
  if (cluster_prepare<C>() != cudaSuccess) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C * 64, 1, 1);
  cfg.blockDim = dim3(kT, 1, 1);
  cfg.dynamicSmemBytes = cl_smem_bytes(C, 8, 8);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, corr_cluster_kernel<C>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  cached.store(n, std::memory_order_relaxed);
  return n;
}

}  // namespace

int corr_cluster_size(uint32_t n) { return n == 16384 ? 2 : (n == 32768 ? 4 : (n == 65536 ? 8 : 0)); }

int corr_cluster_capacity(uint32_t n) {
  switch (corr_cluster_size(n)) {
    case 2: return cluster_capacity<2>();
    case 4: return cluster_capacity<4>();
    case 8: return cluster_capacity<8>();
    default: return 0;
  }
}

int corr_cluster_count(uint32_t n, uint64_t nf) {
  const int cap = corr_cluster_capacity(n);
  if (cap <= 0) return 0;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(nf, (uint64_t)cap));
}

cudaError_t launch_corr_cluster(uint32_t n, const CorrParams& p, int clusters, cudaStream_t s) {
  const int c = corr_cluster_size(n);
  const int bp = p.st[p.grid == 0 ? 0 : 1].bits, bs = p.st[p.grid == 0 ? 1 : 0].bits;
  const uint32_t smem = cl_smem_bytes(c, bp, bs);
  cudaError_t e;
  switch (c) {
    case 2:
      if ((e = cluster_prepare<2>()) != cudaSuccess) return e;
      corr_cluster_kernel<2><<<2 * clusters, kT, smem, s>>>(p);
      break;
    case 4:
      if ((e = cluster_prepare<4>()) != cudaSuccess) return e;
      corr_cluster_kernel<4><<<4 * clusters, kT, smem, s>>>(p);
      break;
    case 8:
      if ((e = cluster_prepare<8>()) != cudaSuccess) return e;
      corr_cluster_kernel<8><<<8 * clusters, kT, smem, s>>>(p);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fxc
