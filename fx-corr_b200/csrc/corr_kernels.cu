// corr_kernels.cu — the fused FX-correlation kernel for sm_100a.
//
// frame_info_kernel evaluates the FP64 per-frame delay model
// (src/main.rs:184-241) for every frame of a sector, one thread per frame, into
// 48-byte FrameInfo records.
//
// corr_kernel: one CTA processes a contiguous run of frame pairs of a sector.
// Per frame pair (stations 1 and 2 share one complex FFT: z = x1 + i*x2):
//   1. the frame's FrameInfo and the packed .raw words of both stations arrive
//      in shared memory by cp.async.bulk (TMA bulk copy) tracked by an
//      mbarrier, two stages deep;
//   2. decode: 32-bit word shuffle, b-bit codes -> f32 levels, LSB->USB flip of
//      odd samples (src/utils.rs:215-376);
//   3. the first radix-16 pass reads the decoded planes with the integer shift
//      and zero fill (src/utils.rs:126-145); the remaining Stockham passes run
//      in padded shared memory;
//   4. two-for-one split of Z into S1, S2 (the two real FFTs,
//      src/utils.rs:47-59), band alignment, fringe x phase-ramp rotation and
//      |S|^2 / S1 conj(S2) accumulation (src/main.rs:2491-2568) into per-thread
//      f32 registers, flushed every 32 frames into per-CTA f64 partials;
// reduce_partials_kernel then sums the per-CTA partials in a fixed order.
// The frame loop is corr_span: the single-sector kernel runs it once per CTA
// over the CTA's share of the sector, the batched kernel (corr_batch_kernel)
// once per work item taken by ticket from a list spanning many scans, with
// batch_frame_info_kernel and batch_reduce_kernel on either side.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fxc_device.cuh"
#include "fxc_kernels.h"

namespace fxc {

// Per-CTA setup of corr_kernel: mbarriers, error flag, twiddle chains.
template <int N, int FPC>
__device__ __forceinline__ void corr_cta_init(const SmemLayout& L, uint8_t* smem, Twiddles<N>& tw) {
  constexpr int T1 = N / 16;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);
  int* flag = reinterpret_cast<int*>(smem + L.off_flag);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
    *flag = 0;
    fence_proxy_async();
  }
  tw.init(threadIdx.x % T1);
}

__device__ __forceinline__ void corr_cta_drain(const SmemLayout& L, uint8_t* smem) {
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);
  const int* flag = reinterpret_cast<const int*>(smem + L.off_flag);
  // never leave a bulk copy in flight into a finished CTA's shared memory
  if (threadIdx.x == 0 && *flag) {
    for (int s = 0; s < kStages; ++s) mbar_wait(&bars[s], 0, kWaitPolls);
  }
}

// Iterations [it0, it1) (FPC frame pairs each, frames below fend) of the
// sector described by p; MODE_CORR accumulates into the f64 partials at part
// ([4][H]).  seq counts the staging iterations this CTA consumed before (the
// mbarrier slot and phase).  Returns false when a bounded wait gave up.
template <int N, int FPC, int MODE>
__device__ __forceinline__ bool corr_span(const CorrParams& p, uint64_t it0, uint64_t it1,
                                          uint64_t fend, double* part, uint8_t* smem,
                                          const SmemLayout& L, const Twiddles<N>& tw,
                                          uint32_t& seq, uint32_t flush_every) {
  constexpr int T1 = N / 16;
  constexpr int T = FPC * T1;
  constexpr int H = N / 2 + 1;
  constexpr int BPT = (N / 2) / T;
  static_assert(BPT * T == N / 2 && BPT >= 2, "bins per thread");

  float2* bufA = reinterpret_cast<float2*>(smem + L.off_a);
  float2* bufB = reinterpret_cast<float2*>(smem + L.off_b);
  uint8_t* stage = smem + L.off_stage;
  uint32_t* lut = reinterpret_cast<uint32_t*>(smem + L.off_lut);
  float* lv = reinterpret_cast<float*>(smem + L.off_lv);
  FrameInfo* finfo = reinterpret_cast<FrameInfo*>(smem + L.off_fi);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);
  int* flag = reinterpret_cast<int*>(smem + L.off_flag);

  const int tid = threadIdx.x;
  const int g = tid / T1;  // frame slot of this thread in an iteration
  const int t = tid % T1;  // thread index within its frame pair
  const uint32_t seq0 = seq;

  const uint32_t bpf1 = p.st[0].bpf, bpf2 = p.st[1].bpf;
  const uint8_t* raw1 = p.st[0].raw;
  const uint8_t* raw2 = p.st[1].raw;
  const FrameInfo* gfi = p.finfo;
  constexpr uint32_t kRaw1 = FPC * kFiBytes;  // offset of station 1 bytes in a slot

  auto issue = [&](uint64_t it) {
    const int slot = (int)((seq0 + (uint32_t)(it - it0)) % kStages);
    const uint64_t f0 = it * FPC;
    const uint64_t nvalid = (fend - f0) < (uint64_t)FPC ? (fend - f0) : (uint64_t)FPC;
    const uint32_t bf = (uint32_t)(nvalid * kFiBytes);
    const uint32_t b1 = (uint32_t)(nvalid * bpf1), b2 = (uint32_t)(nvalid * bpf2);
    uint8_t* dst = stage + slot * L.stage_stride;
    mbar_expect_tx(&bars[slot], bf + b1 + b2);
    bulk_g2s(dst, gfi + f0, bf, &bars[slot]);
    bulk_g2s(dst + kRaw1, raw1 + f0 * bpf1, b1, &bars[slot]);
    bulk_g2s(dst + kRaw1 + FPC * bpf1, raw2 + f0 * bpf2, b2, &bars[slot]);
  };
  // The previous span, if any, is past its last decode and its last
  // iteration's barriers: the staging ring and the tables are free.  The
  // first iterations' copies go out first, the tables are built meanwhile.
  __syncthreads();
  if (tid == 0) {
    fence_proxy_async();
    for (uint64_t it = it0; it < it1 && it < it0 + kStages; ++it) issue(it);
  }
  for (int i = tid; i < 512; i += T) lv[i] = p.st[i >> 8].levels[i & 255] * p.st[i >> 8].scale;
  for (int s = 0; s < 2; ++s)
    if (p.st[s].shkind == SH_GENERIC)
      for (int i = tid; i < 1024; i += T) lut[s * 1024 + i] = p.st[s].shlut[i];
  __syncthreads();

  float acc[BPT + 1][4];
#pragma unroll
  for (int i = 0; i <= BPT; ++i)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[i][v] = 0.f;
  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s;
  const int ov = a1e - a1s;
  const int sb = a2s - a1s;
  const int a_gs = p.grid == 0 ? a1s : a2s;  // grid start of the overlap
  const bool want_acf = (p.products & 1u) != 0;
  const bool want_xcf = (p.products & 2u) != 0;
  const bool ov_only = (p.products & 16u) != 0;
  uint32_t* err = p.err;
  bool first_flush = true;
  uint32_t since_flush = 0;

  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i <= BPT; ++i) {
      const int bin = (i < BPT) ? (tid + T * i) : N / 2;
      if (i == BPT && tid != 0) continue;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        double* q = part + (size_t)v * H + bin;
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
    const uint64_t frame_local = it * FPC + g;
    const bool valid = frame_local < fend;

    if (!mbar_wait(&bars[slot], parity, kWaitPolls)) {
      atomicOr(flag, 1);
      atomicOr(err, ERR_WAIT_TIMEOUT);
    }
    uint8_t* st = stage + slot * L.stage_stride;
    uint32_t* w1 = reinterpret_cast<uint32_t*>(st + kRaw1);
    uint32_t* w2 = reinterpret_cast<uint32_t*>(st + kRaw1 + FPC * bpf1);
    // non-identity 32-bit shuffles are applied once, in place, to the staged words
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
    // MODE_CORR: station 2 enters odd frames negated, undone in the
    // accumulation, so that the shared FFT's cross-station rounding leak
    // alternates in sign and cancels over frames instead of biasing the XCF
    const PackedStation pb{w2 + g * (bpf2 / 4), lv + 256, (uint32_t)p.st[1].bits,
                           (1u << p.st[1].bits) - 1u, p.st[1].lsb ? 1 : 0, s2,
                           MODE == MODE_CORR ? (uint32_t)(frame_local & 1u) : 0u};

    if constexpr (MODE == MODE_DECODE) {
      if (valid) {
        float* o1 = p.out_a + frame_local * N;
        float* o2 = p.out_b + frame_local * N;
        const float u1 = 1.0f / p.st[0].scale, u2 = 1.0f / p.st[1].scale;  // exact
        for (int n = t; n < N; n += T1) {
          const int m1 = n - s1, m2 = n - s2;
          o1[n] = ((unsigned)m1 < (unsigned)N) ? packed_sample(pa, m1) * u1 : 0.f;
          o2[n] = ((unsigned)m2 < (unsigned)N) ? packed_sample(pb, m2) * u2 : 0.f;
        }
      }
      __syncthreads();
      if (tid == 0 && it + kStages < it1) {
        fence_proxy_async();
        issue(it + kStages);
      }
      continue;
    }

    float2* za = bufA + g * Geom<N>::CSTRIDE;
    float2* zb = bufB + g * Geom<N>::CSTRIDE;
    first_pass_packed<N>(pa, pb, za, t);
    float2* Z0 = fft_rest<N>(za, zb, t, tw);
    // fft_rest opened with a barrier after the fused first pass: the staging
    // slot is consumed, refill it with iteration it + kStages
    if (tid == 0 && it + kStages < it1) {
      fence_proxy_async();
      issue(it + kStages);
    }
    // the final buffer sits at the same offset for every frame slot
    const bool fin_b = Z0 != za;
    __syncthreads();

    if constexpr (MODE == MODE_SPECTRA) {
      if (valid) {
        float2* o1 = reinterpret_cast<float2*>(p.out_a) + frame_local * H;
        float2* o2 = reinterpret_cast<float2*>(p.out_b) + frame_local * H;
        const float u1 = 0.5f / p.st[0].scale, u2 = 0.5f / p.st[1].scale;  // exact
        for (int k = t; k < H; k += T1) {
          const float2 a = Z0[k], b = Z0[(N - k) & (N - 1)];
          o1[k] = make_float2(u1 * (a.x + b.x), u1 * (a.y - b.y));
          o2[k] = make_float2(u2 * (a.y + b.y), -u2 * (a.x - b.x));
        }
      }
      __syncthreads();
      continue;
    }

    // ---- MODE_CORR: accumulate every valid frame of the iteration
#pragma unroll 1
    for (int f = 0; f < FPC; ++f) {
      if (it * FPC + f >= fend) break;
      const float2* Z = (fin_b ? bufB : bufA) + f * Geom<N>::CSTRIDE;
      const FrameInfo& F = finfo[f];
      // Ramp rotation of owned bin tid + T*i: SFU sin/cos (|angle| <= ~pi,
      // absolute error < 4e-7) at i = 0 and i = BPT/2, short recurrences between.
      float sn, cs;
      __sincosf(fmaf((float)(tid - a_gs), F.dphi, F.phi0), &sn, &cs);
      float2 rot = cmul(F.fr_mix, make_float2(cs, sn));
      __sincosf(fmaf((float)(tid + T * (BPT / 2) - a_gs), F.dphi, F.phi0), &sn, &cs);
      const float2 rot_half = cmul(F.fr_mix, make_float2(cs, sn));
      __sincosf((float)T * F.dphi, &sn, &cs);
      const float2 rstep = make_float2(cs, sn);
      const float sg = ((it * FPC + f) & 1u) ? -1.0f : 1.0f;  // station 2 sign of this frame
      auto bin_acc = [&](int bin, float2 r, float* a) {
        const float2 u = Z[bin], w = Z[(N - bin) & (N - 1)];
        if (p.grid == 0) {
          const bool inov = bin >= a1s && bin < a1e;
          const float2 p1 = make_float2(u.x + w.x, u.y - w.y);  // 2*S1[bin]
          if (want_acf && (!ov_only || inov)) a[0] += cnorm2(p1);
          if (inov) {
            const int i2 = bin + sb;
            const float2 c = Z[i2], d = Z[(N - i2) & (N - 1)];
            const float2 q2 = make_float2(sg * (c.y + d.y), sg * (d.x - c.x));  // 2*S2[i2]
            if (want_acf) a[1] += cnorm2(q2);
            if (want_xcf) {
              const float2 x = cmul(cmulc(p1, q2), r);
              a[2] += x.x;
              a[3] += x.y;
            }
          }
        } else {
          const bool inov = bin >= a2s && bin < a2s + ov;
          const float2 p2 = make_float2(sg * (u.y + w.y), sg * (w.x - u.x));  // 2*S2[bin]
          if (want_acf && (!ov_only || inov)) a[1] += cnorm2(p2);
          if (inov) {
            const int i1 = bin - sb;
            const float2 c = Z[i1], d = Z[(N - i1) & (N - 1)];
            const float2 q1 = make_float2(c.x + d.x, c.y - d.y);  // 2*S1[i1]
            if (want_acf) a[0] += cnorm2(q1);
            if (want_xcf) {
              const float2 x = cmul(cmulc(q1, p2), r);
              a[2] += x.x;
              a[3] += x.y;
            }
          }
        }
      };
#pragma unroll
      for (int i = 0; i < BPT; ++i) {
        if (i == BPT / 2) rot = rot_half;
        bin_acc(tid + T * i, rot, acc[i]);
        rot = cmul(rot, rstep);
      }
      if (tid == 0) {
        __sincosf(fmaf((float)(N / 2 - a_gs), F.dphi, F.phi0), &sn, &cs);
        bin_acc(N / 2, cmul(F.fr_mix, make_float2(cs, sn)), acc[BPT]);
      }
    }
    if (++since_flush >= flush_every) flush();
    __syncthreads();
  }
  if constexpr (MODE == MODE_CORR) {
    if (ok && (since_flush > 0 || first_flush)) flush();
  }
  seq = seq0 + (uint32_t)(it1 - it0);
  return ok;
}

template <int N, int FPC, int MODE>
__global__ void __launch_bounds__(FPC * N / 16, (N >= 8192 ? 1 : 2))
corr_kernel(const CorrParams p) {
  constexpr int H = N / 2 + 1;
  extern __shared__ __align__(128) uint8_t smem[];
  const SmemLayout L = smem_layout<N, FPC>(p.stage_bytes);
  Twiddles<N> tw;
  corr_cta_init<N, FPC>(L, smem, tw);
  // ---- this CTA's iterations (FPC frame pairs each)
  const uint64_t iters = (p.nf + FPC - 1) / FPC;
  const uint64_t it0 = (blockIdx.x * iters) / gridDim.x;
  const uint64_t it1 = ((blockIdx.x + 1) * iters) / gridDim.x;
  uint32_t seq = 0;
  corr_span<N, FPC, MODE>(p, it0, it1, p.nf, p.partials + (size_t)blockIdx.x * 4 * H, smem, L, tw,
                          seq, p.flush_every);
  corr_cta_drain(L, smem);
}

// Batched: a persistent grid takes the items of batch group `grp` by ticket;
// every item is a frame range of one scan's sector (frames aligned to FPC)
// with its own partials.  The layout is sized for the largest stage (8-bit
// stations), so one launch serves every bit depth.
template <int N, int FPC, int MINB>
__global__ void __launch_bounds__(FPC * N / 16, MINB) corr_batch_kernel(const BatchArgs a, int grp) {
  extern __shared__ __align__(128) uint8_t smem[];
  const SmemLayout L = smem_layout<N, FPC>(2u * FPC * N);
  uint32_t* ticket = reinterpret_cast<uint32_t*>(smem + L.off_flag + 4);
  Twiddles<N> tw;
  corr_cta_init<N, FPC>(L, smem, tw);
  const uint32_t n_items = a.hdr->nitems[grp];
  const BatchItem* items = a.hdr->items + a.hdr->item0[grp];
  const BatchScan* scans = a.hdr->scans;
  uint32_t seq = 0;
  for (;;) {
    if (threadIdx.x == 0) *ticket = atomicAdd(&a.hdr->ticket[grp], 1u);
    __syncthreads();
    const uint32_t k = *ticket;  // corr_span opens with a barrier before the next write
    if (k >= n_items) break;
    const BatchItem w = items[k];
    // f32 accumulators flushed every 32 frames, whatever the variant
    if (!corr_span<N, FPC, MODE_CORR>(scans[w.scan].p, w.f0 / FPC, (w.f1 + FPC - 1) / FPC, w.f1,
                                      a.partials + w.part, smem, L, tw, seq, 32u / FPC))
      break;
  }
  corr_cta_drain(L, smem);
}

// Fixed-order sum of the per-CTA partials.  The multipliers (exact powers of
// two) undo the two-for-one 2x factor of each spectrum and the per-station
// level scaling.  Writes acf11, acf22, xcf (re,im) and zeroes the phased slot.
// A 256-thread block covers 32 bins: each of its 8 warps sums one contiguous
// eighth of the slots in slot order (coalesced 256-byte rows), then the eight
// warp sums are added in warp order; the order depends only on nblk, so the
// result is deterministic.
constexpr int kRedBins = 32, kRedGroups = 8;

__global__ void __launch_bounds__(kRedBins * kRedGroups)
reduce_partials_kernel(const double* __restrict__ part, int nblk, int h, double m11, double m22,
                       double m12, double* __restrict__ out) {
  __shared__ double sm[kRedGroups][4][kRedBins];
  const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
  const int k = blockIdx.x * kRedBins + lane;
  const int b0 = (nblk * grp) / kRedGroups, b1 = (nblk * (grp + 1)) / kRedGroups;
  double s[4] = {0, 0, 0, 0};
  if (k < h) {
    for (int b = b0; b < b1; ++b) {
      const double* q = part + (size_t)b * 4 * h + k;
#pragma unroll
      for (int v = 0; v < 4; ++v) s[v] += q[(size_t)v * h];
    }
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) sm[grp][v][lane] = s[v];
  __syncthreads();
  if (grp != 0 || k >= h) return;
  double t[4] = {0, 0, 0, 0};
#pragma unroll
  for (int g = 0; g < kRedGroups; ++g)
#pragma unroll
    for (int v = 0; v < 4; ++v) t[v] += sm[g][v][lane];
  out[k] = m11 * t[0];
  out[h + k] = m22 * t[1];
  out[2 * h + 2 * k] = m12 * t[2];
  out[2 * h + 2 * k + 1] = m12 * t[3];
  out[4 * h + k] = 0.0;
}

__global__ void delay_entries_kernel(const DelayParams p, uint64_t first, uint64_t nf,
                                     fxc_frame_delay_dev* out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  int64_t i1, i2;
  double f1, f2;
  float2 l1, l2;
  frame_delay(p, first + i, &i1, &i2, &f1, &f2, &l1, &l2);
  fxc_frame_delay_dev d;
  d.int1 = i1;
  d.int2 = i2;
  d.frac1 = f1;
  d.frac2 = f2;
  d.fr_lo1[0] = l1.x;
  d.fr_lo1[1] = l1.y;
  d.fr_lo2[0] = l2.x;
  d.fr_lo2[1] = l2.y;
  out[i] = d;
}

__global__ void frame_info_kernel(const DelayParams p, uint64_t first, uint64_t nf, int n,
                                  double df_hz, int a1s, int a2s, FrameInfo* out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  FrameInfo fi;
  frame_info(p, first + i, n, df_hz, a1s, a2s, &fi);
  out[i] = fi;
}

// Last sector of the batch whose first frame (bins = false) or first bin
// (bins = true) is <= x; sectors are numbered in ascending order of both.
__device__ __forceinline__ uint32_t batch_find(const BatchScan* sc, uint32_t n, uint64_t x,
                                               bool bins) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t m = (lo + hi) >> 1;
    const uint64_t st = bins ? sc[m].bin0 : sc[m].fi0;
    if (st <= x) lo = m;
    else hi = m;
  }
  return lo;
}

// Frame records of every sector of a batch (grid-stride over all frames);
// also rearms the groups' tickets for the launches that follow.
__global__ void batch_frame_info_kernel(const BatchArgs a) {
  const uint32_t ns = a.hdr->nscans;
  const uint64_t total = a.hdr->nframes;
  if (blockIdx.x == 0 && threadIdx.x < kBatchGroups) a.hdr->ticket[threadIdx.x] = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += stride) {
    const BatchScan& b = a.hdr->scans[batch_find(a.hdr->scans, ns, x, false)];
    const uint64_t i = x - b.fi0;
    FrameInfo fi;
    frame_info(b.p.dl, b.p.first_frame + i, (int)b.n, b.p.df_hz, b.p.a1s, b.p.a2s, &fi);
    const_cast<FrameInfo*>(b.p.finfo)[i] = fi;
  }
}

// Fixed-order sum of each sector's item partials (grid-stride over all bins
// of the batch), with the same multipliers and output layout as
// reduce_partials_kernel (a phased sector: its power in [4H, 5H), the
// correlation columns zero, as reduce_phased_kernel after a zeroed block).
__global__ void batch_reduce_kernel(const BatchArgs a) {
  const uint32_t ns = a.hdr->nscans;
  const uint64_t total = a.hdr->nbins;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += stride) {
    const BatchScan& b = a.hdr->scans[batch_find(a.hdr->scans, ns, x, true)];
    const uint64_t k = x - b.bin0;
    const uint64_t h = b.h;
    const double* q = a.partials + b.part + k;
    double* out = b.acc;
    if (b.phased) {
      // phased power: H partials per item, summed in item order
      double t = 0.0;
      for (uint32_t i = 0; i < b.nparts; ++i, q += h) t += *q;
      out[k] = 0.0;
      out[h + k] = 0.0;
      out[2 * h + 2 * k] = 0.0;
      out[2 * h + 2 * k + 1] = 0.0;
      out[4 * h + k] = t;
      continue;
    }
    double s[4] = {0, 0, 0, 0};
    for (uint32_t i = 0; i < b.nparts; ++i, q += 4 * h) {
#pragma unroll
      for (int v = 0; v < 4; ++v) s[v] += q[(size_t)v * h];
    }
    out[k] = b.m11 * s[0];
    out[h + k] = b.m22 * s[1];
    out[2 * h + 2 * k] = b.m12 * s[2];
    out[2 * h + 2 * k + 1] = b.m12 * s[3];
    out[4 * h + k] = 0.0;
  }
}

// ------------------------------------------------------------- launchers

template <int N, int FPC, int MODE>
static cudaError_t launch_one(const CorrParams& p, int grid, cudaStream_t stream) {
  const SmemLayout L = smem_layout<N, FPC>(p.stage_bytes);
  auto kern = corr_kernel<N, FPC, MODE>;
  // the limit is shared by every host thread: always the largest layout
  // (8-bit stations), never lowered under a concurrent launch
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_layout<N, FPC>(2u * FPC * N).total);
  if (e != cudaSuccess) return e;
  kern<<<grid, FPC * N / 16, L.total, stream>>>(p);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_mode(uint32_t n, const CorrParams& p, int grid, cudaStream_t s) {
  switch (n) {
    case 1024: return launch_one<1024, 4, MODE>(p, grid, s);
    case 2048: return launch_one<2048, 2, MODE>(p, grid, s);
    case 4096: return launch_one<4096, 1, MODE>(p, grid, s);
    case 8192:
      // the FFT-8192 correlation has a kernel of its own (corr_fold.cu)
      if constexpr (MODE == MODE_CORR) return launch_corr_fold(p, grid, s);
      else return launch_one<8192, 1, MODE>(p, grid, s);
    case 16384:
      // FFT 16384 as two 8192-point rows (corr_fold.cu); other modes and odd
      // band shifts take the four-step path (large_kernels.cu)
      if constexpr (MODE == MODE_CORR) return launch_corr_fold2(p, grid, s);
      else return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
  }
}

int corr_frames_per_cta_iter(uint32_t n) {
  return n == 1024 ? 4 : (n == 2048 ? 2 : 1);
}

int corr_ctas_per_sm(uint32_t n) { return n >= 8192 ? 1 : 2; }

cudaError_t launch_corr(uint32_t n, int mode, const CorrParams& p, int grid, cudaStream_t s) {
  if (mode == MODE_CORR) return launch_mode<MODE_CORR>(n, p, grid, s);
  if (mode == MODE_SPECTRA) return launch_mode<MODE_SPECTRA>(n, p, grid, s);
  return launch_mode<MODE_DECODE>(n, p, grid, s);
}

// ------------------------------------------------------- batched launchers

namespace {

// Variants of the batched kernels: FFT length, frames per CTA iteration and
// resident CTAs per SM (shared memory with 8-bit staging: FPC*N = 1024 ->
// 32 KB, 2048 -> 54 KB, 4096 -> 95 KB, 8192 -> 183 KB).
template <int N, int FPC>
constexpr int batch_minb() {
  return FPC * N <= 1024 ? 6 : (FPC * N <= 2048 ? 4 : (FPC * N <= 4096 ? 2 : 1));
}

template <int N, int FPC>
uint32_t batch_smem() {
  return smem_layout<N, FPC>(2u * FPC * N).total;
}

template <int N, int FPC>
cudaError_t batch_prepare_one() {
  return cudaFuncSetAttribute(corr_batch_kernel<N, FPC, batch_minb<N, FPC>()>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_smem<N, FPC>());
}

template <int N, int FPC>
int batch_ctas_one() {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, corr_batch_kernel<N, FPC, batch_minb<N, FPC>()>,
                                                    FPC * N / 16, batch_smem<N, FPC>()) != cudaSuccess)
    return 0;
  return nb;
}

template <int N, int FPC>
cudaError_t batch_launch_one(const BatchArgs& a, int grp, int grid, cudaStream_t s) {
  corr_batch_kernel<N, FPC, batch_minb<N, FPC>()><<<grid, FPC * N / 16, batch_smem<N, FPC>(), s>>>(a, grp);
  return cudaGetLastError();
}

// Calls f.template operator()<N, FPC>() for the variant (g, fpc); returns
// cudaErrorInvalidValue for a variant that does not exist.
#define FXC_BATCH_VARIANTS(g, fpc, CALL)              \
  switch ((g) * 16 + (fpc)) {                         \
    case BG_1024 * 16 + 1: return CALL(1024, 1);      \
    case BG_1024 * 16 + 2: return CALL(1024, 2);      \
    case BG_1024 * 16 + 4: return CALL(1024, 4);      \
    case BG_2048 * 16 + 1: return CALL(2048, 1);      \
    case BG_2048 * 16 + 2: return CALL(2048, 2);      \
    case BG_2048 * 16 + 4: return CALL(2048, 4);      \
    case BG_4096 * 16 + 1: return CALL(4096, 1);      \
    case BG_4096 * 16 + 2: return CALL(4096, 2);      \
    default: break;                                   \
  }

}  // namespace

uint32_t fold_batch_smem_bytes(int rows);
cudaError_t prepare_fold_batch(int rows);
cudaError_t launch_fold_batch(int rows, const BatchArgs& a, int grp, int grid, cudaStream_t s);
int fold_batch_ctas_per_sm(int rows);

cudaError_t batch_prepare(int g, int fpc) {
  if (g == BG_8192 || g == BG_16384) return prepare_fold_batch(g == BG_8192 ? 1 : 2);
#define FXC_PREP(N, F) batch_prepare_one<N, F>()
  FXC_BATCH_VARIANTS(g, fpc, FXC_PREP)
#undef FXC_PREP
  return cudaErrorInvalidValue;
}

int batch_group_ctas_per_sm(int g, int fpc) {
  if (g == BG_8192 || g == BG_16384) return fold_batch_ctas_per_sm(g == BG_8192 ? 1 : 2);
#define FXC_CTAS(N, F) batch_ctas_one<N, F>()
  FXC_BATCH_VARIANTS(g, fpc, FXC_CTAS)
#undef FXC_CTAS
  return 0;
}

cudaError_t launch_batch_group(int g, int fpc, const BatchArgs& a, int grid, cudaStream_t s) {
  if (grid <= 0) return cudaErrorInvalidValue;
  if (g == BG_8192 || g == BG_16384) return launch_fold_batch(g == BG_8192 ? 1 : 2, a, g, grid, s);
#define FXC_LAUNCH(N, F) batch_launch_one<N, F>(a, g, grid, s)
  FXC_BATCH_VARIANTS(g, fpc, FXC_LAUNCH)
#undef FXC_LAUNCH
  return cudaErrorInvalidValue;
}

cudaError_t launch_batch_frame_info(const BatchArgs& a, int grid, cudaStream_t s) {
  batch_frame_info_kernel<<<grid, 128, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_batch_reduce(const BatchArgs& a, int grid, cudaStream_t s) {
  batch_reduce_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const double* part, int nblk, int h, double m11, double m22, double m12,
                          double* out, cudaStream_t s) {
  reduce_partials_kernel<<<(h + kRedBins - 1) / kRedBins, kRedBins * kRedGroups, 0, s>>>(
      part, nblk, h, m11, m22, m12, out);
  return cudaGetLastError();
}

cudaError_t launch_delay_entries(const DelayParams& p, uint64_t first, uint64_t nf,
                                 fxc_frame_delay_dev* out, cudaStream_t s) {
  if (nf == 0) return cudaSuccess;
  delay_entries_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(p, first, nf, out);
  return cudaGetLastError();
}

cudaError_t launch_frame_info(const DelayParams& p, uint64_t first, uint64_t nf, int n,
                              double df_hz, int a1s, int a2s, FrameInfo* out, cudaStream_t s) {
  if (nf == 0) return cudaSuccess;
  frame_info_kernel<<<(unsigned)((nf + 127) / 128), 128, 0, s>>>(p, first, nf, n, df_hz, a1s,
                                                                   a2s, out);
  return cudaGetLastError();
}

}  // namespace fxc
