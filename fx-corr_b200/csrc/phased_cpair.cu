// phased_cpair.cu — phased-array synthesis for FFT 32768 and 65536
// (yi-phasedarray, src/main.rs:2222-2412) with 1- and 2-bit stations and a
// band shift that is a multiple of C = N / 8192: one thread-block cluster of
// C/2 CTAs per frame pair, CTA r owning the mirror rows r and C - r (CTA 0:
// rows 0 and C/2), as in the correlation pair kernel (corr_pair.cu).
//
// Per frame pair:
//   1. forward: the pair kernel's decode, radix-C decimation in frequency
//      across the cluster and two row FFTs per CTA (z = x1 + i x2, station 2
//      negated on odd frames); Z[C j + q] = Z_q[j];
//   2. per bin of the CTA's two rows: both stations' spectra (two-for-one, the
//      mirror row being the CTA's other row), each rotated by its fractional
//      delay with the Nyquist imaginary part zeroed and multiplied by its
//      fringe phasor; the band-aligned secondary term of an output bin lies in
//      the same row (the shift is a multiple of C); cb = w1 a1 + w2 a2 and
//      |cb|^2 into f32 registers (src/main.rs:2264-2280, src/utils.rs:69-124);
//   3. .raw: the inverse real FFT as the forward FFT of the Hermitian-extended
//      conj(cb) scaled by 1/N (src/utils.rs:60-66), by the same radix-C
//      decimation in frequency: the inputs x[m + M c] of column m are bins of
//      row m mod C and of its mirror, i.e. of this CTA when m mod C is one of
//      its rows, so each CTA forms the radix-C step of those columns from its
//      own spectra and stores each output row into the row's owner; two
//      inverse row FFTs per CTA give the samples n = C k + q of its rows, each
//      re-quantised with ant1's levels (odd samples negated when both inputs
//      are LSB) into its bits of the packed output words, which the CTAs of
//      the cluster OR together in global memory (zeroed first) after ant1's
//      output shuffle, a bit permutation (src/utils.rs:378-410).
// Four cluster barriers per frame: after the forward rows are stored (B1),
// before and after the inverse rows are stored (I0, I1), and once every CTA
// has read its row buffers (B0, whose wait sits after the next decode).
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <type_traits>

#include "cluster_frame.cuh"
#include "decode_tables.cuh"
#include "fxc_device.cuh"
#include "fxc_kernels.h"
#include "row_fft.cuh"

namespace fxc {
namespace {

using namespace clu;
using rows::first_pass_regs;
using rows::row_radix2;
constexpr int kJ = kM / 2 / kT;  // bins per thread and row (8)

// Shared memory (bytes): decode tables [0, 4608); the gap [4352, 4608) holds
// the frame record, the staging mbarrier, the error flag and the output
// levels; ant1's output encode LUT in [4608, 12800) (1- and 2-bit stations
// need no byte LUTs); then the row buffers XA, XB (the cluster's forward
// rows; XA then row B's spectrum, XB the secondary terms; then the inverse
// rows), Y (row A's spectrum, then cb of both rows: row A's bins at [0, M/2],
// row B's at M/2 + 1 + j) and one staging slot.
constexpr uint32_t kQpFi = 4352, kQpBar = 4400, kQpFlag = 4408, kQpQl = 4416;
constexpr uint32_t kQpEnc = kTabLut;
constexpr uint32_t kQpBuf = (uint32_t)Geom<kM>::CSTRIDE * (uint32_t)sizeof(float2);
constexpr uint32_t kQpXA = kTabEnd, kQpXB = kQpXA + kQpBuf, kQpY = kQpXB + kQpBuf;
constexpr uint32_t kQpStage = kQpY + kQpBuf;
constexpr uint32_t kQpMaxSmem = 232448;  // 227 KB per CTA on sm_100
static_assert(kQpFi + kFiBytes <= kQpBar && kQpQl + 16 * 4 <= kTabLut, "records fit the gap");

__host__ __device__ constexpr uint32_t qp_smem_bytes(int c, int bits_1, int bits_2) {
  return kQpStage + ((128u + 4u * (uint32_t)c *
                                 (uint32_t)(region_words(2 * kM / c, bits_1) +
                                            region_words(2 * kM / c, bits_2)) +
                      127u) & ~127u);
}
static_assert(qp_smem_bytes(8, 2, 2) <= kQpMaxSmem && qp_smem_bytes(4, 2, 2) <= kQpMaxSmem,
              "2-bit stations fit");

template <int C>
__host__ __device__ constexpr int qp_owner(int k) {
  return k == C / 2 ? 0 : (k < C - k ? k : C - k);
}
template <int C>
__host__ __device__ constexpr bool qp_is_a(int k) {
  return k != C / 2 && k <= C - k;
}

template <int C>
__global__ void __cluster_dims__(C / 2, 1, 1) __launch_bounds__(kT, 1)
    phased_cpair_kernel(const __grid_constant__ PhasedParams p) {
  constexpr int P = C / 2;
  constexpr int N = C * kM, H = N / 2 + 1;
  constexpr int CW = kM / P;   // forward columns per CTA (also inverse columns)
  constexpr int U = CW / kT;   // column groups per thread
  constexpr int UH = 16 / C;   // column groups per decode half
  constexpr int MC = kM / C;   // inverse columns per row
  static_assert(U == 2 * UH && MC % kT == 0, "shapes");
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x, lane = tid & 31;
  const int r = (int)cl_rank();
  const int rowA = r, rowB = r == 0 ? C / 2 : C - r;
  const uint32_t cid = cl_id(), ncl = cl_count();
  FrameInfo* finfo = reinterpret_cast<FrameInfo*>(smem + kQpFi);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kQpBar);
  int* flag = reinterpret_cast<int*>(smem + kQpFlag);
  float* ql = reinterpret_cast<float*>(smem + kQpQl);
  uint32_t* elut = reinterpret_cast<uint32_t*>(smem + kQpEnc);
  const uint32_t* pos = reinterpret_cast<const uint32_t*>(smem + kTabPos);
  float2* XA = reinterpret_cast<float2*>(smem + kQpXA);
  float2* XB = reinterpret_cast<float2*>(smem + kQpXB);
  float2* Y = reinterpret_cast<float2*>(smem + kQpY);
  uint8_t* stage = smem + kQpStage;

  const StationParams& s1 = p.st[0];
  const StationParams& s2 = p.st[1];
  const int bits1 = s1.bits, bits2 = s2.bits;
  const int lg1 = log2_spw(bits1), lg2 = log2_spw(bits2);
  const int L1 = region_words(CW, bits1), L2 = region_words(CW, bits2);
  const uint64_t it0 = ((uint64_t)cid * p.nf) / ncl, it1 = ((uint64_t)(cid + 1) * p.nf) / ncl;
  double* part = p.partials + (size_t)cid * H;

  // Frame `it`'s copies into the staging slot (lanes of warp 0): lane c < C
  // station 1's region c, C + c station 2's, 2C the frame record.
  auto issue = [&](uint64_t it, int sh1, int sh2) {
    uint32_t bytes = 0;
    const uint8_t* src = nullptr;
    uint8_t* d = nullptr;
    if (lane < 2 * C) {
      const bool two = lane >= C;
      const int c = two ? lane - C : lane;
      const int lg = two ? lg2 : lg1, L = two ? L2 : L1;
      const uint32_t bpf = two ? s2.bpf : s1.bpf;
      const int nw = (int)(bpf >> 2);
      const int a = r * CW - (two ? sh2 : sh1);
      const int wa = ((a >> lg) & ~3) + c * (kM >> lg);
      const int lo = max(wa, 0), hi = min(wa + L, nw);
      if (hi > lo) {
        bytes = 4u * (uint32_t)(hi - lo);
        src = (two ? s2.raw : s1.raw) + it * bpf + 4u * (uint32_t)lo;
        d = stage + 128 + (two ? 4 * C * L1 : 0) + 4 * (c * L + lo - wa);
      }
    } else if (lane == 2 * C) {
      bytes = kFiBytes;
      src = reinterpret_cast<const uint8_t*>(p.finfo + it);
      d = stage;
    }
    const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
    if (lane == 0) mbar_expect_tx(bar, total);
    __syncwarp();
    if (bytes) bulk_g2s(d, src, bytes, bar);
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
  __syncthreads();
  if (tid < 32 && it0 < it1) {
    const FrameInfo* g = p.finfo + it0;
    issue(it0, g->s1, g->s2);
  }
  build_decode_tables(s1, s2, false, false, smem, tid, kT);
  for (int i = tid; i < 16; i += kT) ql[i] = i < (int)p.nqlevels ? p.qlevels[i] : 0.f;
  for (int i = tid; i < 1024; i += kT) elut[i] = p.enc_lut[i];
  const bool split1 = split_2bit(s1), split2 = split_2bit(s2);
  Twiddles<kM> tw;
  tw.init(tid);
  cl_sync();
  cl_arrive();  // B0 of the frame before the first

  const int a1s = p.a1s, a1e = p.a1e, a2s = p.a2s;
  const int ov = a1e - a1s, sb = a2s - a1s;
  const bool g0 = p.grid == 0;
  const int ovs = g0 ? a1s : a2s;   // overlap on the output grid: [ovs, ovs + ov)
  const int qoff = g0 ? sb : -sb;   // the other station's bin = output bin + qoff
  const int dq = -qoff / C;
  const int sp = g0 ? 0 : 1;        // the station on the output grid
  const float u1 = 0.5f / s1.scale, u2 = 0.5f / s2.scale;
  const int lsb1 = s1.lsb ? 1 : 0, lsb2 = s2.lsb ? 1 : 0;
  const bool half = r == 0 && tid == 0;  // bin N/2 (row 0, index M/2)
  const uint32_t spw = 32u / p.bits_out, wpf = (uint32_t)N / spw;
  const uint32_t qmask = (1u << p.bits_out) - 1u;
  const float inv_n = 1.0f / (float)N;
  float2* QA = XB;
  float2* QB = XB + kM / 2 + 1;

  // acc[2 i + b]: row b's bin C (t + T i) + row; acc[2 kJ]: bin N/2
  float acc[2 * kJ + 1];
#pragma unroll
  for (int i = 0; i <= 2 * kJ; ++i) acc[i] = 0.f;
  bool first_flush = true;
  uint32_t since_flush = 0;
  auto bin_of = [&](int i) { return C * (tid + kT * (i >> 1)) + ((i & 1) ? rowB : rowA); };
  auto flush = [&]() {
#pragma unroll
    for (int i = 0; i <= 2 * kJ; ++i) {
      if (i == 2 * kJ && !half) continue;
      double* d = part + (i == 2 * kJ ? N / 2 : bin_of(i));
      *d = (first_flush ? 0.0 : *d) + (double)acc[i];
      acc[i] = 0.f;
    }
    first_flush = false;
    since_flush = 0;
  };
  // cb of a bin of this CTA's rows (Y after the synthesis)
  auto cb_at = [&](int k) -> float2 {
    const int row = k % C;
    return row == rowA ? Y[(k - rowA) / C] : Y[kM / 2 + 1 + (k - rowB) / C];
  };

  bool stopped = false;
  uint32_t phase = 0;
  for (uint64_t it = it0; it < it1; ++it) {
    const bool got = mbar_wait(bar, phase, kWaitPolls);
    if (!got) raise();
    phase ^= 1u;
    const uint32_t* w1 = reinterpret_cast<const uint32_t*>(stage + 128);
    const uint32_t* w2 = w1 + C * L1;
    const FrameInfo* fs = reinterpret_cast<const FrameInfo*>(stage);
    const int sh1 = got ? fs->s1 : 0, sh2 = got ? fs->s2 : 0;
    if (tid == 0) *finfo = *fs;  // before the refill overwrites the slot

    // ---- 1. forward: decode, radix-C step, rows to their owners
    {
      const int a1 = r * CW - sh1, a2 = r * CW - sh2;
      const int m1 = a1 + tid, m2 = a2 + tid;
      const int lw1 = (m1 >> lg1) - ((a1 >> lg1) & ~3), lw2 = (m2 >> lg2) - ((a2 >> lg2) & ~3);
      const bool in1 = a1 >= 0 && a1 + CW <= kM, in2 = a2 >= 0 && a2 + CW <= kM;
      const int c1 = m1 & ((32 / bits1) - 1), c2 = m2 & ((32 / bits2) - 1);
      const uint32_t tb1 = (uint32_t)((m1 & lsb1) << (bits1 + 2));
      const uint32_t tb2 = 2048u + (uint32_t)((((uint32_t)m2 & (uint32_t)lsb2) ^ (uint32_t)(it & 1u))
                                              << (bits2 + 2));
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
          const int col = r * CW + tid + kT * (ubase + u);
          float sn, cs;  // W_N^col (col / N exact in f32)
          sincospif(-2.0f * (float)col / (float)N, &sn, &cs);
          twiddle<C, 0>(z, make_float2(cs, sn));
#pragma unroll
          for (int k = 0; k < C; ++k) {
            float2* dst = qp_is_a<C>(k) ? XA : XB;
            if (qp_owner<C>(k) == r) dst[col] = z[k];
            else cl_st(cl_map(dst + col, (uint32_t)qp_owner<C>(k)), z[k]);
          }
        }
      };
      float2 v[16];
      cl_station<C, CW, 0, UH, 2, false>(bits1, split1, w1, smem, m1, lw1, pos[c1], tb1, in1, v);
      cl_station<C, CW, 0, UH, 2, true>(bits2, split2, w2, smem, m2, lw2, pos[32 + c2], tb2, in2, v);
      cl_wait();  // B0
      rows_out(v, std::integral_constant<int, 0>{});
      cl_station<C, CW, UH, UH, 2, false>(bits1, split1, w1, smem, m1, lw1, pos[c1], tb1, in1, v);
      cl_station<C, CW, UH, UH, 2, true>(bits2, split2, w2, smem, m2, lw2, pos[32 + c2], tb2, in2,
                                         v);
      rows_out(v, std::integral_constant<int, UH>{});
    }
    cl_arrive();  // B1
    int nsh1 = 0, nsh2 = 0;
    if (tid < 32 && it + 1 < it1) {
      const FrameInfo* g = p.finfo + it + 1;
      nsh1 = g->s1;
      nsh2 = g->s2;
    }
    cl_wait();
    if (*reinterpret_cast<volatile int*>(flag)) {
      stopped = true;
      break;
    }
    if (tid < 32 && it + 1 < it1) {
      fence_proxy_async();
      issue(it + 1, nsh1, nsh2);
    }

    // ---- forward row FFTs: row A in Y, row B in XA
    {
      float2 v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = XA[tid + kT * q];
      first_pass_regs(v, Y, tid);
    }
    fft_rest<kM, true>(Y, XA, tid, tw);
    __syncthreads();
    row_radix2(Y, tid, tw);
    {
      float2 v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = XB[tid + kT * q];
      first_pass_regs(v, XA, tid);
    }
    fft_rest<kM, true>(XA, XB, tid, tw);
    __syncthreads();
    row_radix2(XA, tid, tw);
    __syncthreads();

    // ---- 2. synthesis per bin
    const FrameInfo& F = *finfo;
    const float sg = (it & 1u) ? -1.0f : 1.0f;
    auto station = [&](float2 u, float2 w, int k, int s) -> float2 {
      float2 v = s == 0 ? make_float2(u1 * (u.x + w.x), u1 * (u.y - w.y))
                        : make_float2(sg * u2 * (u.y + w.y), sg * u2 * (w.x - u.x));
      float sn, cs;
      __sincosf((float)k * (s == 0 ? F.st1 : F.st2), &sn, &cs);
      v = cmul(v, make_float2(cs, sn));
      if (k == N / 2) v.y = 0.f;
      return cmul(v, s == 0 ? F.fr_lo1 : F.fr_lo2);
    };
    float2 prim[2 * kJ + 1];
#pragma unroll
    for (int i = 0; i < 2 * kJ; ++i) {
      const int b = i & 1, j = tid + kT * (i >> 1), k = bin_of(i);
      float2 u, w;
      if (b == 0) {
        u = Y[j];
        w = r == 0 ? Y[(kM - j) & (kM - 1)] : XA[kM - 1 - j];
      } else {
        u = XA[j];
        w = r == 0 ? XA[kM - 1 - j] : Y[kM - 1 - j];
      }
      prim[i] = station(u, w, k, sp);
      const int kp = k - qoff;
      if ((unsigned)(kp - ovs) < (unsigned)ov) (b ? QB : QA)[j + dq] = station(u, w, k, 1 - sp);
    }
    prim[2 * kJ] = make_float2(0.f, 0.f);
    if (half) {  // Z[N/2] pairs with itself
      const float2 u = Y[kM / 2];
      prim[2 * kJ] = station(u, u, N / 2, sp);
      const int kp = N / 2 - qoff;
      if ((unsigned)(kp - ovs) < (unsigned)ov) QA[kM / 2 + dq] = station(u, u, N / 2, 1 - sp);
    }
    __syncthreads();  // the secondary terms are in place; the spectra are read
    auto combine = [&](int bb, float2 pv, const float2* qp) -> float2 {
      float2 sv = make_float2(0.f, 0.f);
      if ((unsigned)(bb - ovs) < (unsigned)ov) sv = *qp;
      const float2 a1 = g0 ? pv : sv, a2 = g0 ? sv : pv;
      return make_float2(a1.x * p.w1 + a2.x * p.w2, a1.y * p.w1 + a2.y * p.w2);
    };
#pragma unroll
    for (int i = 0; i < 2 * kJ; ++i) {
      const int b = i & 1, j = tid + kT * (i >> 1), bb = bin_of(i);
      float2 cb = combine(bb, prim[i], (b ? QB : QA) + j);
      acc[i] += cnorm2(cb);
      if (bb == 0) cb.y = 0.f;
      Y[b ? kM / 2 + 1 + j : j] = cb;
    }
    if (half) {
      float2 cb = combine(N / 2, prim[2 * kJ], QA + kM / 2);
      acc[2 * kJ] += cnorm2(cb);
      cb.y = 0.f;
      Y[kM / 2] = cb;
    }
    if (++since_flush >= p.flush_every) flush();

    if (p.want_raw) {
      // ---- 3. inverse: radix-C step of the columns m = C i + row of this
      // CTA's rows from its own cb, rows to their owners
      cl_arrive();  // I0: this CTA no longer reads XA / XB
      cl_wait();
#pragma unroll 1
      for (int u = 0; u < U; ++u) {
        const int row = (u < U / 2) ? rowA : rowB;  // MC is a multiple of T
        const int i = tid + kT * u - (u < U / 2 ? 0 : MC);
        const int m = C * i + row;
        float2 s[C], z[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
          // x[n] = conj(cb[n]) (n <= N/2), cb[N - n] (n > N/2)
          const int n = m + kM * c;
          if (n <= N / 2) {
            const float2 x = cb_at(n);
            s[c] = make_float2(x.x, -x.y);
          } else {
            s[c] = cb_at(N - n);
          }
        }
        dft_c<C>(s);
#pragma unroll
        for (int k = 0; k < C; ++k) z[k] = s[out_pos<C>(k)];
        float sn, cs;
        sincospif(-2.0f * (float)m / (float)N, &sn, &cs);
        twiddle<C, 0>(z, make_float2(cs, sn));  // z[k] *= W_N^(m k)
#pragma unroll
        for (int k = 0; k < C; ++k) {
          float2* dst = qp_is_a<C>(k) ? XA : XB;
          if (qp_owner<C>(k) == r) dst[m] = z[k];
          else cl_st(cl_map(dst + m, (uint32_t)qp_owner<C>(k)), z[k]);
        }
      }
      cl_arrive();  // I1: the inverse rows are in their owners' buffers
      cl_wait();
      // inverse row FFTs: samples C k + A in Y, C k + B in XA
      {
        float2 v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = XA[tid + kT * q];
        first_pass_regs(v, Y, tid);
      }
      fft_rest<kM, true>(Y, XA, tid, tw);
      __syncthreads();
      row_radix2(Y, tid, tw);
      {
        float2 v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = XB[tid + kT * q];
        first_pass_regs(v, XA, tid);
      }
      fft_rest<kM, true>(XA, XB, tid, tw);
      __syncthreads();
      row_radix2(XA, tid, tw);
      __syncthreads();
      // re-quantise this CTA's samples into their bits of each output word;
      // the cluster's CTAs OR their bits together (the words start at zero)
      uint32_t* out = reinterpret_cast<uint32_t*>(p.raw_out + it * p.bpf_out);
      const uint32_t per = spw / (uint32_t)C;  // samples of one row in a word
      for (uint32_t wdx = (uint32_t)tid; wdx < wpf; wdx += kT) {
        uint32_t word = 0;
        for (uint32_t i = 0; i < per; ++i) {
          const uint32_t k = wdx * per + i;  // index in the rows
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const uint32_t row = (uint32_t)(b ? rowB : rowA);
            const uint32_t n = (uint32_t)C * k + row;
            float x = (b ? XA : Y)[k].x * inv_n;
            if (p.out_lsb && (n & 1u)) x = -x;
            word |= (nearest_level(x, ql, (int)p.nqlevels, p.qmonotonic) & qmask)
                    << ((n - wdx * spw) * p.bits_out);
          }
        }
        const uint32_t sw = elut[word & 255u] | elut[256 + ((word >> 8) & 255u)] |
                            elut[512 + ((word >> 16) & 255u)] | elut[768 + (word >> 24)];
        atomicOr(out + wdx, sw);
      }
    }
    cl_arrive();  // B0: this CTA's row buffers are read
  }
  if (!stopped) cl_wait();
  if (since_flush > 0 || first_flush) flush();
  cl_sync();
  if (stopped && tid == 0) mbar_wait(bar, phase ^ 1u, kWaitPolls);
}

template <int C>
cudaError_t qp_prepare() {
  return cudaFuncSetAttribute(phased_cpair_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kQpMaxSmem);
}

template <int C>
int qp_capacity() {
  static std::atomic<int> cached{-1};
  int v = cached.load(std::memory_order_relaxed);
  if (v >= 0) return v;
  if (qp_prepare<C>() != cudaSuccess) return 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((C / 2) * 64, 1, 1);
  cfg.blockDim = dim3(kT, 1, 1);
  cfg.dynamicSmemBytes = kQpMaxSmem;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, phased_cpair_kernel<C>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  cached.store(n, std::memory_order_relaxed);
  return n;
}

}  // namespace

bool phased_cpair_supported(uint32_t n, const PhasedParams& p) {
  const int c = n == 32768 ? 4 : (n == 65536 ? 8 : 0);
  if (c == 0 || p.st[0].bits > 2 || p.st[1].bits > 2 || p.bits_out > 2) return false;
  if (((p.a2s - p.a1s) % c) != 0) return false;
  return (c == 4 ? qp_capacity<4>() : qp_capacity<8>()) > 0;
}

int phased_cpair_count(uint32_t n, uint64_t nf) {
  const int cap = n == 32768 ? qp_capacity<4>() : (n == 65536 ? qp_capacity<8>() : 0);
  if (cap <= 0) return 0;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(nf, (uint64_t)cap));
}

cudaError_t launch_phased_cpair(uint32_t n, const PhasedParams& p, int clusters, cudaStream_t s) {
  cudaError_t e;
  if (n == 32768) {
    if ((e = qp_prepare<4>()) != cudaSuccess) return e;
    phased_cpair_kernel<4><<<2 * clusters, kT, qp_smem_bytes(4, p.st[0].bits, p.st[1].bits), s>>>(p);
  } else if (n == 65536) {
    if ((e = qp_prepare<8>()) != cudaSuccess) return e;
    phased_cpair_kernel<8><<<4 * clusters, kT, qp_smem_bytes(8, p.st[0].bits, p.st[1].bits), s>>>(p);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fxc
