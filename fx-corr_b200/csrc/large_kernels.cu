// large_kernels.cu — correlation path for FFT lengths above one CTA's shared
// memory (N = C * M with M = 8192, C in {2, 4, 8}: N = 16384 .. 65536).
//
// The N-point complex FFT of z = x1 + i x2 runs as one decimation-in-frequency
// radix-C step over the frame followed by C shared-memory FFTs of M points:
//   y_q[m] = W_N^(m q) * sum_c z[m + M c] W_C^(c q),   Z[C k + q] = FFT_M(y_q)[k].
// Kernels, per batch of frames held in device scratch:
//   decode_global_kernel  decode + LSB flip + integer shift -> z   (src/utils.rs:126-376)
//   dif_kernel<C>         the radix-C step with its twiddles    -> y
//   cfft_kernel<M>        M-point Stockham FFT per row            -> Z (row q, column k)
//   acc_global_kernel     two-for-one split, band alignment, fringe x ramp rotation and
//                         ACF/XCF accumulation (src/main.rs:2491-2568) per bin, in f64,
//                         into per-frame-group partials reduced by reduce_partials_kernel.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

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

// Per-station decode plan of decode_dif_kernel: for a station whose samples
// are contiguous runs of word bits after the shuffle (1- and 2-bit stations
// under any shuffle, wider ones unshuffled), sample slot c of a word is read
// with one or two shifts: code = (w >> p0) & mask, or, for a 2-bit sample whose
// two bits the shuffle separates or swaps, ((w >> p0) & 1) | ((w >> p1) & 1) << 1.
// Bit j of slot c's code is word bit perm[c b + j] (src/utils.rs:159-171).
struct ShiftPlan {
  uint32_t p0[32], p1[32];
  uint32_t split;  // bit c: slot c takes two shifts
};

__device__ __forceinline__ bool shift_decodable(const StationParams& q) {
  return q.bits <= 2 || q.shkind == SH_IDENTITY;
}

__device__ __forceinline__ void build_shift_plan(const StationParams& q, ShiftPlan& sp, int i) {
  const int b = q.bits, spw = 32 / b;
  if (i >= spw) return;
  const bool natural = q.shkind == SH_IDENTITY;
  const uint32_t p0 = natural ? (uint32_t)(i * b) : q.perm[i * b];
  const uint32_t p1 = b == 2 ? (natural ? (uint32_t)(i * b + 1) : q.perm[i * b + 1]) : 0u;
  sp.p0[i] = p0;
  sp.p1[i] = p1;
  if (b == 2 && p1 != p0 + 1) atomicOr(&sp.split, 1u << i);
}

// Decode + shift fused with the first (radix-C, decimation in frequency)
// step of the four-step FFT: thread (frame, m) decodes samples m + M c of both
// stations (z = x1 + i x2, station 2 negated on odd frames as in
// decode_global_kernel), combines them with a C-point DFT and writes row q,
// column m twiddled by W_N^(m q) — the complex frame never goes to HBM.
// M is a whole number of words, so the C samples of a column sit in the same
// slot of C words: the slot's shifts are looked up once per station.
template <int C>
__global__ void decode_dif_kernel(const LargeParams p, uint64_t f0, uint64_t nb,
                                  float2* __restrict__ y) {
  __shared__ uint32_t lut[2048];
  __shared__ float lv[512];
  __shared__ ShiftPlan plan[2];
  for (int i = threadIdx.x; i < 512; i += blockDim.x)
    lv[i] = p.st[i >> 8].levels[i & 255] * p.st[i >> 8].scale;
  for (int s = 0; s < 2; ++s)
    if (p.st[s].shkind == SH_GENERIC && !shift_decodable(p.st[s]))
      for (int i = threadIdx.x; i < 1024; i += blockDim.x) lut[s * 1024 + i] = p.st[s].shlut[i];
  if (threadIdx.x < 2) plan[threadIdx.x].split = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < 64; i += blockDim.x)
    if (shift_decodable(p.st[i >> 5])) build_shift_plan(p.st[i >> 5], plan[i >> 5], i & 31);
  __syncthreads();
  constexpr int M = kLargeM;
  constexpr int N = C * M;
  static_assert(M == 8192, "frame / column split by shifts");
  const bool fast[2] = {shift_decodable(p.st[0]), shift_decodable(p.st[1])};
  const uint64_t total = nb * (uint64_t)M;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t fl = idx >> 13;
    const int m = (int)(idx & (uint64_t)(M - 1));
    const uint64_t f = f0 + fl;
    const FrameInfo& F = p.finfo[f];
    const bool odd = (f & 1u) != 0;
    float xs[2][8];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const StationParams& q = p.st[s];
      const uint8_t* fr = q.raw + f * q.bpf;
      const int m0 = m - (s == 0 ? F.s1 : F.s2);
      const float* lvs = lv + 256 * s;
      if (fast[s]) {
        const int b = q.bits, lg = b == 1 ? 5 : (b == 2 ? 4 : (b == 4 ? 3 : 2));
        const uint32_t spw = 32u / (uint32_t)b, mask = (1u << b) - 1u;
        const int c = m0 & (int)(spw - 1u);
        const uint32_t p0 = plan[s].p0[c], p1 = plan[s].p1[c];
        const bool split = (plan[s].split >> c) & 1u;
        const int w0 = m0 >> lg;  // floor division
        const uint32_t* words = reinterpret_cast<const uint32_t*>(fr);
        const bool neg = q.lsb && (m0 & 1);  // M is even: the same parity on every row
#pragma unroll
        for (int r = 0; r < C; ++r) {
          const int mr = m0 + M * r;
          float x = 0.f;
          if ((unsigned)mr < (unsigned)N) {
            const uint32_t w = words[w0 + r * (M >> lg)];
            const uint32_t code = split ? (((w >> p0) & 1u) | (((w >> p1) & 1u) << 1))
                                        : ((w >> p0) & mask);
            x = lvs[code];
            if (neg) x = -x;
          }
          xs[s][r] = x;
        }
      } else {
#pragma unroll
        for (int r = 0; r < C; ++r)
          xs[s][r] = sample_at(fr, q.bits, q.shkind, lut + 1024 * s, lvs, q.lsb, m0 + M * r, N);
      }
    }
    float2 v[16];
#pragma unroll
    for (int c = 0; c < C; ++c) v[c] = make_float2(xs[0][c], odd ? -xs[1][c] : xs[1][c]);
    if constexpr (C == 2) {
      dft2<0>(v);
    } else if constexpr (C == 4) {
      dft4<0>(v);
    } else {
      dft8<0>(v);
    }
    float2* yf = y + fl * (uint64_t)N;
#pragma unroll
    for (int q = 0; q < C; ++q) {
      float2 val = v[out_pos<C>(q)];
      if (q > 0) val = cmul(val, p.tw[m * q]);
      yf[q * M + m] = val;
    }
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

// In-place M-point FFT of each row of y (rows of M complex values), natural order.
template <int M>
__global__ void __launch_bounds__(M / 16, 1) cfft_kernel(float2* __restrict__ y, uint64_t rows) {
  extern __shared__ __align__(128) uint8_t smem[];
  constexpr int T1 = M / 16;
  float2* bufA = reinterpret_cast<float2*>(smem);
  float2* bufB = bufA + Geom<M>::CSTRIDE;
  float* x1 = reinterpret_cast<float*>(bufB);
  float* x2 = x1 + Geom<M>::FSTRIDE;
  const int t = threadIdx.x;
  Twiddles<M> tw;
  tw.init(t);
  for (uint64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    float2* row = y + r * M;
    for (int i = t; i < M; i += T1) {
      const float2 v = row[i];
      x1[fpad(i)] = v.x;
      x2[fpad(i)] = v.y;
    }
    __syncthreads();
    first_pass<M>(x1, x2, 0, 0, bufA, t);
    float2* Z = fft_rest<M>(bufA, bufB, t, tw);
    __syncthreads();
    for (int i = t; i < M; i += T1) row[i] = Z[i];
    __syncthreads();
  }
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
  double a[4] = {0, 0, 0, 0};
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
      if (want_acf && (!ov_only || inov)) a[0] += (double)cnorm2(p1);
      if (inov) {
        const int i2 = bin + sb;
        const float2 c = zi(Zf, i2), d = zi(Zf, N - i2);
        const float2 q2 = make_float2(sg * (c.y + d.y), sg * (d.x - c.x));
        if (want_acf) a[1] += (double)cnorm2(q2);
        if (want_xcf) {
          const float2 x = cmul(cmulc(p1, q2), r);
          a[2] += (double)x.x;
          a[3] += (double)x.y;
        }
      }
    } else {
      const bool inov = bin >= a2s && bin < a2s + ov;
      const float2 p2 = make_float2(sg * (u.y + w.y), sg * (w.x - u.x));
      if (want_acf && (!ov_only || inov)) a[1] += (double)cnorm2(p2);
      if (inov) {
        const int i1 = bin - sb;
        const float2 c = zi(Zf, i1), d = zi(Zf, N - i1);
        const float2 q1 = make_float2(c.x + d.x, c.y - d.y);
        if (want_acf) a[0] += (double)cnorm2(q1);
        if (want_xcf) {
          const float2 x = cmul(cmulc(q1, p2), r);
          a[2] += (double)x.x;
          a[3] += (double)x.y;
        }
      }
    }
  }
  double* pg = part + (size_t)blockIdx.z * 4 * H;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double* d = pg + (size_t)v * H + bin;
    *d = (first_batch ? 0.0 : *d) + a[v];
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
  double acc = 0.0;
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
      float sn, cs;
      sincosf((float)k * (s == 0 ? F.st1 : F.st2), &sn, &cs);
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
    acc += (double)cnorm2(cb);
    if (pp.want_raw) {
      float2* wf = W + fl * (uint64_t)N;
      if (bin == 0 || bin == N / 2) cb.y = 0.f;
      wf[bin] = make_float2(cb.x, -cb.y);
      if (bin != 0 && bin != N / 2) wf[N - bin] = cb;
    }
  }
  double* d = part + (size_t)blockIdx.z * H + bin;
  *d = (first_batch ? 0.0 : *d) + acc;
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
  // two scratch buffers of batch * n complex f32 each, 64 MiB apiece
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
  const uint32_t smem = 2 * Geom<kLargeM>::CSTRIDE * sizeof(float2);
  auto kern = cfft_kernel<kLargeM>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const uint64_t rows = nb * (uint64_t)p.c;
  kern<<<(unsigned)std::min<uint64_t>(rows, (uint64_t)sms), kLargeM / 16, smem, s>>>(buf1, rows);
  return cudaGetLastError();
}

cudaError_t launch_large_fft(const LargeParams& p, uint64_t f0, uint64_t nb, float2* buf0,
                             float2* buf1, int sms, cudaStream_t s) {
  // decode + DIF -> buf1, row FFTs in place on buf1 (buf0 is not used)
  (void)buf0;
  const uint64_t work = nb * kLargeM;
  switch (p.c) {
    case 2: decode_dif_kernel<2><<<grid_for(work, 256, sms), 256, 0, s>>>(p, f0, nb, buf1); break;
    case 4: decode_dif_kernel<4><<<grid_for(work, 256, sms), 256, 0, s>>>(p, f0, nb, buf1); break;
    case 8: decode_dif_kernel<8><<<grid_for(work, 256, sms), 256, 0, s>>>(p, f0, nb, buf1); break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return row_ffts(p, nb, buf1, sms, s);
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
  if ((e = large_fft_core(p, nb, buf0, buf1, sms, s)) != cudaSuccess) return e;
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
