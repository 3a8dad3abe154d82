// fxc_device.cuh — device building blocks shared by the sm_100a kernels:
// complex arithmetic, in-register DFT butterflies, Stockham radix passes over
// padded shared memory, the FP64 per-frame delay model and the packed-sample
// decoder.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fxc {

// ------------------------------------------------------------ parameters

// DelayEvalConfig (src/main.rs:161-182) with the 1-s table in device memory.
struct DelayParams {
  double frame_dt, fs, time_offset_s;
  const double* table;  // nullptr -> polynomial branch
  uint64_t table_len;
  double coarse, user_samples, extra_rate;
  double c1d, c1r, c2d, c2r, d_seek;
  double d1, r1, a1, d2, r2, a2;
  double lo1, lo2;
};

// Per-frame values the kernels consume, produced by frame_info_kernel from
// the FP64 delay model (FrameDelayEntry, src/main.rs:151-159) and staged into
// shared memory with the frame's packed words.  48 bytes (bulk-copy sized).
struct __align__(16) FrameInfo {
  int32_t s1, s2;     // integer shifts int1 / int2 clamped to [-N, N]
  float phi0, dphi;   // XCF ramp (src/main.rs:132-149): angle at overlap bin 0, slope per bin
  float2 fr_mix;      // fr_lo1 * conj(fr_lo2) (src/main.rs:2488)
  float2 fr_lo1, fr_lo2;
  float st1, st2;     // per-station fractional-delay slopes -2 pi df frac_i (src/utils.rs:114)
};
static_assert(sizeof(FrameInfo) == 48, "FrameInfo is staged by 16-byte bulk copies");

struct StationParams {
  const uint8_t* raw;      // first byte of frame 0 of the sector
  const uint32_t* shlut;   // [4][256] byte LUTs for a generic shuffle
  const float* levels;     // [256] f32 levels
  uint32_t bpf;            // bytes per frame
  int32_t bits;            // 1, 2, 4, 8
  int32_t lsb;             // negate odd samples
  int32_t shkind;          // 0 identity, 1 pair swap, 2 generic
  float scale;             // power of two equalising the two stations' RMS level
                           // inside the shared complex FFT (exact to undo)
  uint8_t perm[32];        // the 32-bit shuffle: decoder bit o is word bit perm[o]
};

enum { SH_IDENTITY = 0, SH_PAIRSWAP = 1, SH_GENERIC = 2 };

enum : uint32_t {
  ERR_WAIT_TIMEOUT = 1u,   // a bounded mbarrier wait gave up
  ERR_BAD_CONFIG = 2u,
};

// ------------------------------------------------------------ complex ops

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 mul_mj(float2 a) { return make_float2(a.y, -a.x); }  // a*(-i)
__device__ __forceinline__ float cnorm2(float2 a) { return a.x * a.x + a.y * a.y; }

// Multiplication by the compile-time root exp(-2 pi i m / 16), m in [0,16).
template <int M>
__device__ __forceinline__ float2 mul_w16(float2 a) {
  constexpr float C1 = 0.92387953251128674f;  // cos(pi/8)
  constexpr float S1 = 0.38268343236508977f;  // sin(pi/8)
  constexpr float R2 = 0.70710678118654752f;  // sqrt(1/2)
  constexpr int m = M & 15;
  if constexpr (m == 0) return a;
  else if constexpr (m == 1) return cmul(a, make_float2(C1, -S1));
  else if constexpr (m == 2) return make_float2(R2 * (a.x + a.y), R2 * (a.y - a.x));
  else if constexpr (m == 3) return cmul(a, make_float2(S1, -C1));
  else if constexpr (m == 4) return mul_mj(a);
  else if constexpr (m == 5) return cmul(a, make_float2(-S1, -C1));
  else if constexpr (m == 6) return make_float2(R2 * (a.y - a.x), -R2 * (a.x + a.y));
  else if constexpr (m == 7) return cmul(a, make_float2(-C1, -S1));
  else if constexpr (m == 8) return make_float2(-a.x, -a.y);
  else return make_float2(0.f, 0.f) /* unused */;
}

// ---------------------------------------------------------- butterflies
// Forward DFTs on a register array slice starting at B.  Output X[k] ends
// at register position out_pos<R>(k).

template <int B>
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[B], b = v[B + 1];
  v[B] = cadd(a, b);
  v[B + 1] = csub(a, b);
}

template <int I0, int I1, int I2, int I3>
__device__ __forceinline__ void dft4_idx(float2* v) {
  float2 t0 = cadd(v[I0], v[I2]);
  float2 t1 = csub(v[I0], v[I2]);
  float2 t2 = cadd(v[I1], v[I3]);
  float2 t3 = mul_mj(csub(v[I1], v[I3]));
  v[I0] = cadd(t0, t2);
  v[I1] = cadd(t1, t3);
  v[I2] = csub(t0, t2);
  v[I3] = csub(t1, t3);
}

template <int B>
__device__ __forceinline__ void dft4(float2* v) { dft4_idx<B, B + 1, B + 2, B + 3>(v); }

template <int B>
__device__ __forceinline__ void dft8(float2* v) {
  // n = 4 n1 + n2, k = k1 + 2 k2: radix 2 over n1, twiddle W8^(n2 k1), radix 4 over n2
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    float2 a = v[B + n2], b = v[B + 4 + n2];
    v[B + n2] = cadd(a, b);
    v[B + 4 + n2] = csub(a, b);
  }
  v[B + 5] = mul_w16<2>(v[B + 5]);
  v[B + 6] = mul_w16<4>(v[B + 6]);
  v[B + 7] = mul_w16<6>(v[B + 7]);
  dft4<B>(v);
  dft4<B + 4>(v);
}

__device__ __forceinline__ void dft16(float2* v) {
  // n = 4 n1 + n2, k = k1 + 4 k2
  dft4_idx<0, 4, 8, 12>(v);
  dft4_idx<1, 5, 9, 13>(v);
  dft4_idx<2, 6, 10, 14>(v);
  dft4_idx<3, 7, 11, 15>(v);
  // A[n2][k1] at n2 + 4 k1 times W16^(n2 k1)
  v[5] = mul_w16<1>(v[5]);
  v[6] = mul_w16<2>(v[6]);
  v[7] = mul_w16<3>(v[7]);
  v[9] = mul_w16<2>(v[9]);
  v[10] = mul_w16<4>(v[10]);
  v[11] = mul_w16<6>(v[11]);
  v[13] = mul_w16<3>(v[13]);
  v[14] = mul_w16<6>(v[14]);
  v[15] = make_float2(-v[15].x, -v[15].y);
  v[15] = mul_w16<1>(v[15]);  // W16^9 = -W16^1
  dft4<0>(v);
  dft4<4>(v);
  dft4<8>(v);
  dft4<12>(v);
}

template <int R>
__host__ __device__ constexpr int out_pos(int k) {
  return R == 16 ? 4 * (k & 3) + (k >> 2) : (R == 8 ? 4 * (k & 1) + (k >> 1) : k);
}

// v[B + r] *= w^r for r = 1..R-1, powers by a short product chain.
template <int R, int B>
__device__ __forceinline__ void twiddle(float2* v, float2 w) {
  if constexpr (R == 2) {
    v[B + 1] = cmul(v[B + 1], w);
  } else {
    float2 p[R];
    p[1] = w;
    p[2] = cmul(w, w);
#pragma unroll
    for (int r = 3; r < R; ++r) {
      // r = hi + lo with hi the largest power of two below r: depth <= log2 R
      const int hi = (r >= 8) ? 8 : ((r >= 4) ? 4 : 2);
      if (r == hi) p[r] = cmul(p[hi / 2], p[hi / 2]);
      else p[r] = cmul(p[hi], p[r - hi]);
    }
#pragma unroll
    for (int r = 1; r < R; ++r) v[B + r] = cmul(v[B + r], p[r]);
  }
}

// ---------------------------------------------------------- smem layout

// Complex buffers: one pad slot per 16 elements keeps the radix-16 Stockham
// loads and stores free of bank conflicts for 8-byte accesses.
__device__ __forceinline__ int cpad(int i) { return i + (i >> 4); }
// Planar float buffers (decoded samples): one pad word per 32.
__device__ __forceinline__ int fpad(int i) { return i + (i >> 5); }

template <int N>
struct Geom {
  static constexpr int T1 = N / 16;            // threads per frame pair
  static constexpr int CSTRIDE = N + N / 16;   // float2 per padded frame
  static constexpr int FSTRIDE = N + N / 32;   // floats per padded station plane
  static constexpr int LOG2N = (N == 1024) ? 10 : (N == 2048) ? 11 : (N == 4096) ? 12
                             : (N == 8192) ? 13 : (N == 16384) ? 14 : 0;
  static constexpr int P16 = LOG2N / 4;            // radix-16 passes
  static constexpr int RL = 1 << (LOG2N % 4);      // trailing radix (1 = none)
  static constexpr int NPASS = P16 + (RL > 1 ? 1 : 0);
};

// Per-thread twiddle bases (frame invariant): pass p (1 <= p < P16) uses
// exp(-2 pi i (t mod 16^p) / 16^(p+1)); the trailing pass uses exp(-2 pi i t / N).
// A shared-memory table of the powers would trade the 14 complex products of
// a power chain for 15 8-byte shared loads, and the shared-memory pipe, not
// the FMA pipe, is the tighter resource of these kernels.
template <int N>
struct Twiddles {
  float2 w[Geom<N>::NPASS];
  __device__ __forceinline__ void init(int t) {
    constexpr int P16 = Geom<N>::P16;
#pragma unroll
    for (int p = 0; p < Geom<N>::NPASS; ++p) {
      double frac;
      if (p == 0) {
        frac = 0.0;
      } else if (p < P16) {
        const int ns = 1 << (4 * p);
        frac = (double)(t & (ns - 1)) / (double)(ns * 16);
      } else {
        frac = (double)t / (double)N;
      }
      double s, c;
      sincospi(-2.0 * frac, &s, &c);
      w[p] = make_float2((float)c, (float)s);
    }
  }
};

// One Stockham pass (radix R, stride NS) over padded complex buffers: every
// thread handles 16/R work items j = t + T1*w.  The last pass of a transform
// (OUT_PAD = false) stores an unpadded natural-order spectrum: its stores are
// consecutive runs, and unpadded consecutive runs of any alignment (the
// Z[N-k], Z[k+sb] reads of the consumers) are free of bank conflicts.
template <int N, int R, int NS, bool OUT_PAD = true>
__device__ __forceinline__ void stockham_pass(const float2* __restrict__ in, float2* __restrict__ out,
                                              int t, float2 w) {
  constexpr int T1 = N / 16;
  constexpr int WI = 16 / R;
  static_assert((N / R) % 16 == 0 && NS % 16 == 0, "padded strides");
  // cpad(j + r*M) = cpad(j) + r*(M + M/16) whenever M is a multiple of 16
  constexpr int LS = N / R + N / (16 * R);
  constexpr int SS = NS + NS / 16;
  float2 v[16];
#pragma unroll
  for (int wi = 0; wi < WI; ++wi) {
    const int j = t + T1 * wi;
    const float2* src = in + cpad(j);
#pragma unroll
    for (int r = 0; r < R; ++r) v[wi * R + r] = src[r * LS];
  }
  if constexpr (NS > 1) {
    if constexpr (R == 16) {
      twiddle<16, 0>(v, w);
    } else {
      // trailing pass: k = j, exp(-2 pi i (t + T1 wi) / N) = w * W16^wi
#pragma unroll
      for (int wi = 0; wi < WI; ++wi) {
        float2 ww;
        switch (wi) {  // compile-time after unrolling
          case 0: ww = w; break;
          case 1: ww = mul_w16<1>(w); break;
          case 2: ww = mul_w16<2>(w); break;
          case 3: ww = mul_w16<3>(w); break;
          case 4: ww = mul_w16<4>(w); break;
          case 5: ww = mul_w16<5>(w); break;
          case 6: ww = mul_w16<6>(w); break;
          default: ww = mul_w16<7>(w); break;
        }
        if constexpr (R == 2) {
          v[wi * 2 + 1] = cmul(v[wi * 2 + 1], ww);
        } else if constexpr (R == 4) {
          float2 w2 = cmul(ww, ww);
          v[wi * 4 + 1] = cmul(v[wi * 4 + 1], ww);
          v[wi * 4 + 2] = cmul(v[wi * 4 + 2], w2);
          v[wi * 4 + 3] = cmul(v[wi * 4 + 3], cmul(w2, ww));
        } else {  // R == 8
          float2 p2 = cmul(ww, ww), p4 = cmul(p2, p2);
          float2 p3 = cmul(p2, ww);
          v[wi * 8 + 1] = cmul(v[wi * 8 + 1], ww);
          v[wi * 8 + 2] = cmul(v[wi * 8 + 2], p2);
          v[wi * 8 + 3] = cmul(v[wi * 8 + 3], p3);
          v[wi * 8 + 4] = cmul(v[wi * 8 + 4], p4);
          v[wi * 8 + 5] = cmul(v[wi * 8 + 5], cmul(p4, ww));
          v[wi * 8 + 6] = cmul(v[wi * 8 + 6], cmul(p4, p2));
          v[wi * 8 + 7] = cmul(v[wi * 8 + 7], cmul(p4, p3));
        }
      }
    }
  }
  if constexpr (R == 16) {
    dft16(v);
  } else {
#pragma unroll
    for (int wi = 0; wi < WI; ++wi) {
      if constexpr (R == 2) {
        float2 a = v[wi * 2], b = v[wi * 2 + 1];
        v[wi * 2] = cadd(a, b);
        v[wi * 2 + 1] = csub(a, b);
      } else if constexpr (R == 4) {
        float2 a0 = v[wi * 4], a1 = v[wi * 4 + 1], a2 = v[wi * 4 + 2], a3 = v[wi * 4 + 3];
        float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_mj(csub(a1, a3));
        v[wi * 4] = cadd(t0, t2);
        v[wi * 4 + 1] = cadd(t1, t3);
        v[wi * 4 + 2] = csub(t0, t2);
        v[wi * 4 + 3] = csub(t1, t3);
      } else {
        float2 u[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) u[r] = v[wi * 8 + r];
        dft8<0>(u);
#pragma unroll
        for (int r = 0; r < 8; ++r) v[wi * 8 + r] = u[r];
      }
    }
  }
#pragma unroll
  for (int wi = 0; wi < WI; ++wi) {
    const int j = t + T1 * wi;
    const int k = j & (NS - 1);
    if constexpr (OUT_PAD) {
      float2* dst = out + cpad((j - k) * R + k);
#pragma unroll
      for (int r = 0; r < R; ++r) dst[r * SS] = v[wi * R + out_pos<R>(r)];
    } else {
      float2* dst = out + (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) dst[r * NS] = v[wi * R + out_pos<R>(r)];
    }
  }
}

// First pass: reads the two decoded station planes with their integer shifts
// (zero fill, src/utils.rs:126-145) and packs z[n] = x1[n-s1] + i x2[n-s2].
template <int N>
__device__ __forceinline__ void first_pass(const float* __restrict__ x1, const float* __restrict__ x2,
                                           int s1, int s2, float2* __restrict__ out, int t) {
  constexpr int T1 = N / 16;
  static_assert(T1 % 32 == 0, "plane stride");
  // fpad(t + r*T1) = fpad(t) + r*(T1 + T1/32) since T1 is a multiple of 32
  constexpr int PS = T1 + T1 / 32;
  float2 v[16];
  // the shift is uniform per frame: unshifted stations take the unchecked path
  if (s1 == 0) {
    const float* p = x1 + fpad(t);
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r].x = p[r * PS];
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m = t + r * T1 - s1;
      v[r].x = ((unsigned)m < (unsigned)N) ? x1[fpad(m)] : 0.0f;
    }
  }
  if (s2 == 0) {
    const float* p = x2 + fpad(t);
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r].y = p[r * PS];
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m = t + r * T1 - s2;
      v[r].y = ((unsigned)m < (unsigned)N) ? x2[fpad(m)] : 0.0f;
    }
  }
  dft16(v);
  float2* dst = out + 17 * t;  // cpad(16 t + r) = 17 t + r
#pragma unroll
  for (int r = 0; r < 16; ++r) dst[r] = v[out_pos<16>(r)];
}

// One station of a frame as staged packed words (already shuffled into the
// decoder's bit order), decoded on the fly by first_pass_packed.
struct PackedStation {
  const uint32_t* words;  // the frame's words in shared memory
  const float* lv;        // levels (scaled) in shared memory
  uint32_t bits, mask;
  int lsb;                // negate odd samples (LSB -> USB, src/utils.rs:196-197)
  int shift;              // integer shift of this frame, clamped to [-N, N]
  uint32_t flip = 0;      // 1: negate the whole frame (first_pass_packed only)
};

// Sample m of the frame (0 <= m < N): b-bit code taken LSB-first from the
// packed words (src/utils.rs:215-376), mapped to its level, odd samples negated
// for LSB input.
__device__ __forceinline__ float packed_sample(const PackedStation& p, int m) {
  const uint32_t bit = (uint32_t)m * p.bits;
  const uint32_t w = p.words[bit >> 5];
  const float v = p.lv[(w >> (bit & 31u)) & p.mask];
  return __int_as_float(__float_as_int(v) ^ (int)((uint32_t)(m & p.lsb) << 31));
}

// The 16 first-pass inputs of one station, x[t + r*T1 - shift] for r < 16,
// decoded from the packed words.  Since T1 is a multiple of the samples per
// word, the bit position and the odd/even sign of a thread's 16 samples are
// constant and the word offsets step by a compile-time stride.
template <int N, int BITS, bool IMAG>
__device__ __forceinline__ void station_inputs(const PackedStation& p, float2 (&v)[16], int t) {
  constexpr int T1 = N / 16;
  constexpr int SPW = 32 / BITS;                 // samples per word
  constexpr int LOG2_SPW = BITS == 1 ? 5 : (BITS == 2 ? 4 : (BITS == 4 ? 3 : 2));
  constexpr int WSTEP = T1 / SPW;                // word stride between r and r+1
  constexpr uint32_t MASK = (1u << BITS) - 1u;
  static_assert(T1 % SPW == 0, "frame stride is a whole number of words");
  const int m0 = t - p.shift;
  const uint32_t bitpos = (uint32_t)(m0 & (SPW - 1)) * BITS;
  // odd samples of LSB input are negated; `flip` negates the frame
  const uint32_t sign = ((uint32_t)(m0 & p.lsb) ^ p.flip) << 31;
  const int w0 = m0 >> LOG2_SPW;                 // floor division (m0 may be negative)
  if (p.shift == 0) {
    const uint32_t* w = p.words + w0;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const float x = __uint_as_float(__float_as_uint(p.lv[(w[r * WSTEP] >> bitpos) & MASK]) ^ sign);
      if (IMAG) v[r].y = x; else v[r].x = x;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m = m0 + r * T1;
      const bool in = (unsigned)m < (unsigned)N;
      const uint32_t w = p.words[in ? w0 + r * WSTEP : 0];
      const float x = __uint_as_float(__float_as_uint(p.lv[(w >> bitpos) & MASK]) ^ sign);
      if (IMAG) v[r].y = in ? x : 0.0f; else v[r].x = in ? x : 0.0f;
    }
  }
}

template <int N, bool IMAG>
__device__ __forceinline__ void station_inputs_any(const PackedStation& p, float2 (&v)[16], int t) {
  switch (p.bits) {
    case 1: station_inputs<N, 1, IMAG>(p, v, t); break;
    case 2: station_inputs<N, 2, IMAG>(p, v, t); break;
    case 4: station_inputs<N, 4, IMAG>(p, v, t); break;
    default: station_inputs<N, 8, IMAG>(p, v, t); break;
  }
}

// First pass fused with the decode: z[n] = x1[n - s1] + i x2[n - s2] read
// straight from the packed words with the integer shift and zero fill
// (src/utils.rs:126-145).  Lanes take consecutive n, so each word load is a
// broadcast; a station with zero shift takes the unchecked path.
template <int N>
__device__ __forceinline__ void first_pass_packed(const PackedStation& a, const PackedStation& b,
                                                  float2* __restrict__ out, int t) {
  float2 v[16];
  station_inputs_any<N, false>(a, v, t);
  station_inputs_any<N, true>(b, v, t);
  dft16(v);
  float2* dst = out + 17 * t;  // cpad(16 t + r) = 17 t + r
#pragma unroll
  for (int r = 0; r < 16; ++r) dst[r] = v[out_pos<16>(r)];
}

// Runs passes 2..NPASS; `a` holds the first pass output, returns the buffer
// with the natural-order spectrum Z[0..N).  With NO_TRAIL the trailing radix-2
// pass (RL == 2) is left to the consumer: the returned buffer then holds its
// input Y unpadded, and Z[k] = Y[k] + W_N^k Y[k + N/2],
// Z[k + N/2] = Y[k] - W_N^k Y[k + N/2] for k < N/2.
template <int N, bool NO_TRAIL = false>
__device__ __forceinline__ float2* fft_rest(float2* a, float2* b, int t, const Twiddles<N>& tw) {
  constexpr int P16 = Geom<N>::P16;
  constexpr int RL = Geom<N>::RL;
  static_assert(!NO_TRAIL || RL == 2, "only a trailing radix-2 pass is left out");
  constexpr bool TRAIL = RL > 1 && !NO_TRAIL;
  float2* in = a;
  float2* out = b;
  // the returned buffer is unpadded
  static_assert(P16 >= 2, "at least two radix-16 passes");
  {
    __syncthreads();
    stockham_pass<N, 16, 16, (P16 >= 3 || TRAIL)>(in, out, t, tw.w[1]);
    float2* x = in; in = out; out = x;
  }
  if constexpr (P16 >= 3) {
    __syncthreads();
    stockham_pass<N, 16, 256, TRAIL>(in, out, t, tw.w[2]);
    float2* x = in; in = out; out = x;
  }
  if constexpr (TRAIL) {
    constexpr int NS = 1 << (4 * P16);
    __syncthreads();
    stockham_pass<N, RL, NS, false>(in, out, t, tw.w[P16]);
    float2* x = in; in = out; out = x;
  }
  return in;
}

// ------------------------------------------------------------ delay model
// Restatement of compute_frame_delay_entry (src/main.rs:184-241) in IEEE
// f64 with every operation explicitly rounded (no contraction), so the
// integer sample shifts round exactly as the reference's.

__device__ __forceinline__ double dA(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dS(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dM(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dD(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ int64_t f64_as_i64(double v) {
  if (v != v) return 0;
  if (v >= 9223372036854775807.0) return INT64_MAX;
  if (v <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)v;
}

__device__ __forceinline__ float2 carrier_phase(double f_hz, double tau) {
  // src/main.rs:110-120
  if (f_hz == 0.0) return make_float2(1.0f, 0.0f);
  const double pi = 3.141592653589793;
  const double two_pi = 6.283185307179586;  // 2.0 * PI, exact doubling
  const double phase = dM(dM(-two_pi, f_hz), tau);
  double m = fmod(dA(phase, pi), two_pi);  // rem_euclid
  if (m < 0.0) m = dA(m, two_pi);
  const float th = (float)dS(m, pi);
  float s, c;
  sincosf(th, &s, &c);
  return make_float2(c, s);
}

__device__ __forceinline__ void split_delay(double tau, double fs, int64_t* ip, double* fp) {
  // src/main.rs:126-130
  const int64_t i = f64_as_i64(round(dM(tau, fs)));
  *ip = i;
  *fp = dS(tau, dD((double)i, fs));
}

__device__ __forceinline__ void frame_delay(const DelayParams& p, uint64_t frame_idx, int64_t* int1,
                                            int64_t* int2, double* frac1, double* frac2,
                                            float2* lo1, float2* lo2) {
  const double t_mid_local = dM(dA((double)frame_idx, 0.5), p.frame_dt);
  const double t_mid = dA(t_mid_local, p.time_offset_s);
  double tau1, tau2, t1f, t2f;
  if (p.table != nullptr) {
    const uint64_t last = p.table_len > 0 ? p.table_len - 1 : 0;
    double fl = floor(t_mid_local);
    if (!(fl > 0.0)) fl = 0.0;
    const uint64_t sec = fl >= 18446744073709551615.0 ? ~0ull : (uint64_t)fl;
    const uint64_t i0 = sec < last ? sec : last;
    const uint64_t i1 = (i0 + 1) < last ? (i0 + 1) : last;
    double frac = 0.0;
    if (i1 != i0) {
      frac = dS(t_mid_local, (double)i0);
      frac = frac < 0.0 ? 0.0 : (frac > 1.0 ? 1.0 : frac);
    }
    const double gd_t = dA(dM(p.table[i0], dS(1.0, frac)), dM(p.table[i1], frac));
    const double net = dA(dA(dA(gd_t, p.coarse), dD(p.user_samples, p.fs)), dM(p.extra_rate, t_mid));
    const double c1 = dA(p.c1d, dM(p.c1r, t_mid));
    const double c2 = dA(p.c2d, dM(p.c2r, t_mid));
    const double full = dA(net, dS(c2, c1));
    tau1 = dS(full, p.d_seek);
    tau2 = 0.0;
    t1f = full;
    t2f = 0.0;
  } else {
    const double tt = dM(t_mid, t_mid);
    tau1 = dA(dA(p.d1, dM(p.r1, t_mid)), dM(dM(0.5, p.a1), tt));
    tau2 = dA(dA(p.d2, dM(p.r2, t_mid)), dM(dM(0.5, p.a2), tt));
    t1f = dA(tau1, p.d_seek);
    t2f = tau2;
  }
  split_delay(tau1, p.fs, int1, frac1);
  split_delay(tau2, p.fs, int2, frac2);
  *lo1 = carrier_phase(p.lo1, t1f);
  *lo2 = carrier_phase(p.lo2, t2f);
}

// Full per-frame record used by the correlation kernels.
__device__ __forceinline__ void frame_info(const DelayParams& p, uint64_t frame_idx, int n,
                                           double df_hz, int a1s, int a2s, FrameInfo* fi) {
  int64_t i1, i2;
  double f1, f2;
  float2 l1, l2;
  frame_delay(p, frame_idx, &i1, &i2, &f1, &f2, &l1, &l2);
  fi->s1 = (int32_t)(i1 > n ? n : (i1 < -n ? -n : i1));
  fi->s2 = (int32_t)(i2 > n ? n : (i2 < -n ? -n : i2));
  fi->fr_lo1 = l1;
  fi->fr_lo2 = l2;
  fi->fr_mix = cmulc(l1, l2);  // fr_lo1 * conj(fr_lo2) (src/main.rs:2488)
  // xcf_phase_start_and_step (src/main.rs:132-149): angle(k) = phi0 + k*dphi
  const double two_pi_df = dM(-6.283185307179586, df_hz);
  const double st1 = dM(two_pi_df, f1), st2 = dM(two_pi_df, f2);
  fi->phi0 = (float)dS(dM(st1, (double)a1s), dM(st2, (double)a2s));
  fi->dphi = (float)dS(st1, st2);
  fi->st1 = (float)st1;
  fi->st2 = (float)st2;
}

// ----------------------------------------------------------------- decode
// 32-bit word shuffle of the decoder (src/utils.rs:159-171).

__device__ __forceinline__ uint32_t shuffle_word(uint32_t w, int kind, const uint32_t* lut) {
  if (kind == SH_PAIRSWAP) return ((w & 0xAAAAAAAAu) >> 1) | ((w & 0x55555555u) << 1);
  if (kind == SH_GENERIC)
    return lut[w & 255u] | lut[256 + ((w >> 8) & 255u)] | lut[512 + ((w >> 16) & 255u)] |
           lut[768 + (w >> 24)];
  return w;
}

// Applies the stations' 32-bit shuffles (src/utils.rs:159-171) in place to the
// staged words of a slot: [FPC frames of station 1][FPC frames of station 2].
__device__ __forceinline__ void preshuffle_slot(uint32_t* w1, uint32_t n1, int kind1,
                                                const uint32_t* lut1, uint32_t* w2, uint32_t n2,
                                                int kind2, const uint32_t* lut2, int tid,
                                                int nthreads) {
  if (kind1 != SH_IDENTITY)
    for (uint32_t i = tid; i < n1; i += nthreads) w1[i] = shuffle_word(w1[i], kind1, lut1);
  if (kind2 != SH_IDENTITY)
    for (uint32_t i = tid; i < n2; i += nthreads) w2[i] = shuffle_word(w2[i], kind2, lut2);
}

// Bounded mbarrier helpers (cp.async.bulk staging).
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
               : "memory");
}
// Returns true when the phase completed, false after max_iters polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t max_iters) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  for (uint32_t it = 0; it < max_iters; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
      "l"(src), "r"(bytes), "r"(b)
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Nearest level, first index wins ties (utils.rs:384-389).  For tables with
// more than 16 entries that are strictly monotonic (flag set by the host) a
// binary search finds the bracket and the exact f32 comparison runs over a
// window of +-2 entries around it.
__device__ __forceinline__ uint32_t nearest_level(float x, const float* __restrict__ ql, int n,
                                                  int monotonic) {
  int lo = 0, hi = n;
  if (monotonic != 0 && n > 16) {
    // ascending (monotonic > 0) or descending (< 0): find first index past x
    int a = 0, b = n;
    while (a < b) {
      const int m = (a + b) >> 1;
      const bool past = monotonic > 0 ? (ql[m] > x) : (ql[m] < x);
      if (past) b = m;
      else a = m + 1;
    }
    lo = max(0, a - 2);
    hi = min(n, a + 2);
  }
  uint32_t best = (uint32_t)lo;
  float min_err = 3.40282347e38f;
  for (int i = lo; i < hi; ++i) {
    const float err = fabsf(x - ql[i]);
    if (err < min_err) {
      min_err = err;
      best = (uint32_t)i;
    }
  }
  return best;
}

// ------------------------------------------------------ staging layout

constexpr int kStages = 2;
// Bounded mbarrier wait: an unsatisfied try_wait returns after about 3.3 us
// on B200 (measured with the failure-injection hook), so 2^19 polls give up
// after about 1.7 s, three orders of magnitude above any staging copy.
constexpr uint32_t kWaitPolls = 1u << 19;
constexpr uint32_t kFiBytes = sizeof(FrameInfo);

struct SmemLayout {
  uint32_t off_a, off_b, off_stage, stage_stride, off_lut, off_lv, off_fi, off_bar, off_flag, total;
};

// Staging slot: [FPC FrameInfo][FPC frames of station 1][FPC frames of station 2]
template <int N, int FPC>
__host__ __device__ inline SmemLayout smem_layout(uint32_t raw_bytes) {
  SmemLayout L;
  const uint32_t cbytes = (uint32_t)(FPC * Geom<N>::CSTRIDE * sizeof(float2));
  L.off_a = 0;
  L.off_b = L.off_a + cbytes;
  L.off_stage = L.off_b + cbytes;
  L.stage_stride = (FPC * kFiBytes + raw_bytes + 127u) & ~127u;
  L.off_lut = L.off_stage + kStages * L.stage_stride;
  L.off_lv = L.off_lut + 2 * 1024 * 4;
  L.off_fi = L.off_lv + 2 * 256 * 4;
  L.off_bar = L.off_fi + FPC * kFiBytes;
  L.off_flag = L.off_bar + kStages * 8;
  L.total = L.off_flag + 16;
  return L;
}

}  // namespace fxc
