// row_fft.cuh — pieces of the 8192-point row FFTs shared by the kernels that
// hold whole rows in shared memory (phased_pair.cu, phased_cpair.cu): the
// trailing radix-2 pass in place or folded into its reader, a radix-2
// decimation-in-frequency twiddle, and the first radix-16 pass from registers.
#pragma once

#include "fxc_device.cuh"

namespace fxc {
namespace rows {

constexpr int kM = 8192;       // row length
constexpr int kT = kM / 16;    // threads per CTA
constexpr int kJ = kM / 2 / kT;  // radix-2 butterflies per thread

// The trailing radix-2 pass of a row in place: Z[j], Z[j + M/2] from the last
// radix-16 pass's output, j = t + T i.
__device__ __forceinline__ void row_radix2(float2* Z, int tid, const Twiddles<kM>& tw) {
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
    const float2 a = Z[j], wb = cmul(wj, Z[j + kM / 2]);
    Z[j] = cadd(a, wb);
    Z[j + kM / 2] = csub(a, wb);
  }
}

// The trailing radix-2 pass folded into a reader (no write-back): with Y the
// last radix-16 pass's output (unpadded) and j = t + T i, j < M/2,
//   Z[j]            = Y[j] + W^j Y[j + M/2]
//   Z[c + M/2]      = Y[c] + conj(W^(M/2 - c)) Y[c + M/2]     (W^c = -conj(W^(M/2-c)))
// so the mirror's upper-half values at c = M/2 - 1 - j (index M - 1 - j) take
// W^(j+1) and at c = M/2 - j (index M - j) take W^j.  wb1 = W_M^(t+1).
__device__ __forceinline__ void fold_twiddles(const Twiddles<kM>& tw, float2 wb1, int i, float2& wj,
                                              float2& wj1) {
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
}
// Z[j] of a row (j < M/2).
__device__ __forceinline__ float2 fold_lower(const float2* Y, int j, float2 wj) {
  return cadd(Y[j], cmul(wj, Y[j + kM / 2]));
}
// Z[M - 1 - j] (self0 false: wk = W^(j+1)) or Z[(M - j) mod M] (self0 true:
// wk = W^j; j = 0 gives Z[0]) of a row, j < M/2.
__device__ __forceinline__ float2 fold_mirror(const float2* Y, int j, bool self0, float2 wj,
                                              float2 wj1) {
  if (self0 && j == 0) return fold_lower(Y, 0, wj);
  const int c = self0 ? kM / 2 - j : kM / 2 - 1 - j;
  return cadd(Y[c], cmulc(Y[c + kM / 2], self0 ? wj : wj1));
}
// W_M^(t+1), correctly rounded.
__device__ __forceinline__ float2 fold_base1(int t) {
  double sn, cs;
  sincospi(-2.0 * (double)(t + 1) / (double)kM, &sn, &cs);
  return make_float2((float)cs, (float)sn);
}

// Row 1's twiddle W_N^m of a radix-2 decimation in frequency (N = 2 M),
// m = t + T r: W^t W_32^r from the bases b0 = W_N^t and b1 = W_N^(t + T)
// (even / odd r) times W_16^(r/2).
__device__ __forceinline__ void row1_twiddle(float2 (&v)[16], float2 b0, float2 b1) {
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    float2 w;
    switch (r >> 1) {  // compile-time after unrolling
      case 0: w = (r & 1) ? b1 : b0; break;
      case 1: w = mul_w16<1>((r & 1) ? b1 : b0); break;
      case 2: w = mul_w16<2>((r & 1) ? b1 : b0); break;
      case 3: w = mul_w16<3>((r & 1) ? b1 : b0); break;
      case 4: w = mul_w16<4>((r & 1) ? b1 : b0); break;
      case 5: w = mul_w16<5>((r & 1) ? b1 : b0); break;
      case 6: w = mul_w16<6>((r & 1) ? b1 : b0); break;
      default: w = mul_w16<7>((r & 1) ? b1 : b0); break;
    }
    v[r] = cmul(v[r], w);
  }
}

// First radix-16 pass of a row from its 16 inputs (t + T r) into a padded buffer.
__device__ __forceinline__ void first_pass_regs(float2 (&v)[16], float2* dst, int tid) {
  dft16(v);
  float2* d = dst + 17 * tid;  // cpad(16 t + r) = 17 t + r
#pragma unroll
  for (int r = 0; r < 16; ++r) d[r] = v[out_pos<16>(r)];
}

}  // namespace rows
}  // namespace fxc
