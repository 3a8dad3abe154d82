// fold_decode.cuh — the decode of the FFT-8192 / 16384 fold kernels: a
// thread's 16 first-pass inputs of one station straight from the staged .raw
// words (corr_fold.cu, phased_pair.cu).
#pragma once

#include <stdint.h>

#include "fxc_device.cuh"

namespace fxc {
namespace fold {

constexpr int kN = 8192;  // row length

// 16 inputs of one station: x[t + r N/16 - shift] (zero outside the frame),
// r < 16, as a byte offset of the level table: rotate the word so that the
// sample's bits land at byte-offset bits 2.., mask, merge the table base
// (which also selects the negated copy for odd samples of an LSB station).
// ROWS = 2 (FFT 16384 as two 8192-point rows): input r of row 0 is
// x[m] + x[m + 8192], of row 1 x[m] - x[m + 8192] (neg_hi), m = t + 512 r - shift,
// the first radix-2 step of a decimation in frequency; the row-1 twiddle is
// applied by the caller.
template <int BITS, bool IMAG, bool SPLIT, int ROWS>
__device__ __forceinline__ void fold_inputs(const uint32_t* __restrict__ words, const uint8_t* lvbase,
                                            int shift, uint32_t rots, uint32_t tbase,
                                            float2 (&v)[16], int t, bool neg_hi) {
  constexpr int T1 = kN / 16;
  constexpr int NF = kN * ROWS;                  // frame length
  constexpr int SPW = 32 / BITS;
  constexpr int LOG2_SPW = BITS == 1 ? 5 : (BITS == 2 ? 4 : (BITS == 4 ? 3 : 2));
  constexpr int WSTEP = T1 / SPW;
  constexpr int HW = kN / SPW;                   // words of the upper half's offset
  constexpr uint32_t OMASK = ((1u << BITS) - 1u) << 2;
  static_assert(T1 % SPW == 0, "frame stride is a whole number of words");
  const int m0 = t - shift;
  const int w0 = m0 >> LOG2_SPW;  // floor division
  const uint32_t r0 = rots & 31u, r1 = (rots >> 8) & 31u;
  auto level = [&](uint32_t w) -> float {
    uint32_t off;
    if constexpr (SPLIT) {
      off = (__funnelshift_r(w, w, r0) & 4u) | tbase;
      off |= __funnelshift_r(w, w, r1) & 8u;
    } else {
      off = (__funnelshift_r(w, w, r0) & OMASK) | tbase;
    }
    return *reinterpret_cast<const float*>(lvbase + off);
  };
  // sample m (+ kN for the upper half) with the zero fill
  auto checked = [&](int r, int half) -> float {
    const int m = m0 + r * T1 + half * kN;
    const bool in = (unsigned)m < (unsigned)NF;
    const float x = level(words[in ? w0 + r * WSTEP + half * HW : 0]);
    return in ? x : 0.0f;
  };
  auto put = [&](int r, float x) {
    if (IMAG) v[r].y = x; else v[r].x = x;
  };
  const uint32_t* w = words + w0;
  if (shift == 0) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      float x = level(w[r * WSTEP]);
      if constexpr (ROWS == 2) {
        const float hi = level(w[r * WSTEP + HW]);
        x = neg_hi ? x - hi : x + hi;
      }
      put(r, x);
    }
  } else if ((unsigned)(shift + (T1 - 1)) < (unsigned)(2 * T1 - 1)) {
    // |shift| < N/16: only the first sample of the lower half and the last
    // of the upper half (or, one row, of the frame) can fall outside it
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      float x;
      if constexpr (ROWS == 1) {
        x = (r == 0 || r == 15) ? checked(r, 0) : level(w[r * WSTEP]);
      } else {
        const float lo = r == 0 ? checked(r, 0) : level(w[r * WSTEP]);
        const float hi = r == 15 ? checked(r, 1) : level(w[r * WSTEP + HW]);
        x = neg_hi ? lo - hi : lo + hi;
      }
      put(r, x);
    }
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      float x = checked(r, 0);
      if constexpr (ROWS == 2) {
        const float hi = checked(r, 1);
        x = neg_hi ? x - hi : x + hi;
      }
      put(r, x);
    }
  }
}

template <bool IMAG, int ROWS>
__device__ __forceinline__ void fold_station(int bits, bool split, const uint32_t* words,
                                             const uint8_t* lvbase, int shift, uint32_t rots,
                                             uint32_t tbase, float2 (&v)[16], int t, bool neg_hi) {
  switch (bits) {
    case 1: fold_inputs<1, IMAG, false, ROWS>(words, lvbase, shift, rots, tbase, v, t, neg_hi); break;
    case 2:
      if (split) fold_inputs<2, IMAG, true, ROWS>(words, lvbase, shift, rots, tbase, v, t, neg_hi);
      else fold_inputs<2, IMAG, false, ROWS>(words, lvbase, shift, rots, tbase, v, t, neg_hi);
      break;
    case 4: fold_inputs<4, IMAG, false, ROWS>(words, lvbase, shift, rots, tbase, v, t, neg_hi); break;
    default: fold_inputs<8, IMAG, false, ROWS>(words, lvbase, shift, rots, tbase, v, t, neg_hi); break;
  }
}

}  // namespace fold
}  // namespace fxc
