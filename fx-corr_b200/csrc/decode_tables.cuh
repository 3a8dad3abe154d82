// decode_tables.cuh — the shared-memory decode tables of the kernels that
// decode straight from staged .raw words (the FFT-8192/16384 fold kernels, the
// large-FFT staged kernels and the cluster kernel).
//
// Layout, in bytes from the start of dynamic shared memory:
//   [0, 4096)      levels: station a at 0, station b at 2048 (2^b f32 each,
//                  scaled by the station's power of two, then their negations)
//   [4096, 4352)   rotate amounts: [2 stations][32 sample slots] u32
//   [4608, 12800)  byte LUTs of 4- and 8-bit generic shuffles (2 x 1024 u32)
// A sample of word w at slot c is then the f32 at byte offset
//   (rotr(w, rot[c] & 31) & (((1 << bits) - 1) << 2)) | tbase
// of the level table, tbase selecting the station's table and its negated copy
// (odd samples of an LSB station, src/utils.rs:196-197).  A 2-bit shuffle that
// splits a sample's bits takes a second rotate (rot[c] >> 8) for the high bit.
#pragma once

#include <stdint.h>

#include "fxc_device.cuh"

namespace fxc {

constexpr uint32_t kTabPos = 4096, kTabLut = 4608, kTabEnd = kTabLut + 8192;

// Builds the tables of stations a and b (needs a barrier before use).
// preA / preB: the station's words are rewritten in place by its byte LUTs
// before decoding (4- and 8-bit stations with a non-identity shuffle), so its
// rotate amounts are those of the natural bit order.
__device__ __forceinline__ void build_decode_tables(const StationParams& sa, const StationParams& sb,
                                                    bool preA, bool preB, uint8_t* smem, int tid,
                                                    int nthreads) {
  float* lv = reinterpret_cast<float*>(smem);
  uint32_t* pos = reinterpret_cast<uint32_t*>(smem + kTabPos);
  uint32_t* lut = reinterpret_cast<uint32_t*>(smem + kTabLut);
  for (int i = tid; i < 1024; i += nthreads) {
    // per station: 2^b levels, then their negations (the two sign groups of a
    // warp's table loads fall in different banks)
    const StationParams& q = (i < 512) ? sa : sb;
    const int n = 1 << q.bits, c2 = i & 511;
    const float x = c2 < 2 * n ? q.levels[c2 & (n - 1)] * q.scale : 0.0f;
    lv[i] = c2 >= n ? -x : x;
  }
  for (int i = tid; i < 64; i += nthreads) {
    // rotate amounts of sample slot c: bit j of the sample is word bit p_j
    const int k = i >> 5, cc = i & 31;
    const StationParams& q = k ? sb : sa;
    const int b = q.bits;
    const bool natural = (k ? preB : preA) || q.shkind == SH_IDENTITY;
    uint32_t r = 0;
    if (cc * b < 32) {
      const int p0 = natural ? cc * b : q.perm[cc * b];
      const int p1 = b >= 2 ? (natural ? cc * b + 1 : q.perm[cc * b + 1]) : 0;
      r = (uint32_t)((p0 - 2) & 31) | ((uint32_t)((p1 - 3) & 31) << 8);
    }
    pos[i] = r;
  }
  for (int k = 0; k < 2; ++k) {
    const StationParams& q = k ? sb : sa;
    if ((k ? preB : preA) && q.shkind == SH_GENERIC)
      for (int i = tid; i < 1024; i += nthreads) lut[k * 1024 + i] = q.shlut[i];
  }
}

// A 2-bit shuffle keeps every sample's two bits adjacent and in order, or it
// splits them (two rotates per sample).
__device__ __forceinline__ bool split_2bit(const StationParams& q) {
  if (q.bits != 2 || q.shkind == SH_IDENTITY) return false;
  for (int cc = 0; cc < 16; ++cc)
    if (q.perm[2 * cc + 1] != q.perm[2 * cc] + 1 || (q.perm[2 * cc] & 1)) return true;
  return false;
}

}  // namespace fxc
