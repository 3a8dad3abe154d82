// cluster_frame.cuh — pieces shared by the kernels that run one frame pair
// per thread-block cluster (corr_cluster.cu, corr_pair.cu): the cluster
// special registers, barriers and distributed-shared-memory stores, the
// radix-C butterflies, and the decode of a CTA's column range of every
// segment of a frame from its staged words.
#pragma once

#include <stdint.h>

#include "fxc_device.cuh"

namespace fxc {
namespace clu {

constexpr int kM = 8192;  // row length
constexpr int kT = 512;   // threads per CTA

// Words of one staged region: `cw` columns of a segment plus the slack of a
// start rounded down to 16 bytes and a shift that is not a whole number of
// words (a multiple of 4 words, so every copy is 16-byte sized).
__host__ __device__ constexpr int region_words(int cw, int bits) { return cw / (32 / bits) + 4; }

__device__ __forceinline__ uint32_t cl_rank() {
  uint32_t r;
  asm("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cl_id() {
  uint32_t r;
  asm("mov.u32 %0, %%clusterid.x;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cl_count() {
  uint32_t r;
  asm("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
  return r;
}
// Split cluster barrier: every thread of every CTA of the cluster arrives;
// release / acquire order the shared-memory stores (local and remote) before it
// with the loads after it.
__device__ __forceinline__ void cl_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cl_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void cl_sync() {
  cl_arrive();
  cl_wait();
}
// Address of the same shared-memory object in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cl_map(const void* p, uint32_t rank) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  uint32_t r;
  asm("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void cl_st(uint32_t addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y)
               : "memory");
}
__device__ __forceinline__ void cl_st_u32(uint32_t addr, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

template <int C>
__device__ __forceinline__ void dft_c(float2* v) {
  if constexpr (C == 2) dft2<0>(v);
  else if constexpr (C == 4) dft4<0>(v);
  else dft8<0>(v);
}

// Inputs u in [U0, U0 + UN) of one station for thread t of a CTA that owns
// CW columns of each of the C segments: the sample m = m0 + T u + M c
// (m0 = first column + t - shift; zero outside [0, N)) into v[(u - U0) C + c]
// (.x primary, .y secondary).  Region c starts at words + c L and lw is the
// thread's word index in a region; the sample's bits are rotated into a byte
// offset of the level table (decode_tables.cuh) as in the FFT-8192 kernel.
template <int C, int CW, int U0, int UN, int BITS, bool SPLIT, bool IMAG>
__device__ __forceinline__ void cl_inputs(const uint32_t* __restrict__ words, const uint8_t* lvbase,
                                          int m0, int lw, uint32_t rots, uint32_t tbase,
                                          bool inside, float2 (&v)[16]) {
  constexpr int N = C * kM;
  constexpr int SPW = 32 / BITS;
  constexpr int L = region_words(CW, BITS);
  constexpr int USTEP = kT / SPW;
  constexpr uint32_t OMASK = ((1u << BITS) - 1u) << 2;
  static_assert(UN * C == 16 && (U0 + UN) * kT <= CW, "16 inputs per thread");
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
  auto put = [&](int i, float x) {
    if (IMAG) v[i].y = x; else v[i].x = x;
  };
  if (inside) {
    const uint32_t* w = words + lw;
#pragma unroll
    for (int u = U0; u < U0 + UN; ++u)
#pragma unroll
      for (int c = 0; c < C; ++c) put((u - U0) * C + c, level(w[c * L + u * USTEP]));
  } else {
#pragma unroll
    for (int u = U0; u < U0 + UN; ++u)
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int m = m0 + kT * u + kM * c;
        const bool in = (unsigned)m < (unsigned)N;
        const float x = level(words[in ? lw + c * L + u * USTEP : 0]);
        put((u - U0) * C + c, in ? x : 0.0f);
      }
  }
}

// The same for a station of any bit depth up to MAXBITS (2 or 8).
template <int C, int CW, int U0, int UN, int MAXBITS, bool IMAG>
__device__ __forceinline__ void cl_station(int bits, bool split, const uint32_t* words,
                                           const uint8_t* lvbase, int m0, int lw, uint32_t rots,
                                           uint32_t tbase, bool inside, float2 (&v)[16]) {
  if (bits == 1) {
    cl_inputs<C, CW, U0, UN, 1, false, IMAG>(words, lvbase, m0, lw, rots, tbase, inside, v);
  } else if (MAXBITS == 2 || bits == 2) {
    if (split) cl_inputs<C, CW, U0, UN, 2, true, IMAG>(words, lvbase, m0, lw, rots, tbase, inside, v);
    else cl_inputs<C, CW, U0, UN, 2, false, IMAG>(words, lvbase, m0, lw, rots, tbase, inside, v);
  } else if constexpr (MAXBITS == 8) {
    if (bits == 4) cl_inputs<C, CW, U0, UN, 4, false, IMAG>(words, lvbase, m0, lw, rots, tbase, inside, v);
    else cl_inputs<C, CW, U0, UN, 8, false, IMAG>(words, lvbase, m0, lw, rots, tbase, inside, v);
  }
}

__device__ __forceinline__ int log2_spw(int bits) {
  return bits == 1 ? 5 : (bits == 2 ? 4 : (bits == 4 ? 3 : 2));
}

}  // namespace clu
}  // namespace fxc
