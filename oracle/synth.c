/*
 * synth.c — seeded synthetic station data for the CPU legs of the benchmark.
 *
 * TEST INFRASTRUCTURE ONLY, like the rest of oracle/: the product never links
 * it.  It is not a restatement of the reference (the reference ships no data
 * generator); it writes the .raw layout the reference reads
 * (src/main.rs:445-503: headerless little-endian u32 words, codes LSB-first,
 * b bits each) from quantised Gaussian noise, as the synthetic workloads
 * describe: two stations sharing a common component at correlation rho, the
 * common part reaching station 2 `lag` whole samples later, optionally with a
 * tone of `tone_cyc` cycles per sample added to both.
 *
 * Every sample is a pure function of (seed, stream, sample index), so the
 * output does not depend on the thread count: a counter-based generator
 * (the SplitMix64 finaliser of Steele, Lea and Flood, "Fast splittable
 * pseudorandom number generators", OOPSLA 2014) feeds the Box-Muller
 * transform.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fxc_oracle.h"

static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Two independent standard normals for counter i of stream s. */
static inline void normal2(uint64_t seed, uint64_t s, uint64_t i, double* a, double* b) {
  const uint64_t k = mix64(seed ^ (s * 0xD1B54A32D192ED03ull)) ^ i;
  const uint64_t h1 = mix64(2 * k), h2 = mix64(2 * k + 1);
  const double u1 = ((double)(h1 >> 11) + 0.5) * (1.0 / 9007199254740992.0); /* (0, 1) */
  const double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
  const double r = sqrt(-2.0 * log(u1));
  const double t = 6.283185307179586 * u2;
  *a = r * cos(t);
  *b = r * sin(t);
}

/* Nearest level, first index wins ties, compared in f32 as the quantiser of
 * the test-data encoder does. */
static inline uint32_t nearest(float x, const float* lv, uint32_t n) {
  uint32_t best = 0;
  float e = fabsf(x - lv[0]);
  for (uint32_t j = 1; j < n; ++j) {
    const float d = fabsf(x - lv[j]);
    if (d < e) {
      e = d;
      best = j;
    }
  }
  return best;
}

int orc_synth_pack_pair(uint64_t seed, uint64_t nsamp, double rho, uint32_t lag,
                        double tone_amp, double tone_cyc, double tone_phase, uint32_t bits,
                        const double* levels, uint32_t nlevels, double gain,
                        const uint8_t shuffle_out1[32], int32_t lsb1,
                        const uint8_t shuffle_out2[32], int32_t lsb2, uint8_t* out1,
                        uint8_t* out2, int32_t nthreads) {
  if (!(bits == 1 || bits == 2 || bits == 4 || bits == 8) || nlevels != (1u << bits)) return -1;
  const uint32_t per = 32 / bits;
  if (nsamp % per) return -1;
  float lv[256];
  for (uint32_t j = 0; j < nlevels; ++j) lv[j] = (float)levels[j];
  const double a = sqrt(rho), b = sqrt(1.0 - rho);
  const int64_t nwords = (int64_t)(nsamp / per);
  const uint8_t* sh[2] = {shuffle_out1, shuffle_out2};
  const int32_t lsb[2] = {lsb1, lsb2};
  uint8_t* out[2] = {out1, out2};
  int ident[2];
  for (int s = 0; s < 2; ++s) {
    ident[s] = 1;
    for (int p = 0; p < 32; ++p)
      if (sh[s][p] != p) ident[s] = 0;
  }
  (void)nthreads;
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1) if (nthreads != 1)
  for (int64_t w = 0; w < nwords; ++w) {
    uint32_t word[2] = {0, 0};
    for (uint32_t j = 0; j < per; ++j) {
      const uint64_t i = (uint64_t)w * per + j;
      /* common component c at index i (station 1) and i - lag (station 2);
       * indices are offset so that i - lag never wraps */
      double c1, n1, c2, n2, unused;
      normal2(seed, 0, i + 4096, &c1, &n1);
      normal2(seed, 0, i + 4096 - lag, &c2, &unused);
      normal2(seed, 1, i, &n2, &unused);
      double x[2] = {a * c1 + b * n1, a * c2 + b * n2};
      if (tone_amp != 0.0) {
        /* the same tone at both stations; the cycle count's fraction keeps
         * the argument small for any sample index */
        const double cyc = tone_cyc * (double)i;
        const double t = tone_amp * cos(6.283185307179586 * (cyc - floor(cyc)) + tone_phase);
        x[0] += t;
        x[1] += t;
      }
      for (int s = 0; s < 2; ++s) {
        double y = x[s] * gain;
        if (lsb[s] && (i & 1)) y = -y; /* the decoder negates odd LSB samples back */
        word[s] |= nearest((float)y, lv, nlevels) << (j * bits);
      }
    }
    for (int s = 0; s < 2; ++s) {
      uint32_t v = word[s];
      if (!ident[s]) {
        uint32_t o = 0;
        for (int p = 0; p < 32; ++p) o |= ((v >> p) & 1u) << sh[s][p];
        v = o;
      }
      memcpy(out[s] + 4 * w, &v, 4);
    }
  }
  return 0;
}
