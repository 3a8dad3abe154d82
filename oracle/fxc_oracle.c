/*
 * fxc_oracle.c — CPU restatement of the fx-corr correlation path.
 *
 * TEST INFRASTRUCTURE ONLY (see fxc_oracle.h).  The product never links this.
 * Parity status: UNPINNED by reference-produced vectors (the Rust reference
 * cannot be built here); pinned instead by the hand-derived known-answer
 * vectors in tests/golden and by the FP64 NumPy oracle in oracle/oracle.py.
 *
 * Reference file:line citations are relative to the fx-corr project root.
 */
#include "fxc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

typedef struct {
  float re, im;
} cf32;

static inline cf32 cmul(cf32 a, cf32 b) {
  /* num-complex 0.4 Mul: (ac - bd, ad + bc), no fused multiply-add */
  cf32 r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}
static inline cf32 cconj(cf32 a) {
  a.im = -a.im;
  return a;
}
static inline cf32 cpolar(float theta) {
  /* Complex::from_polar(1.0_f32, theta) = (1*cos, 1*sin) */
  cf32 r;
  r.re = 1.0f * cosf(theta);
  r.im = 1.0f * sinf(theta);
  return r;
}
static inline float cnorm2(cf32 a) { return a.re * a.re + a.im * a.im; }

/* ---------------------------------------------------------------- shuffle */

int orc_parse_shuffle(const int32_t ext[32], uint8_t internal[32]) {
  /* args.rs:202-210 — must be a permutation of 0..31; internal[31-idx] = ext[idx] */
  int seen[32] = {0};
  for (int i = 0; i < 32; ++i) {
    if (ext[i] < 0 || ext[i] > 31 || seen[ext[i]]) return -1;
    seen[ext[i]] = 1;
  }
  for (int idx = 0; idx < 32; ++idx) internal[31 - idx] = (uint8_t)ext[idx];
  return 0;
}

enum { SH_IDENTITY = 0, SH_PAIRSWAP = 1, SH_GENERIC = 2 };

static int shuffle_kind(const uint8_t sh[32]) {
  /* utils.rs:176-178 */
  int ident = 1, pair = 1;
  for (int i = 0; i < 32; ++i) {
    if (sh[i] != i) ident = 0;
    if (sh[i] != (i ^ 1)) pair = 0;
  }
  return ident ? SH_IDENTITY : (pair ? SH_PAIRSWAP : SH_GENERIC);
}

static inline uint32_t apply_shuffle(uint32_t w, const uint8_t sh[32], int kind) {
  /* utils.rs:159-171 */
  if (kind == SH_PAIRSWAP) {
    w = ((w & 0xAAAAAAAAu) >> 1) | ((w & 0x55555555u) << 1);
  } else if (kind == SH_GENERIC) {
    uint32_t s = 0;
    for (int o = 0; o < 32; ++o) s |= ((w >> sh[o]) & 1u) << o;
    w = s;
  }
  return w;
}

static inline uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

/* ----------------------------------------------------------------- decode */

int64_t orc_decode(const uint8_t* raw, uint64_t raw_len, uint64_t samples, uint32_t bits,
                   const uint8_t shuffle[32], const double* levels, uint32_t nlevels,
                   int32_t lsb_to_usb, float* out) {
  /* utils.rs:215-376 (with build_decode_plan, utils.rs:173-213) */
  if (bits < 1 || bits > 8 || nlevels != (1u << bits)) return -1;
  float lv[256];
  for (uint32_t i = 0; i < nlevels; ++i) lv[i] = (float)levels[i];
  const int kind = shuffle_kind(shuffle);
  uint64_t oi = 0;
  int odd = 0;
  const uint64_t nwords = raw_len / 4; /* chunks_exact(4) drops a ragged tail */
#define EMIT(code_expr)                          \
  do {                                           \
    float v_ = lv[(code_expr)];                  \
    if (lsb_to_usb && odd) v_ = -v_;             \
    out[oi++] = v_;                              \
    odd = !odd;                                  \
  } while (0)
  if (bits == 2 && kind == SH_IDENTITY) {
    /* utils.rs:248-299: 16-bit LUT over byte pairs, tail path, remainder byte */
    const uint64_t npairs = raw_len / 2;
    for (uint64_t p = 0; p < npairs; ++p) {
      uint32_t w = (uint32_t)raw[2 * p] | ((uint32_t)raw[2 * p + 1] << 8);
      if (oi + 8 <= samples) {
        /* LUT entry i flips when (i & 1); oi is a multiple of 8 here */
        for (int i = 0; i < 8; ++i) {
          float v = lv[(w >> (2 * i)) & 3u];
          if (lsb_to_usb && (i & 1)) v = -v;
          out[oi + i] = v;
        }
        oi += 8;
      } else {
        for (int i = 0; i < 8; ++i) {
          if (oi >= samples) break;
          EMIT(w & 3u);
          w >>= 2;
        }
      }
    }
    if (raw_len & 1) {
      uint32_t b = raw[raw_len - 1];
      for (int i = 0; i < 4; ++i) {
        if (oi >= samples) break;
        EMIT(b & 3u);
        b >>= 2;
      }
    }
  } else if (bits == 1 || bits == 2 || bits == 4 || bits == 8) {
    const uint32_t per = 32 / bits, mask = (1u << bits) - 1u;
    for (uint64_t c = 0; c < nwords; ++c) {
      uint32_t w = apply_shuffle(le32(raw + 4 * c), shuffle, kind);
      for (uint32_t i = 0; i < per; ++i) {
        if (oi >= samples) break;
        EMIT(w & mask);
        w >>= bits;
      }
    }
  } else {
    /* utils.rs:349-369 generic bit accumulator */
    const uint64_t mask = (1ull << bits) - 1ull;
    uint64_t acc = 0;
    uint32_t acc_bits = 0;
    for (uint64_t c = 0; c < nwords; ++c) {
      uint32_t w = apply_shuffle(le32(raw + 4 * c), shuffle, kind);
      acc |= (uint64_t)w << acc_bits;
      acc_bits += 32;
      while (acc_bits >= bits && oi < samples) {
        EMIT((uint32_t)(acc & mask));
        acc_bits -= bits;
        acc >>= bits;
      }
    }
  }
#undef EMIT
  if (oi != samples) return -1; /* utils.rs:372-374 */
  return (int64_t)oi;
}

void orc_shift_zerofill(float* x, uint64_t n, int64_t s) {
  /* utils.rs:126-145 */
  if (n == 0 || s == 0) return;
  uint64_t a = s < 0 ? (uint64_t)(-(s + 1)) + 1u : (uint64_t)s;
  if (a >= n) {
    memset(x, 0, n * sizeof(float));
    return;
  }
  if (s > 0) {
    memmove(x + a, x, (n - a) * sizeof(float));
    memset(x, 0, a * sizeof(float));
  } else {
    memmove(x, x + a, (n - a) * sizeof(float));
    memset(x + (n - a), 0, a * sizeof(float));
  }
}

/* -------------------------------------------------------------------- FFT */
/* Complex Stockham autosort FFT (radix 4, final radix 2), f32 data, twiddles
 * rounded from f64.  Restates the DFT X[k] = sum x[n] exp(-2 pi i k n / N)
 * that rustfft computes; operation order differs from rustfft's. */

typedef struct {
  uint32_t n;
  int npass;
  int radix[40];
  uint32_t ns[40];
  cf32* tw[40];
  float* twr[40]; /* the same twiddles split: [(q - 1) * ns + k] */
  float* twi[40];
  cf32* post; /* real-FFT split twiddles exp(-2 pi i k / (2n)), k < n */
} cfft_plan;

static cfft_plan* g_plans[40];

static cfft_plan* plan_get(uint32_t n) {
  int lg = 0;
  while ((1u << lg) < n) ++lg;
  if ((1u << lg) != n) return NULL;
  cfft_plan* p = __atomic_load_n(&g_plans[lg], __ATOMIC_ACQUIRE);
  if (p) return p;
  p = (cfft_plan*)calloc(1, sizeof(cfft_plan));
  p->n = n;
  uint32_t rem = n, ns = 1;
  while (rem > 1) {
    int r = (rem % 4 == 0) ? 4 : 2;
    p->radix[p->npass] = r;
    p->ns[p->npass] = ns;
    cf32* tw = (cf32*)malloc(sizeof(cf32) * (size_t)ns * (size_t)(r - 1) + sizeof(cf32));
    float* twr = (float*)malloc(sizeof(float) * ((size_t)ns * (size_t)(r - 1) + 1));
    float* twi = (float*)malloc(sizeof(float) * ((size_t)ns * (size_t)(r - 1) + 1));
    for (uint32_t k = 0; k < ns; ++k)
      for (int q = 1; q < r; ++q) {
        double ang = -2.0 * ORC_PI * (double)k * (double)q / ((double)ns * (double)r);
        tw[k * (r - 1) + (q - 1)].re = (float)cos(ang);
        tw[k * (r - 1) + (q - 1)].im = (float)sin(ang);
        twr[(size_t)(q - 1) * ns + k] = tw[k * (r - 1) + (q - 1)].re;
        twi[(size_t)(q - 1) * ns + k] = tw[k * (r - 1) + (q - 1)].im;
      }
    p->twr[p->npass] = twr;
    p->twi[p->npass] = twi;
    p->tw[p->npass++] = tw;
    ns *= (uint32_t)r;
    rem /= (uint32_t)r;
  }
  p->post = (cf32*)malloc(sizeof(cf32) * ((size_t)n + 1));
  for (uint32_t k = 0; k <= n; ++k) {
    double ang = -2.0 * ORC_PI * (double)k / (2.0 * (double)n);
    p->post[k].re = (float)cos(ang);
    p->post[k].im = (float)sin(ang);
  }
  cfft_plan* expected = NULL;
  if (!__atomic_compare_exchange_n(&g_plans[lg], &expected, p, 0, __ATOMIC_ACQ_REL,
                                   __ATOMIC_ACQUIRE)) {
    return expected; /* another thread won; leak ours (test code) */
  }
  return p;
}

/* Forward complex FFT of a[0..n); b is scratch of n; returns the buffer that
 * holds the result (a or b). */
static cf32* cfft_forward(const cfft_plan* p, cf32* a, cf32* b) {
  const uint32_t n = p->n;
  cf32* in = a;
  cf32* out = b;
  for (int ps = 0; ps < p->npass; ++ps) {
    const int r = p->radix[ps];
    const uint32_t ns = p->ns[ps];
    const uint32_t stride = n / (uint32_t)r;
    const cf32* tw = p->tw[ps];
    for (uint32_t blk = 0; blk < stride / ns; ++blk) {
      for (uint32_t k = 0; k < ns; ++k) {
        const uint32_t j = blk * ns + k;
        const uint32_t od = blk * ns * (uint32_t)r + k;
        if (r == 4) {
          cf32 v0 = in[j], v1 = in[j + stride], v2 = in[j + 2 * stride], v3 = in[j + 3 * stride];
          if (ns > 1) {
            v1 = cmul(v1, tw[k * 3 + 0]);
            v2 = cmul(v2, tw[k * 3 + 1]);
            v3 = cmul(v3, tw[k * 3 + 2]);
          }
          cf32 t0 = {v0.re + v2.re, v0.im + v2.im};
          cf32 t1 = {v0.re - v2.re, v0.im - v2.im};
          cf32 t2 = {v1.re + v3.re, v1.im + v3.im};
          cf32 t3 = {v1.im - v3.im, v3.re - v1.re}; /* (v1 - v3) * (-i) */
          out[od] = (cf32){t0.re + t2.re, t0.im + t2.im};
          out[od + ns] = (cf32){t1.re + t3.re, t1.im + t3.im};
          out[od + 2 * ns] = (cf32){t0.re - t2.re, t0.im - t2.im};
          out[od + 3 * ns] = (cf32){t1.re - t3.re, t1.im - t3.im};
        } else {
          cf32 v0 = in[j], v1 = in[j + stride];
          if (ns > 1) v1 = cmul(v1, tw[k]);
          out[od] = (cf32){v0.re + v1.re, v0.im + v1.im};
          out[od + ns] = (cf32){v0.re - v1.re, v0.im - v1.im};
        }
      }
    }
    cf32* t = in;
    in = out;
    out = t;
  }
  return in;
}

/* One radix-4 pass of cfft_forward on split (re, im) arrays: every
 * operation and its order are those of cfft_forward, so the results are
 * identical bit for bit.  The innermost loop walks k, the position inside a
 * block of ns outputs, contiguously in its inputs and outputs (vectorised
 * for ns >= 8); the first pass (ns = 1, no twiddles) loops over blocks. */
static void pass4_split(size_t n, size_t ns, const float* restrict inr,
                        const float* restrict ini, float* restrict outr, float* restrict outi,
                        const float* restrict wr, const float* restrict wi) {
  const size_t stride = n / 4;
  if (ns == 1) {
    for (size_t j = 0; j < stride; ++j) {
      const float v0r = inr[j], v0i = ini[j], v1r = inr[j + stride], v1i = ini[j + stride];
      const float v2r = inr[j + 2 * stride], v2i = ini[j + 2 * stride];
      const float v3r = inr[j + 3 * stride], v3i = ini[j + 3 * stride];
      const float t0r = v0r + v2r, t0i = v0i + v2i;
      const float t1r = v0r - v2r, t1i = v0i - v2i;
      const float t2r = v1r + v3r, t2i = v1i + v3i;
      const float t3r = v1i - v3i, t3i = v3r - v1r; /* (v1 - v3) * (-i) */
      outr[4 * j] = t0r + t2r;
      outi[4 * j] = t0i + t2i;
      outr[4 * j + 1] = t1r + t3r;
      outi[4 * j + 1] = t1i + t3i;
      outr[4 * j + 2] = t0r - t2r;
      outi[4 * j + 2] = t0i - t2i;
      outr[4 * j + 3] = t1r - t3r;
      outi[4 * j + 3] = t1i - t3i;
    }
    return;
  }
  for (size_t blk = 0; blk < stride / ns; ++blk) {
    const size_t j = blk * ns, od = blk * ns * 4;
#pragma GCC ivdep
    for (size_t k = 0; k < ns; ++k) {
      const float v0r = inr[j + k], v0i = ini[j + k];
      const float a1r = inr[j + k + stride], a1i = ini[j + k + stride];
      const float a2r = inr[j + k + 2 * stride], a2i = ini[j + k + 2 * stride];
      const float a3r = inr[j + k + 3 * stride], a3i = ini[j + k + 3 * stride];
      const float v1r = a1r * wr[k] - a1i * wi[k];
      const float v1i = a1r * wi[k] + a1i * wr[k];
      const float v2r = a2r * wr[ns + k] - a2i * wi[ns + k];
      const float v2i = a2r * wi[ns + k] + a2i * wr[ns + k];
      const float v3r = a3r * wr[2 * ns + k] - a3i * wi[2 * ns + k];
      const float v3i = a3r * wi[2 * ns + k] + a3i * wr[2 * ns + k];
      const float t0r = v0r + v2r, t0i = v0i + v2i;
      const float t1r = v0r - v2r, t1i = v0i - v2i;
      const float t2r = v1r + v3r, t2i = v1i + v3i;
      const float t3r = v1i - v3i, t3i = v3r - v1r; /* (v1 - v3) * (-i) */
      outr[od + k] = t0r + t2r;
      outi[od + k] = t0i + t2i;
      outr[od + ns + k] = t1r + t3r;
      outi[od + ns + k] = t1i + t3i;
      outr[od + 2 * ns + k] = t0r - t2r;
      outi[od + 2 * ns + k] = t0i - t2i;
      outr[od + 3 * ns + k] = t1r - t3r;
      outi[od + 3 * ns + k] = t1i - t3i;
    }
  }
}

/* The final radix-2 pass (odd log2 n) of cfft_forward on split arrays. */
static void pass2_split(size_t n, size_t ns, const float* restrict inr,
                        const float* restrict ini, float* restrict outr, float* restrict outi,
                        const float* restrict wr, const float* restrict wi) {
  const size_t stride = n / 2;
  for (size_t blk = 0; blk < stride / ns; ++blk) {
    const size_t j = blk * ns, od = blk * ns * 2;
    for (size_t k = 0; k < ns; ++k) {
      const float v0r = inr[j + k], v0i = ini[j + k];
      float v1r = inr[j + k + stride], v1i = ini[j + k + stride];
      if (ns > 1) {
        const float ar1 = v1r, ai1 = v1i;
        v1r = ar1 * wr[k] - ai1 * wi[k];
        v1i = ar1 * wi[k] + ai1 * wr[k];
      }
      outr[od + k] = v0r + v1r;
      outi[od + k] = v0i + v1i;
      outr[od + k + ns] = v0r - v1r;
      outi[od + k + ns] = v0i - v1i;
    }
  }
}

/* cfft_forward on split (re, im) arrays; returns the pair holding the result. */
static void cfft_forward_split(const cfft_plan* p, float* ar, float* ai, float* br, float* bi,
                               float** zr, float** zi) {
  float* inr = ar;
  float* ini = ai;
  float* outr = br;
  float* outi = bi;
  for (int ps = 0; ps < p->npass; ++ps) {
    if (p->radix[ps] == 4)
      pass4_split(p->n, p->ns[ps], inr, ini, outr, outi, p->twr[ps], p->twi[ps]);
    else
      pass2_split(p->n, p->ns[ps], inr, ini, outr, outi, p->twr[ps], p->twi[ps]);
    float* t = inr;
    inr = outr;
    outr = t;
    t = ini;
    ini = outi;
    outi = t;
  }
  *zr = inr;
  *zi = ini;
}

/* Bin k of the real FFT from the half-length complex FFT z (split arrays):
 * E = (Z[kk] + conj Z[kc]) / 2, O = (Z[kk] - conj Z[kc]) / (2i), X[k] = E + w^k O. */
static inline void split_bins(const float* restrict zr, const float* restrict zi,
                              const cf32* restrict post, size_t m, size_t k, size_t kk, size_t kc,
                              float* restrict out) {
  (void)m;
  const float zkr = zr[kk], zki = zi[kk];
  const float zcr = zr[kc], zci = -zi[kc];
  const float er = 0.5f * (zkr + zcr), ei = 0.5f * (zki + zci);
  const float dr = zkr - zcr, di = zki - zci;
  const float orr = 0.5f * di, oi = -0.5f * dr; /* d / (2i) */
  const float wor = post[k].re * orr - post[k].im * oi;
  const float woi = post[k].re * oi + post[k].im * orr;
  out[2 * k] = er + wor;
  out[2 * k + 1] = ei + woi;
}

/* Per-thread scratch of the real FFT (test infrastructure: kept until exit). */
static __thread float* g_rfft_buf = NULL;
static __thread size_t g_rfft_cap = 0;

int orc_rfft_f32(uint32_t n, const float* in, float* out) {
  /* realfft R2C via an n/2-point complex FFT of (x[2m], x[2m+1]) and the
   * even/odd split X[k] = E[k] + exp(-2 pi i k / n) O[k], k = 0..n/2. */
  if (n < 2 || (n & (n - 1))) return -1;
  const uint32_t m = n / 2;
  cfft_plan* p = plan_get(m);
  if (!p) return -1;
  if (g_rfft_cap < 4 * (size_t)m) {
    free(g_rfft_buf);
    g_rfft_buf = (float*)malloc(sizeof(float) * 4 * (size_t)m);
    if (!g_rfft_buf) {
      g_rfft_cap = 0;
      return -1;
    }
    g_rfft_cap = 4 * (size_t)m;
  }
  float* ar = g_rfft_buf;
  float* ai = ar + m;
  float* br = ai + m;
  float* bi = br + m;
  for (uint32_t i = 0; i < m; ++i) {
    ar[i] = in[2 * i];
    ai[i] = in[2 * i + 1];
  }
  float *zr, *zi;
  cfft_forward_split(p, ar, ai, br, bi, &zr, &zi);
  /* X[k] from Z[k mod m] and conj Z[(m - k) mod m]: k = 0 and k = m both pair
   * Z[0] with itself, 0 < k < m pairs Z[k] with Z[m - k] */
  const cf32* restrict post = p->post;
  split_bins(zr, zi, post, m, 0, 0, 0, out);
  for (size_t k = 1; k < m; ++k) split_bins(zr, zi, post, m, k, k, m - k, out);
  split_bins(zr, zi, post, m, m, 0, 0, out);
  return 0;
}

int orc_irfft_f32(uint32_t n, const float* in, float* out) {
  /* realfft C2R (unnormalised) then * (1/n) as utils.rs:60-66 */
  if (n < 2 || (n & (n - 1))) return -1;
  const uint32_t m = n / 2;
  cfft_plan* p = plan_get(m);
  if (!p) return -1;
  cf32* a = (cf32*)malloc(sizeof(cf32) * m * 2);
  cf32* b = a + m;
  for (uint32_t k = 0; k < m; ++k) {
    cf32 xk = {in[2 * k], (k == 0) ? 0.0f : in[2 * k + 1]};
    uint32_t mk = m - k;
    cf32 xm = {in[2 * mk], (mk == m || mk == 0) ? 0.0f : in[2 * mk + 1]};
    cf32 xmc = cconj(xm);
    cf32 e = {xk.re + xmc.re, xk.im + xmc.im};
    cf32 d = {xk.re - xmc.re, xk.im - xmc.im};
    cf32 o = cmul(d, cconj(p->post[k]));
    /* Z = E + i O, conjugated for the inverse-by-forward trick */
    a[k].re = e.re - o.im;
    a[k].im = -(e.im + o.re);
  }
  cf32* z = cfft_forward(p, a, b);
  const float scale = 1.0f / (float)n;
  for (uint32_t i = 0; i < m; ++i) {
    out[2 * i] = z[i].re * scale;
    out[2 * i + 1] = -z[i].im * scale;
  }
  free(a);
  return 0;
}

/* ----------------------------------------------------------- delay model */

static inline int64_t f64_as_i64(double v) {
  /* Rust `as i64`: saturating, NaN -> 0 */
  if (v != v) return 0;
  if (v >= 9223372036854775807.0) return INT64_MAX;
  if (v <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)v;
}
static inline double rem_euclid(double x, double r) {
  double m = fmod(x, r);
  return m < 0.0 ? m + fabs(r) : m;
}

static void split_delay(double tau, double fs, int64_t* ip, double* fp) {
  /* main.rs:126-130 */
  int64_t i = f64_as_i64(round(tau * fs));
  *ip = i;
  *fp = tau - ((double)i / fs);
}

static void carrier_phase(double f_hz, double tau_s, float out[2]) {
  /* main.rs:110-120 */
  if (f_hz == 0.0) {
    out[0] = 1.0f;
    out[1] = 0.0f;
    return;
  }
  const double two_pi = 2.0 * ORC_PI;
  const double phase = -two_pi * f_hz * tau_s;
  const double wrapped = rem_euclid(phase + ORC_PI, two_pi) - ORC_PI;
  cf32 c = cpolar((float)wrapped);
  out[0] = c.re;
  out[1] = c.im;
}

void orc_delay_entry(const orc_delay_cfg* cfg, uint64_t frame_idx, orc_frame_delay* out) {
  /* main.rs:184-241 */
  const double t_mid_local = ((double)frame_idx + 0.5) * cfg->frame_dt;
  const double t_mid = t_mid_local + cfg->time_offset_s;
  double tau1, tau2, tau1_fr, tau2_fr;
  if (cfg->geom_table) {
    const uint64_t len = cfg->geom_len;
    const uint64_t last = len > 0 ? len - 1 : 0;
    double fl = floor(t_mid_local);
    if (!(fl > 0.0)) fl = 0.0; /* .max(0.0), NaN -> 0 */
    uint64_t sec_idx = fl >= 18446744073709551615.0 ? UINT64_MAX : (uint64_t)fl;
    uint64_t i0 = sec_idx < last ? sec_idx : last;
    uint64_t i1 = (i0 + 1) < last ? (i0 + 1) : last;
    double frac = 0.0;
    if (i1 != i0) {
      frac = t_mid_local - (double)i0;
      if (frac < 0.0) frac = 0.0;
      if (frac > 1.0) frac = 1.0;
    }
    const double gd_t = cfg->geom_table[i0] * (1.0 - frac) + cfg->geom_table[i1] * frac;
    const double net = gd_t + cfg->coarse_delay_s + cfg->delay_user_samples / cfg->fs +
                       cfg->extra_delay_rate_sps * t_mid;
    const double c1 = cfg->clock1_delay_s + cfg->clock1_rate_sps * t_mid;
    const double c2 = cfg->clock2_delay_s + cfg->clock2_rate_sps * t_mid;
    const double rel = c2 - c1;
    const double full = net + rel;
    tau1 = full - cfg->d_seek;
    tau2 = 0.0;
    tau1_fr = full;
    tau2_fr = 0.0;
  } else {
    /* main.rs:122-124 delay_seconds_at_time */
    tau1 = cfg->net_d1_base + cfg->total_rate1_base * t_mid +
           0.5 * cfg->total_accel1_base * (t_mid * t_mid);
    tau2 = cfg->net_d2_base + cfg->total_rate2_base * t_mid +
           0.5 * cfg->total_accel2_base * (t_mid * t_mid);
    tau1_fr = tau1 + cfg->d_seek;
    tau2_fr = tau2;
  }
  split_delay(tau1, cfg->fs, &out->int1, &out->frac1);
  split_delay(tau2, cfg->fs, &out->int2, &out->frac2);
  carrier_phase(cfg->lo1_hz, tau1_fr, out->fr_lo1);
  carrier_phase(cfg->lo2_hz, tau2_fr, out->fr_lo2);
}

int orc_band_alignment(uint32_t fft, double fs, double c1, double c2, double bw1, double bw2,
                       int64_t out[4]) {
  /* main.rs:363-372 */
  const double df = fs / (double)fft;
  const uint64_t h = fft / 2 + 1;
  const uint64_t lim = (fft % 2 == 0) ? h - 1 : h;
  double q1 = floor((bw1 * 1e6) / df), q2 = floor((bw2 * 1e6) / df);
  uint64_t v1 = (q1 > 0.0 ? (uint64_t)q1 : 0) + 1;
  uint64_t v2 = (q2 > 0.0 ? (uint64_t)q2 : 0) + 1;
  if (v1 > lim) v1 = lim;
  if (v2 > lim) v2 = lim;
  const double sr = (c1 * 1e6 - c2 * 1e6) / df;
  const int64_t sb = f64_as_i64(round(sr));
  const int64_t a1s = (-sb) > 0 ? -sb : 0;
  const int64_t a1e_i = (int64_t)v1 < ((int64_t)v2 - sb) ? (int64_t)v1 : ((int64_t)v2 - sb);
  if (a1e_i <= a1s) return -1;
  out[0] = sb;
  out[1] = a1s;
  out[2] = a1e_i;
  out[3] = a1s + sb;
  return 0;
}

void orc_xcf_phase_start_and_step(double df_hz, double frac1, double frac2, uint64_t a1s,
                                  uint64_t a2s, float out[4]) {
  /* main.rs:132-149 */
  const double two_pi_df = -2.0 * ORC_PI * df_hz;
  const double step1 = two_pi_df * frac1;
  const double step2 = two_pi_df * frac2;
  cf32 s = cpolar((float)(step1 * (double)a1s - step2 * (double)a2s));
  cf32 t = cpolar((float)(step1 - step2));
  out[0] = s.re;
  out[1] = s.im;
  out[2] = t.re;
  out[3] = t.im;
}

/* ------------------------------------------------------------ quantise */

int64_t orc_quantise_frame(const float* samples, uint64_t n, uint32_t bits, const double* levels,
                           uint32_t nlevels, const uint8_t shuffle_out[32], uint8_t* out,
                           uint64_t out_cap) {
  /* utils.rs:378-410 */
  if (bits < 1 || bits > 32) return -1;
  const uint64_t mask = (bits >= 64) ? ~0ull : ((1ull << bits) - 1ull);
  uint64_t acc = 0;
  uint32_t acc_bits = 0;
  uint64_t ow = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const float val = samples[i];
    uint32_t best = 0;
    float min_err = 3.40282347e38f;
    for (uint32_t l = 0; l < nlevels; ++l) {
      float err = fabsf(val - (float)levels[l]);
      if (err < min_err) {
        min_err = err;
        best = l;
      }
    }
    acc |= ((uint64_t)best & mask) << acc_bits;
    acc_bits += bits;
    while (acc_bits >= 32) {
      uint32_t w = (uint32_t)(acc & 0xFFFFFFFFull), s = 0;
      for (int pos = 0; pos < 32; ++pos) s |= ((w >> pos) & 1u) << shuffle_out[pos];
      if (ow + 4 > out_cap) return -1;
      out[ow] = (uint8_t)s;
      out[ow + 1] = (uint8_t)(s >> 8);
      out[ow + 2] = (uint8_t)(s >> 16);
      out[ow + 3] = (uint8_t)(s >> 24);
      ow += 4;
      acc >>= 32;
      acc_bits -= 32;
    }
  }
  if (acc_bits > 0) {
    uint32_t w = (uint32_t)(acc & 0xFFFFFFFFull), s = 0;
    for (int pos = 0; pos < 32; ++pos) s |= ((w >> pos) & 1u) << shuffle_out[pos];
    if (ow + 4 > out_cap) return -1;
    out[ow] = (uint8_t)s;
    out[ow + 1] = (uint8_t)(s >> 8);
    out[ow + 2] = (uint8_t)(s >> 16);
    out[ow + 3] = (uint8_t)(s >> 24);
    ow += 4;
  }
  return (int64_t)ow;
}

/* ------------------------------------------------------- sector: corr path */

static uint64_t bytes_per_frame(uint32_t n, uint32_t bits) {
  return ((uint64_t)n * bits + 7) / 8; /* main.rs:1214-1215 */
}

int64_t orc_sector_corr(const orc_scan_cfg* cfg, const uint8_t* raw1, const uint8_t* raw2,
                        uint64_t nf, uint64_t first_frame, double* acc11, double* acc22,
                        double* acc12, int32_t nthreads) {
  /* main.rs:2413-2591 (rayon map/reduce -> OpenMP per-thread accumulators
   * reduced in thread order). */
  const uint32_t n = cfg->fft_len;
  const uint64_t h = n / 2 + 1;
  const uint64_t bpf1 = bytes_per_frame(n, cfg->bits1), bpf2 = bytes_per_frame(n, cfg->bits2);
  const double df_hz = cfg->fs_hz / (double)n;
  const uint64_t ov = cfg->a1e - cfg->a1s;
  const int need_acf = (cfg->products & ORC_PROD_ACF) != 0;
  const int need_xcf = (cfg->products & ORC_PROD_XCF) != 0;
  const int overlap_only = (cfg->products & ORC_PROD_ACF_OVERLAP_ONLY) != 0;
  memset(acc11, 0, h * sizeof(double));
  memset(acc22, 0, h * sizeof(double));
  memset(acc12, 0, 2 * h * sizeof(double));
  if (!plan_get(n / 2)) return -1;
  int nt = 1;
#ifdef _OPENMP
  nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
  double* part = (double*)calloc((size_t)nt * 4 * h, sizeof(double));
  int64_t failed = 0;
#pragma omp parallel num_threads(nt) reduction(+ : failed)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* p11 = part + (size_t)tid * 4 * h;
    double* p22 = p11 + h;
    double* p12 = p22 + h;
    float* f1 = (float*)malloc(sizeof(float) * n);
    float* f2 = (float*)malloc(sizeof(float) * n);
    cf32* s1 = (cf32*)malloc(sizeof(cf32) * h);
    cf32* s2 = (cf32*)malloc(sizeof(cf32) * h);
#pragma omp for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nf; ++ii) {
      const uint64_t i = (uint64_t)ii;
      orc_frame_delay d;
      orc_delay_entry(&cfg->delay, first_frame + i, &d);
      if (orc_decode(raw1 + i * bpf1, bpf1, n, cfg->bits1, cfg->shuffle1, cfg->levels1,
                     cfg->nlevels1, cfg->lsb1, f1) < 0) {
        failed++;
        continue;
      }
      if (orc_decode(raw2 + i * bpf2, bpf2, n, cfg->bits2, cfg->shuffle2, cfg->levels2,
                     cfg->nlevels2, cfg->lsb2, f2) < 0) {
        failed++;
        continue;
      }
      orc_shift_zerofill(f1, n, d.int1);
      orc_shift_zerofill(f2, n, d.int2);
      orc_rfft_f32(n, f1, (float*)s1);
      orc_rfft_f32(n, f2, (float*)s2);
      const cf32 lo1 = {d.fr_lo1[0], d.fr_lo1[1]}, lo2 = {d.fr_lo2[0], d.fr_lo2[1]};
      const cf32 fr_mix = cmul(lo1, cconj(lo2));
      float ph[4];
      if (cfg->grid == 0) {
        if (need_acf) {
          if (overlap_only) {
            for (uint64_t k = 0; k < ov; ++k) {
              p11[cfg->a1s + k] += (double)cnorm2(s1[cfg->a1s + k]);
              p22[cfg->a1s + k] += (double)cnorm2(s2[cfg->a2s + k]);
            }
          } else {
            for (uint64_t k = 0; k < h; ++k) p11[k] += (double)cnorm2(s1[k]);
            for (uint64_t k = 0; k < ov; ++k) p22[cfg->a1s + k] += (double)cnorm2(s2[cfg->a2s + k]);
          }
        }
        if (need_xcf) {
          orc_xcf_phase_start_and_step(df_hz, d.frac1, d.frac2, cfg->a1s, cfg->a2s, ph);
          cf32 pc = {ph[0], ph[1]};
          const cf32 st = {ph[2], ph[3]};
          for (uint64_t k = 0; k < ov; ++k) {
            const uint64_t i1 = cfg->a1s + k, i2 = cfg->a2s + k;
            cf32 v = cmul(cmul(cmul(s1[i1], cconj(s2[i2])), fr_mix), pc);
            p12[2 * i1] += (double)v.re;
            p12[2 * i1 + 1] += (double)v.im;
            pc = cmul(pc, st);
          }
        }
      } else {
        if (need_acf) {
          if (overlap_only) {
            for (uint64_t k = 0; k < ov; ++k) {
              p11[cfg->a2s + k] += (double)cnorm2(s1[cfg->a1s + k]);
              p22[cfg->a2s + k] += (double)cnorm2(s2[cfg->a2s + k]);
            }
          } else {
            for (uint64_t k = 0; k < h; ++k) p22[k] += (double)cnorm2(s2[k]);
            for (uint64_t k = 0; k < ov; ++k) p11[cfg->a2s + k] += (double)cnorm2(s1[cfg->a1s + k]);
          }
        }
        if (need_xcf) {
          orc_xcf_phase_start_and_step(df_hz, d.frac1, d.frac2, cfg->a1s, cfg->a2s, ph);
          cf32 pc = {ph[0], ph[1]};
          const cf32 st = {ph[2], ph[3]};
          for (uint64_t k = 0; k < ov; ++k) {
            const uint64_t i1 = cfg->a1s + k, i2 = cfg->a2s + k;
            cf32 v = cmul(cmul(cmul(s1[i1], cconj(s2[i2])), fr_mix), pc);
            p12[2 * i2] += (double)v.re;
            p12[2 * i2 + 1] += (double)v.im;
            pc = cmul(pc, st);
          }
        }
      }
    }
    free(f1);
    free(f2);
    free(s1);
    free(s2);
  }
  for (int t = 0; t < nt; ++t) {
    const double* p = part + (size_t)t * 4 * h;
    for (uint64_t k = 0; k < h; ++k) {
      acc11[k] += p[k];
      acc22[k] += p[h + k];
      acc12[2 * k] += p[2 * h + 2 * k];
      acc12[2 * k + 1] += p[2 * h + 2 * k + 1];
    }
  }
  free(part);
  return failed;
}

/* ----------------------------------------------------- sector: phased path */

static void rotate_regular_bins(cf32* s, uint64_t len, uint32_t fft, double df, double tau) {
  /* utils.rs:69-124 with rate = accel = time = 0 and is_lsb = false */
  const double total = tau + 0.0 * 0.0 + 0.5 * 0.0 * (0.0 * 0.0);
  const double sign = -1.0;
  const double phase_step = sign * 2.0 * ORC_PI * df * total;
  cf32 rot = cpolar((float)(phase_step * 0.0));
  const cf32 step = cpolar((float)phase_step);
  for (uint64_t b = 0; b < len; ++b) {
    s[b] = cmul(s[b], rot);
    rot = cmul(rot, step);
  }
  if (fft % 2 == 0 && fft / 2 < len) s[fft / 2].im = 0.0f;
}

int64_t orc_sector_phased(const orc_scan_cfg* cfg, const uint8_t* raw1, const uint8_t* raw2,
                          uint64_t nf, uint64_t first_frame, double* acc_ph, uint8_t* raw_out,
                          int32_t nthreads) {
  /* main.rs:2222-2412 (process_frame + par_chunks_mut fold/reduce) */
  const uint32_t n = cfg->fft_len;
  const uint64_t h = n / 2 + 1;
  const uint64_t bpf1 = bytes_per_frame(n, cfg->bits1), bpf2 = bytes_per_frame(n, cfg->bits2);
  const uint64_t bpfo = bytes_per_frame(n, cfg->bits_out);
  const double df = cfg->fs_hz / (double)n;
  const uint64_t ov = cfg->a1e - cfg->a1s;
  const int output_lsb = cfg->lsb1 && cfg->lsb2;
  const float w1 = (float)cfg->w1, w2 = (float)cfg->w2;
  memset(acc_ph, 0, h * sizeof(double));
  if (!plan_get(n / 2)) return -1;
  int nt = 1;
#ifdef _OPENMP
  nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
  double* part = (double*)calloc((size_t)nt * h, sizeof(double));
  int64_t failed = 0;
#pragma omp parallel num_threads(nt) reduction(+ : failed)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* pp = part + (size_t)tid * h;
    float* f1 = (float*)malloc(sizeof(float) * n);
    float* f2 = (float*)malloc(sizeof(float) * n);
    float* ot = (float*)malloc(sizeof(float) * n);
    cf32* s1 = (cf32*)malloc(sizeof(cf32) * h);
    cf32* s2 = (cf32*)malloc(sizeof(cf32) * h);
    cf32* al = (cf32*)malloc(sizeof(cf32) * h);
    cf32* cb = (cf32*)malloc(sizeof(cf32) * h);
#pragma omp for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)nf; ++ii) {
      const uint64_t i = (uint64_t)ii;
      uint8_t* of = raw_out ? raw_out + i * bpfo : NULL;
      orc_frame_delay d;
      orc_delay_entry(&cfg->delay, first_frame + i, &d);
      if (orc_decode(raw1 + i * bpf1, bpf1, n, cfg->bits1, cfg->shuffle1, cfg->levels1,
                     cfg->nlevels1, cfg->lsb1, f1) < 0 ||
          orc_decode(raw2 + i * bpf2, bpf2, n, cfg->bits2, cfg->shuffle2, cfg->levels2,
                     cfg->nlevels2, cfg->lsb2, f2) < 0) {
        if (of) memset(of, 0, bpfo);
        failed++;
        continue;
      }
      orc_shift_zerofill(f1, n, d.int1);
      orc_shift_zerofill(f2, n, d.int2);
      orc_rfft_f32(n, f1, (float*)s1);
      orc_rfft_f32(n, f2, (float*)s2);
      rotate_regular_bins(s1, h, n, df, d.frac1);
      rotate_regular_bins(s2, h, n, df, d.frac2);
      const cf32 lo1 = {d.fr_lo1[0], d.fr_lo1[1]}, lo2 = {d.fr_lo2[0], d.fr_lo2[1]};
      memset(al, 0, sizeof(cf32) * h);
      if (cfg->grid == 0) {
        for (uint64_t k = 0; k < ov; ++k) al[cfg->a1s + k] = cmul(s2[cfg->a2s + k], lo2);
        for (uint64_t k = 0; k < h; ++k) {
          cf32 a = cmul(s1[k], lo1);
          cb[k].re = a.re * w1 + al[k].re * w2;
          cb[k].im = a.im * w1 + al[k].im * w2;
        }
      } else {
        for (uint64_t k = 0; k < ov; ++k) al[cfg->a2s + k] = cmul(s1[cfg->a1s + k], lo1);
        for (uint64_t k = 0; k < h; ++k) {
          cf32 b = cmul(s2[k], lo2);
          cb[k].re = al[k].re * w1 + b.re * w2;
          cb[k].im = al[k].im * w1 + b.im * w2;
        }
      }
      for (uint64_t k = 0; k < h; ++k) pp[k] += (double)cnorm2(cb[k]);
      if (of) {
        cb[0].im = 0.0f;
        if (n % 2 == 0) cb[n / 2].im = 0.0f;
        orc_irfft_f32(n, (const float*)cb, ot);
        if (output_lsb)
          for (uint64_t q = 1; q < n; q += 2) ot[q] = -ot[q];
        if (orc_quantise_frame(ot, n, cfg->bits_out, cfg->levels1, cfg->nlevels1, cfg->shuffle1,
                               of, bpfo) < 0) {
          memset(of, 0, bpfo);
          failed++;
        }
      }
    }
    free(f1);
    free(f2);
    free(ot);
    free(s1);
    free(s2);
    free(al);
    free(cb);
  }
  for (int t = 0; t < nt; ++t)
    for (uint64_t k = 0; k < h; ++k) acc_ph[k] += part[(size_t)t * h + k];
  free(part);
  return failed;
}

/* ------------------------------------------------------------- normalise */

double orc_level_power(const double* levels, uint32_t n) {
  /* main.rs:378-387 */
  double s = 0.0;
  for (uint32_t i = 0; i < n; ++i) s += levels[i] * levels[i];
  return s / (double)n;
}

void orc_normalize(uint32_t fft, uint64_t nf, double level_power, const double* acc_real,
                   const double* acc_cplx, float* out) {
  /* main.rs:2645-2683: inv = 1 / (0.5 * P * nf * N^2); first N/2 bins */
  const double norm_base = (double)nf * ((double)fft * (double)fft);
  const double inv = 1.0 / (0.5 * level_power * norm_base);
  for (uint32_t k = 0; k < fft / 2; ++k) {
    if (acc_cplx) {
      out[2 * k] = (float)(acc_cplx[2 * k] * inv);
      out[2 * k + 1] = (float)(acc_cplx[2 * k + 1] * inv);
    } else {
      out[2 * k] = (float)(acc_real[k] * inv);
      out[2 * k + 1] = 0.0f;
    }
  }
}
