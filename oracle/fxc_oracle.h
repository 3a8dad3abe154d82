/*
 * fxc_oracle.h — CPU restatement of the fx-corr correlation path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libfxc, the CLI, the
 * kernels) includes, links or calls this code.  Only tests/, the smoke check
 * in __graft_entry__.py and the cpu_baseline / --impl reference legs of
 * bench.py load it, and only as the checker or as the timed CPU baseline.
 *
 * Parity status: UNPINNED by reference-produced vectors.  The reference
 * (Rust, fx-corr 1.0.0) cannot be compiled here (no Rust toolchain) and its
 * own tests cover only epoch/RA/Dec parsing (src/geom.rs:387-437).  Every
 * function below restates the cited reference lines; the FFT restates the
 * mathematical DFT that rustfft 6.4.0 / realfft 3.5.0 compute
 * (src/utils.rs:22-66 call sites).  tests/golden holds hand-derived
 * known-answer vectors that pin this restatement to the cited semantics.
 *
 * Floating-point: built with -ffp-contract=off so f32/f64 expressions round
 * exactly as the reference's (Rust never fuses a*b+c).
 */
#ifndef FXC_ORACLE_H
#define FXC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_PROD_ACF = 1,
  ORC_PROD_XCF = 2,
  ORC_PROD_PHASED = 4,
  ORC_PROD_RAW = 8,
  ORC_PROD_ACF_OVERLAP_ONLY = 16,
};

/* DelayEvalConfig (src/main.rs:161-182). geom_table == NULL selects the
 * polynomial branch (src/main.rs:209-230). */
typedef struct {
  double frame_dt, fs, time_offset_s;
  const double* geom_table;
  uint64_t geom_len;
  double coarse_delay_s, delay_user_samples, extra_delay_rate_sps;
  double clock1_delay_s, clock1_rate_sps, clock2_delay_s, clock2_rate_sps;
  double d_seek;
  double net_d1_base, total_rate1_base, total_accel1_base;
  double net_d2_base, total_rate2_base, total_accel2_base;
  double lo1_hz, lo2_hz;
} orc_delay_cfg;

/* FrameDelayEntry (src/main.rs:151-159). */
typedef struct {
  int64_t int1, int2;
  double frac1, frac2;
  float fr_lo1[2], fr_lo2[2];
} orc_frame_delay;

typedef struct {
  uint32_t fft_len;
  uint32_t bits1, bits2, bits_out;
  double fs_hz;
  double levels1[256], levels2[256];
  uint32_t nlevels1, nlevels2;
  uint8_t shuffle1[32], shuffle2[32]; /* internal maps: out bit o <- word bit shuffle[o] */
  int32_t lsb1, lsb2;
  int32_t shift_bins;
  uint32_t a1s, a1e, a2s;
  int32_t grid; /* 0 = ant1 grid, 1 = ant2 grid (src/main.rs:1212) */
  uint32_t products;
  double w1, w2;
  orc_delay_cfg delay;
} orc_scan_cfg;

/* args.rs:202-210: external MSB-first list -> internal map. 0 ok, -1 error. */
int orc_parse_shuffle(const int32_t ext[32], uint8_t internal[32]);

/* utils.rs:215-376 for one frame. Returns number of samples decoded, or -1 on
 * the reference's error conditions (output too short / count mismatch). */
int64_t orc_decode(const uint8_t* raw, uint64_t raw_len, uint64_t samples, uint32_t bits,
                   const uint8_t shuffle[32], const double* levels, uint32_t nlevels,
                   int32_t lsb_to_usb, float* out);

/* utils.rs:126-145 */
void orc_shift_zerofill(float* x, uint64_t n, int64_t s);

/* Forward real DFT, unnormalised, f32 (utils.rs:47-59): out has n/2+1
 * interleaved (re, im) pairs. n must be a power of two >= 2. */
int orc_rfft_f32(uint32_t n, const float* in, float* out);
/* Inverse C2R scaled by 1/n (utils.rs:60-66); imag of DC / Nyquist ignored. */
int orc_irfft_f32(uint32_t n, const float* in, float* out);

/* main.rs:184-241 */
void orc_delay_entry(const orc_delay_cfg* cfg, uint64_t frame_idx, orc_frame_delay* out);

/* main.rs:363-372. Returns 0 ok, -1 "No band overlap". out = {sb, a1s, a1e, a2s}. */
int orc_band_alignment(uint32_t fft, double fs, double c1, double c2, double bw1, double bw2,
                       int64_t out[4]);

/* main.rs:132-149: out = {start.re, start.im, step.re, step.im} */
void orc_xcf_phase_start_and_step(double df_hz, double frac1, double frac2, uint64_t a1s,
                                  uint64_t a2s, float out[4]);

/* utils.rs:378-410: returns bytes written to out (capacity out_cap). */
int64_t orc_quantise_frame(const float* samples, uint64_t n, uint32_t bits, const double* levels,
                           uint32_t nlevels, const uint8_t shuffle_out[32], uint8_t* out,
                           uint64_t out_cap);

/* One sector of the yi-acf/xcf/corr path (main.rs:2413-2591): accumulators of
 * length H = fft/2+1 are overwritten. acc12 is interleaved (re, im).
 * first_frame is the scan-global index of frame 0 (the reference's `emitted`).
 * nthreads <= 0 uses the OpenMP default. Returns number of failed frames. */
int64_t orc_sector_corr(const orc_scan_cfg* cfg, const uint8_t* raw1, const uint8_t* raw2,
                        uint64_t nf, uint64_t first_frame, double* acc11, double* acc22,
                        double* acc12, int32_t nthreads);

/* One sector of the yi-phasedarray path (main.rs:2222-2412): acc_ph (H doubles)
 * overwritten; raw_out (nf * bpf_out bytes) written when non-NULL. */
int64_t orc_sector_phased(const orc_scan_cfg* cfg, const uint8_t* raw1, const uint8_t* raw2,
                          uint64_t nf, uint64_t first_frame, double* acc_ph, uint8_t* raw_out,
                          int32_t nthreads);

/* main.rs:2645-2683: f64 accumulators -> first fft/2 bins as f32 (re, im). */
void orc_normalize(uint32_t fft, uint64_t nf, double level_power, const double* acc_real,
                   const double* acc_cplx, float* out);
/* main.rs:378-387 */
double orc_level_power(const double* levels, uint32_t n);

/* Test data (synth.c, not a restatement): nsamp samples per station of
 * quantised Gaussian noise (unit variance times `gain`, nearest of the
 * nlevels = 2^bits levels) sharing a common component at correlation rho,
 * station 2's copy `lag` samples late, plus tone_amp * cos(2 pi tone_cyc n +
 * tone_phase) at both stations when tone_amp != 0, odd samples of an LSB station negated,
 * packed LSB-first into little-endian words with word bit p moved to bit
 * shuffle_out[p].  nsamp must fill whole words.  Returns 0, or -1 on bad
 * arguments.  The output does not depend on nthreads. */
int orc_synth_pack_pair(uint64_t seed, uint64_t nsamp, double rho, uint32_t lag,
                        double tone_amp, double tone_cyc, double tone_phase, uint32_t bits,
                        const double* levels, uint32_t nlevels, double gain,
                        const uint8_t shuffle_out1[32], int32_t lsb1,
                        const uint8_t shuffle_out2[32], int32_t lsb2, uint8_t* out1,
                        uint8_t* out2, int32_t nthreads);

#ifdef __cplusplus
}
#endif
#endif
