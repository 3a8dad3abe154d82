/*
 * fxc.h — C ABI of the B200 FX-correlation engine (libfxc.so).
 *
 * The reference (fx-corr, a Rust CPU correlator) has no plugin or FFI API;
 * its hot path is the per-sector body of `run_once` (src/main.rs:2173-2683).
 * This header exposes that seam as plain C: a caller that today runs the
 * reference's sector loop hands one sector of packed .raw bytes per station
 * to the engine and receives the same f64 accumulators the reference's rayon
 * map/reduce produces (src/main.rs:2413-2591), computed on the GPU.
 *
 * Conventions
 *  - Every function returns fxc_status: 0 = FXC_OK, negative = error.  On
 *    error, fxc_last_error() returns a message for the calling thread.
 *  - No C++ types, exceptions or torch types cross this boundary: plain
 *    pointers and sizes only.  "d_" pointers are device (HBM) pointers,
 *    everything else is host memory.
 *  - Bins: H = fft_len/2 + 1 per product, index k = 0..H-1, exactly the
 *    reference's accumulator length (src/main.rs:2166-2167, 2425).
 *  - Device accumulator block (fxc_*_device): 5*H doubles laid out as
 *      [0,H)      acf11          (src/main.rs:2432)
 *      [H,2H)     acf22          (src/main.rs:2434)
 *      [2H,4H)    xcf, (re,im) interleaved (src/main.rs:2433)
 *      [4H,5H)    phased power   (src/main.rs:2427)
 *  - Thread safety: one fxc_scan per host thread; an fxc_engine may be shared
 *    by several threads, each with its own scans.
 */
#ifndef FXC_H
#define FXC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FXC_ABI_VERSION 1

#if defined(__GNUC__)
#define FXC_API __attribute__((visibility("default")))
#else
#define FXC_API
#endif

typedef int32_t fxc_status;
enum {
  FXC_OK = 0,
  FXC_EINVAL = -1,       /* invalid argument / configuration */
  FXC_ENOMEM = -2,       /* device or pinned host allocation failed */
  FXC_ECUDA = -3,        /* CUDA runtime error */
  FXC_ETIMEDOUT = -4,    /* fxc_sector_wait ran out of time, or a bounded
                            device-side wait gave up */
  FXC_ENOTFOUND = -5,    /* unknown sector id */
  FXC_EBUSY = -6,        /* admission refused: HBM budget or queue depth */
  FXC_EUNSUPPORTED = -7, /* configuration outside what the kernels handle */
  FXC_EDEVICE = -8,      /* a kernel reported an error status */
};

/* Products (which accumulators a scan computes). */
enum {
  FXC_PROD_ACF = 1,              /* write_acf_cor  (src/main.rs:1021) */
  FXC_PROD_XCF = 2,              /* write_xcf_cor  (src/main.rs:1022) */
  FXC_PROD_PHASED = 4,           /* phased power   (src/main.rs:2154) */
  FXC_PROD_RAW = 8,              /* phased .raw    (src/main.rs:1020) */
  FXC_PROD_ACF_OVERLAP_ONLY = 16 /* yi-acf: both ACFs over overlap bins
                                    only (src/main.rs:2157-2160) */
};

/* DelayEvalConfig (src/main.rs:161-182).  geom_table == NULL selects the
 * polynomial branch (src/main.rs:209-230); otherwise the 1-s geometric-delay
 * table (src/main.rs:1629-1644) is copied by fxc_scan_open. */
typedef struct fxc_delay_cfg {
  double frame_dt, fs, time_offset_s;
  const double* geom_table;
  uint64_t geom_len;
  double coarse_delay_s, delay_user_samples, extra_delay_rate_sps;
  double clock1_delay_s, clock1_rate_sps, clock2_delay_s, clock2_rate_sps;
  double d_seek;
  double net_d1_base, total_rate1_base, total_accel1_base;
  double net_d2_base, total_rate2_base, total_accel2_base;
  double lo1_hz, lo2_hz;
} fxc_delay_cfg;

/* FrameDelayEntry (src/main.rs:151-159). */
typedef struct fxc_frame_delay {
  int64_t int1, int2;
  double frac1, frac2;
  float fr_lo1[2], fr_lo2[2];
} fxc_frame_delay;

/* Per-scan configuration: the values run_once resolves before its sector
 * loop (src/main.rs:1063-1212, 1618-1673, 2073-2074). */
typedef struct fxc_scan_cfg {
  uint32_t fft_len;  /* N: power of two, 1024..65536 */
  uint32_t bits1, bits2, bits_out; /* 1,2,4,8; bits_out = max(bits1,bits2) (main.rs:1067) */
  double fs_hz;
  double levels1[256], levels2[256]; /* parse_levels (args.rs:194-200) */
  uint32_t nlevels1, nlevels2;       /* must equal 1 << bits */
  uint8_t shuffle1[32], shuffle2[32]; /* internal maps from parse_shuffle
                                         (args.rs:202-210): decoded bit o =
                                         raw word bit shuffle[o] */
  int32_t lsb1, lsb2;                /* LSB input: odd samples negated */
  int32_t shift_bins;                /* BandAlignment (main.rs:360-372) */
  uint32_t a1s, a1e, a2s;
  int32_t grid;                      /* 0 = ant1 grid, 1 = ant2 (main.rs:1212) */
  uint32_t products;                 /* FXC_PROD_* */
  double w1, w2;                     /* phased weights (args.rs:212-226) */
  fxc_delay_cfg delay;
} fxc_scan_cfg;

typedef struct fxc_device_opts {
  int32_t device;             /* CUDA ordinal */
  int32_t max_inflight;       /* sectors in flight per scan (0 = 2) */
  uint64_t hbm_budget_bytes;  /* admission budget for scans (0 = 80% of free) */
} fxc_device_opts;

/* Host-side results of one sector.  Any pointer may be NULL to skip it. */
typedef struct fxc_sector_out {
  double* acf11;   /* H doubles */
  double* acf22;   /* H doubles */
  double* xcf;     /* 2*H doubles, (re,im) interleaved */
  double* phased;  /* H doubles */
  uint8_t* raw_out;       /* nf * bytes_per_frame(bits_out) bytes */
  uint64_t raw_out_len;
  uint64_t frames_failed; /* frames skipped (src/main.rs:2592-2599) */
} fxc_sector_out;

typedef struct fxc_engine fxc_engine;
typedef struct fxc_scan fxc_scan;

/* ---- library ---------------------------------------------------------- */
FXC_API int32_t fxc_abi_version(void);
FXC_API const char* fxc_status_string(fxc_status s);
/* Message of the last error on the calling thread ("" if none). */
FXC_API const char* fxc_last_error(void);

/* ---- engine (owns device memory, streams, graphs) ---------------------- */
FXC_API fxc_status fxc_engine_create(const fxc_device_opts* opts, fxc_engine** out);
FXC_API fxc_status fxc_engine_destroy(fxc_engine* e);

/* ---- scan (replaces run_once's per-scan set-up, src/main.rs:1013-2172) -- */
FXC_API fxc_status fxc_scan_open(fxc_engine* e, const fxc_scan_cfg* cfg, fxc_scan** out);
FXC_API fxc_status fxc_scan_close(fxc_scan* s);

/* Asynchronous per-sector call on host buffers (replaces the body of the
 * sector loop, src/main.rs:2173-2591).  raw1/raw2 hold nf frames of
 * bytes_per_frame(bits) bytes each, exactly the reader thread's message
 * (src/main.rs:2135-2147).  first_frame is the scan-global index of frame 0
 * (the reference's `emitted`).  The buffers must stay unchanged until
 * fxc_sector_wait returns for the returned id. */
FXC_API fxc_status fxc_sector_submit(fxc_scan* s, const uint8_t* raw1, uint64_t n1, const uint8_t* raw2,
                             uint64_t n2, uint64_t nf, uint64_t first_frame, uint64_t* sector_id);
/* Wait (timeout_ms < 0: no limit) and copy results out. */
FXC_API fxc_status fxc_sector_wait(fxc_scan* s, uint64_t sector_id, int32_t timeout_ms,
                           fxc_sector_out* out);

/* ---- device-resident entry points (inputs already in HBM) -------------- */
/* One sector with inputs resident in device memory; enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default).  d_acc receives the 5*H-double
 * accumulator block.  d_raw_out (nf*bytes_per_frame(bits_out) bytes) is
 * written when the scan has FXC_PROD_RAW.  Device inputs must be 16-byte
 * aligned.  Asynchronous: call fxc_scan_check(s) after synchronising. */
FXC_API fxc_status fxc_sector_run_device(fxc_scan* s, const uint8_t* d_raw1, const uint8_t* d_raw2,
                                 uint64_t nf, uint64_t first_frame, double* d_acc,
                                 uint8_t* d_raw_out, void* stream);
/* Reads and clears the scan's device error word (bounded waits, bad sizes);
 * FXC_OK when no kernel reported an error.  Synchronises the scan's work. */
FXC_API fxc_status fxc_scan_check(fxc_scan* s);

/* Failure-injection test hook, no reference counterpart (the reference has
 * no device-side waits).  Process-wide, for the correlation launches that
 * follow: wait_polls > 0 bounds every staging wait of the FFT-8192 / 16384
 * correlation kernels to that many mbarrier polls (0 restores the built-in
 * limit); withhold_copies != 0 makes those kernels announce their staging
 * copies without issuing them, so that each CTA's first wait runs out with
 * no copy in flight, the kernel sets its error word and stops, and
 * fxc_scan_check / fxc_sector_wait / fxc_sector_noalloc_check report
 * FXC_ETIMEDOUT while the CUDA context stays usable.  Not for production
 * use; (0, 0) is the normal setting. */
FXC_API fxc_status fxc_debug_inject_wait_timeout(uint32_t wait_polls, int32_t withhold_copies);

/* Kernel timing: when enabled, every correlation-kernel launch of this scan
 * is bracketed by CUDA events on its launch stream.  fxc_scan_profile sums
 * their elapsed device time (synchronising on the last event) and reports the
 * number of those launches and of all library kernel launches since the last
 * reset. */
FXC_API fxc_status fxc_scan_set_profiling(fxc_scan* s, int32_t enable);
FXC_API fxc_status fxc_scan_profile(fxc_scan* s, double* kernel_ms, uint64_t* kernel_launches,
                                    uint64_t* all_launches, int32_t reset);

/* ---- allocation-free correlation call ----------------------------------
 * No counterpart in the reference (its CPU path allocates per sector); this
 * entry point exists for callers that cannot allocate device memory where
 * they correlate: a real-time streaming loop that must not pay the implicit
 * device synchronisation of cudaMalloc/cudaFree, or a host application whose
 * memory manager owns all device memory.
 *
 * Same result as opening a scan with `cfg` and calling fxc_sector_run_device
 * (ACF/XCF products), without an engine or scan and without allocating: the
 * kernels' scratch is a fixed FXC_NOALLOC_SCRATCH_MIB MiB array that every
 * GPU loading the library holds until the process exits.  Limits: fft_len
 * <= 8192, nf <= FXC_NOALLOC_MAX_FRAMES per call (add the results of several
 * calls for a longer sector), geometric table <= FXC_NOALLOC_MAX_GEOM entries;
 * larger requests fail with FXC_EINVAL / FXC_EUNSUPPORTED.  Runs on the
 * current device, enqueued on `stream`, which must belong to that device
 * (FXC_EINVAL otherwise).  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) and caches it.  All
 * calls share the array: calls whose work overlaps on one GPU (other streams
 * or host threads) race and must be serialised by the caller.
 *
 * Errors inside the kernels: when a bounded device-side wait gives up, the
 * call fills d_acc with NaN; fxc_sector_noalloc_check(stream) then
 * synchronises `stream` and returns FXC_ETIMEDOUT (FXC_EDEVICE for another
 * kernel error, FXC_OK when the last call on this device completed cleanly),
 * again without allocating.  Check before the next call on the device, which
 * clears the error word. */
#define FXC_NOALLOC_MAX_FRAMES 32768
#define FXC_NOALLOC_MAX_GEOM 4096
#define FXC_NOALLOC_SCRATCH_MIB 24
FXC_API fxc_status fxc_sector_run_device_noalloc(const fxc_scan_cfg* cfg, const uint8_t* d_raw1,
                                                 const uint8_t* d_raw2, uint64_t nf,
                                                 uint64_t first_frame, double* d_acc,
                                                 void* stream);
FXC_API fxc_status fxc_sector_noalloc_check(void* stream);

/* ---- serving loop -------------------------------------------------------
 * No reference counterpart: the reference correlates one scan per process
 * (the run_once sector loop, src/main.rs:2173-2591).  A server admits jobs
 * (one scan's frames from host memory, dumped every sector_frames frames)
 * into `slots` concurrent device contexts; a job that arrives while others
 * run starts as soon as a slot is free and the engine's HBM budget admits
 * its buffers, and the jobs' copies and kernels overlap on the device.  The
 * device state of a finished job (partials, frame records, staging buffers,
 * tables) is reused by the next job of its slot.  Each job's products are
 * those of fxc_sector_submit/wait over the same sectors, bit for bit, alone
 * or in any mix; with opts.batch they are those of fxc_batch_run_device over
 * the same sectors (within the FP32 tolerance of the per-scan path), again
 * identical alone and in any mix. */
typedef struct fxc_server fxc_server;

typedef struct fxc_server_opts {
  int32_t slots;             /* jobs on the device at once (0 = 4, at most 256) */
  int32_t batch;             /* 1: the sectors of all running jobs are computed
                                together, one fxc_batch call (CUDA graphs,
                                autotuned shapes) per round of ready sectors;
                                2: the same with the default kernel shapes, so
                                that the products do not depend on timing */
} fxc_server_opts;

typedef struct fxc_job {
  const fxc_scan_cfg* cfg;   /* copied at submit, geometric table included */
  const uint8_t* raw1;       /* nf * bytes_per_frame(bits1) bytes; page-locked memory
                                lets the copies overlap other jobs' work */
  const uint8_t* raw2;       /* nf * bytes_per_frame(bits2) bytes */
  uint64_t nf;               /* frames in the job */
  uint64_t first_frame;      /* scan frame index of raw1[0] (delay-model time) */
  uint64_t sector_frames;    /* frames per dump; 0 = one dump for the whole job */
  double* out;               /* per dump: acf11[H] | acf22[H] | xcf[2H] | phased[H] */
  uint8_t* raw_out;          /* FXC_PROD_RAW: nf * bytes_per_frame(bits_out) bytes */
} fxc_job;

typedef struct fxc_job_stats {
  int32_t status;            /* the job's fxc_status */
  uint32_t sectors;          /* dumps written */
  uint64_t t_submit_ns;      /* steady clock: submitted, started on a slot, done */
  uint64_t t_start_ns;
  uint64_t t_done_ns;
} fxc_job_stats;

FXC_API fxc_status fxc_server_create(fxc_engine* e, const fxc_server_opts* opts, fxc_server** out);
/* Queues a job; the caller's buffers stay untouched until fxc_server_wait
 * returns for the id. */
FXC_API fxc_status fxc_server_submit(fxc_server* sv, const fxc_job* job, uint64_t* job_id);
/* Waits for a job (timeout_ms < 0: no limit) and forgets it. */
FXC_API fxc_status fxc_server_wait(fxc_server* sv, uint64_t job_id, int32_t timeout_ms,
                                   fxc_job_stats* stats);
/* Finishes the running jobs, fails the queued ones that have not started
 * (FXC_EBUSY), then releases the slots. */
FXC_API fxc_status fxc_server_destroy(fxc_server* sv);

/* ---- batched sectors of many scans --------------------------------------
 * No reference counterpart (the reference runs one scan per process).  A
 * batch runs one sector of each of many distinct scans in a few launches:
 * the frame records of every sector in one launch, every sector of one FFT
 * length in one persistent kernel (1-8 bit stations mixed; work items of a
 * few hundred frames handed out to the CTAs by an atomic ticket), and one
 * fixed-order reduction for all.  With use_graphs the launches of each set of
 * FFT lengths are captured once in a CUDA graph and replayed.  The frames per
 * CTA iteration and frames per work item of each FFT length come from an
 * autotuner that times the kernel variants on a synthetic batch (at first use
 * of the length when opts.autotune is set, or by fxc_batch_autotune).
 * Phased sectors (yi-phasedarray: phased power and .raw frames, FFT
 * 1024..16384) run in persistent phased kernels of the same batch.  Sectors
 * the batch kernels do not cover (phased products or correlation above FFT
 * 16384, correlation at FFT 16384 with an odd band shift, scans with both
 * correlation and phased products, empty sectors) run through the per-scan
 * path on the same stream.  A sector's products equal fxc_sector_run_device's within the
 * library's FP32 tolerance (phased .raw frames byte for byte), and are
 * identical bit for bit whatever else shares the batch (the item split
 * depends only on the sector's frame count and the batch's tuning). */
typedef struct fxc_batch fxc_batch;

typedef struct fxc_batch_opts {
  int32_t use_graphs;        /* capture and replay CUDA graphs */
  int32_t autotune;          /* tune an FFT length at its first batch */
  uint32_t item_frames;      /* frames per work item; 0 = tuned or the default */
} fxc_batch_opts;

FXC_API fxc_status fxc_batch_create(fxc_engine* e, const fxc_batch_opts* opts, fxc_batch** out);
FXC_API fxc_status fxc_batch_destroy(fxc_batch* b);
/* One sector of each of `count` distinct scans of b's engine: device inputs
 * (16-byte aligned), device outputs d_acc[i] of 5 * H doubles as in
 * fxc_sector_run_device, enqueued on `stream`.  Host arrays are read before
 * the call returns.  Calls on one batch are serialised (a later call may use
 * another stream; it waits for the earlier call's device work). */
FXC_API fxc_status fxc_batch_run_device(fxc_batch* b, fxc_scan* const* scans,
                                        const uint8_t* const* d_raw1,
                                        const uint8_t* const* d_raw2, const uint64_t* nf,
                                        const uint64_t* first_frame, double* const* d_acc,
                                        uint32_t count, void* stream);
/* The same with phased .raw output: d_raw_out[i] (nf[i] * bytes_per_frame(
 * bits_out) device bytes) receives scan i's re-quantised phased frames when
 * the scan has FXC_PROD_RAW (NULL entries for the other scans). */
FXC_API fxc_status fxc_batch_run_device_raw(fxc_batch* b, fxc_scan* const* scans,
                                            const uint8_t* const* d_raw1,
                                            const uint8_t* const* d_raw2, const uint64_t* nf,
                                            const uint64_t* first_frame, double* const* d_acc,
                                            uint8_t* const* d_raw_out, uint32_t count,
                                            void* stream);
/* Times every kernel variant x work-item size of one FFT length (1024..16384)
 * on a synthetic 2-bit batch and keeps the fastest (blocks the host for tens
 * of milliseconds). */
FXC_API fxc_status fxc_batch_autotune(fxc_batch* b, uint32_t fft_len);
/* The shape in use for an FFT length: frame pairs per CTA iteration, frames
 * per work item, resident CTAs per SM, and the tuner's measured
 * Gsample/s (0 if not tuned). */
FXC_API fxc_status fxc_batch_shape(fxc_batch* b, uint32_t fft_len, int32_t* fpc,
                                   uint32_t* item_frames, int32_t* ctas_per_sm, double* gsps);
/* Pins the shape of an FFT length: fpc a variant the length has (1024 and
 * 2048: 1, 2, 4; 4096: 1, 2; 8192 and 16384: 1), item_frames a positive
 * multiple of 32. */
FXC_API fxc_status fxc_batch_set_shape(fxc_batch* b, uint32_t fft_len, int32_t fpc,
                                       uint32_t item_frames);
/* Kernels the batch launched so far (graph replays count their kernels). */
FXC_API uint64_t fxc_batch_launches(fxc_batch* b);

/* Page-locked host memory for sector buffers (no reference counterpart: the
 * reference reads into pageable Vec<u8>, src/main.rs:2133-2147); copies from
 * it overlap device work. */
FXC_API fxc_status fxc_host_alloc(uint64_t bytes, void** out);
FXC_API fxc_status fxc_host_free(void* p);
/* Page-locks a caller-owned host buffer in place, so that a reader that owns
 * its sector buffers (the reference's Vec<u8> per station, filled by the
 * reader thread, src/main.rs:2133-2147) passes them to fxc_sector_submit
 * without a staging copy and the host-to-device copies overlap device work.
 * The buffer must stay allocated until fxc_host_unregister; registering
 * costs a page-table walk, so register long-lived buffers once.  A buffer
 * that is already registered (or page-locked by fxc_host_alloc) is
 * accepted as is. */
FXC_API fxc_status fxc_host_register(void* p, uint64_t bytes);
FXC_API fxc_status fxc_host_unregister(void* p);

/* Stage entry points, for parity tests of the individual steps. */
/* Per-frame delay model on the device (src/main.rs:184-241). */
FXC_API fxc_status fxc_delay_entries_device(fxc_scan* s, uint64_t first_frame, uint64_t nf,
                                    fxc_frame_delay* d_out, void* stream);
/* Decode + LSB flip + integer shift of both stations (src/utils.rs:215-376,
 * 126-145): d_x1, d_x2 = nf*fft_len f32 each, shifted by the delay model's
 * int1 / int2 for each frame. */
FXC_API fxc_status fxc_decode_device(fxc_scan* s, const uint8_t* d_raw1, const uint8_t* d_raw2,
                             uint64_t nf, uint64_t first_frame, float* d_x1, float* d_x2,
                             void* stream);
/* R2C spectra of both stations after decode+shift (src/utils.rs:47-59):
 * d_s1, d_s2 = nf*H complex f32 ((re,im) interleaved). */
FXC_API fxc_status fxc_spectra_device(fxc_scan* s, const uint8_t* d_raw1, const uint8_t* d_raw2,
                              uint64_t nf, uint64_t first_frame, float* d_s1, float* d_s2,
                              void* stream);

/* ---- host helpers (no GPU needed) --------------------------------------- */
/* parse_shuffle (args.rs:202-210): external MSB-first list -> internal map. */
FXC_API fxc_status fxc_parse_shuffle(const int32_t ext[32], uint8_t internal[32]);
/* compute_band_alignment (main.rs:363-372): out = {shift_bins, a1s, a1e, a2s}. */
FXC_API fxc_status fxc_band_alignment(uint32_t fft, double fs_hz, double c1_mhz, double c2_mhz,
                              double bw1_mhz, double bw2_mhz, int64_t out[4]);
/* quantization_mean_power (main.rs:378-387). */
FXC_API fxc_status fxc_level_power(const double* levels, uint32_t n, double* out);
/* Sector normalisation + .cor dump values (main.rs:2645-2683): first fft/2
 * bins as f32 (re,im) pairs; acc_cplx (2*H doubles) for XCF, else acc_real. */
FXC_API fxc_status fxc_normalize(uint32_t fft, uint64_t nf, double level_power, const double* acc_real,
                         const double* acc_cplx, float* out);
/* bytes per frame, (fft*bits + 7)/8 (main.rs:1214-1215). */
FXC_API uint64_t fxc_bytes_per_frame(uint32_t fft, uint32_t bits);
/* Measured FP32 FMA throughput of the device (TFLOP/s), for rooflines. */
FXC_API fxc_status fxc_probe_fp32_peak(int32_t device, double* tflops);
/* Design-choice probes (no reference counterpart), measured on `device`:
 * smem_ns / shfl_ns = time for one SM to redistribute a frame's 8192 complex
 * values among 512 threads (16 per thread) through padded shared memory
 * (the exchange between two radix-16 passes) / by warp shuffles (a 16 x 16
 * transpose within each half-warp); tflops = throughput of mma.sync m16n8k16
 * (f16 inputs, f32 accumulation) over the whole GPU. */
FXC_API fxc_status fxc_probe_exchange(int32_t device, double* smem_ns, double* shfl_ns);
FXC_API fxc_status fxc_probe_mma_f16(int32_t device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif
