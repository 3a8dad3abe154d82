// fxc_kernels.h — host-visible launch interface of the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fxc_device.cuh"

namespace fxc {

enum { MODE_CORR = 0, MODE_SPECTRA = 1, MODE_DECODE = 2 };

struct CorrParams {
  StationParams st[2];
  DelayParams dl;
  uint64_t nf, first_frame;
  int32_t a1s, a1e, a2s, grid;
  uint32_t products;
  uint32_t stage_bytes;  // FPC * (bpf1 + bpf2)
  uint32_t flush_every;  // iterations between f32 -> f64 flushes
  double df_hz;
  const FrameInfo* finfo; // per-frame records of the sector (frame_info_kernel)
  double* partials;      // MODE_CORR: [grid][4][H] f64
  float* out_a;          // MODE_SPECTRA: S1 [nf][H] complex; MODE_DECODE: x1 [nf][N]
  float* out_b;          // S2 / x2
  uint32_t* err;         // device error word (ERR_*)
  uint32_t wait_polls;   // polls before a staging wait gives up (0: kWaitPolls)
  uint32_t debug_flags;  // DBG_* (failure-injection test hook; 0 in normal use)
};

// Failure injection for the tests of the bounded waits: the staging copies
// of the fold kernels are announced on their mbarriers but never issued, so
// every wait runs out after wait_polls polls with nothing in flight.
enum : uint32_t { DBG_WITHHOLD_COPIES = 1u };

// Layout-compatible with fxc_frame_delay in include/fxc.h.
struct fxc_frame_delay_dev {
  int64_t int1, int2;
  double frac1, frac2;
  float fr_lo1[2], fr_lo2[2];
};

// Phased-array kernel parameters (weighted sum, power, C2R, re-quantise).
struct PhasedParams {
  StationParams st[2];
  DelayParams dl;
  uint64_t nf, first_frame;
  int32_t a1s, a1e, a2s, grid;
  uint32_t stage_bytes;
  uint32_t flush_every;
  uint32_t bits_out, bpf_out;
  int32_t out_lsb;       // negate odd output samples (both stations LSB)
  int32_t want_raw;
  float w1, w2;
  const float* qlevels;  // levels1 as f32 (device)
  uint32_t nqlevels;
  int32_t qmonotonic;    // +1 / -1 strictly ascending / descending levels, else 0
  const uint32_t* enc_lut;  // [4][256] byte LUTs of ant1's output shuffle (device)
  const FrameInfo* finfo;
  double* partials;      // [grid][H] f64
  uint8_t* raw_out;      // nf * bpf_out
  uint32_t* err;
};

int corr_frames_per_cta_iter(uint32_t n);
int corr_ctas_per_sm(uint32_t n);
cudaError_t launch_corr(uint32_t n, int mode, const CorrParams& p, int grid, cudaStream_t s);
// FFT-8192 correlation (MODE_CORR), one frame pair per CTA iteration (corr_fold.cu)
cudaError_t launch_corr_fold(const CorrParams& p, int grid, cudaStream_t s);
// FFT-8192 decode + integer shift through the correlation kernel's own decode
// path (fold_inputs), written out as f32 samples (MODE_DECODE semantics)
cudaError_t launch_fold_decode(const CorrParams& p, int grid, cudaStream_t s);
// FFT-16384 correlation as two 8192-point rows (corr_fold.cu); needs an even
// band shift (a row holds the bins of one parity)
bool corr_fold2_supported(const CorrParams& p);
cudaError_t launch_corr_fold2(const CorrParams& p, int grid, cudaStream_t s);
uint32_t fold_smem_bytes(uint32_t stage_bytes);
// FFT 16384 / 32768 / 65536 correlation (MODE_CORR) by clusters of C = N / 8192
// CTAs exchanging through distributed shared memory (corr_cluster.cu): every
// band shift and bit depth; partials [clusters][4][H].
int corr_cluster_size(uint32_t n);      // C, 0 when N has no cluster kernel
int corr_cluster_capacity(uint32_t n);  // clusters resident at once (0: none)
int corr_cluster_count(uint32_t n, uint64_t nf);  // clusters of a sector's launch
cudaError_t launch_corr_cluster(uint32_t n, const CorrParams& p, int clusters, cudaStream_t s);
// FFT 32768 / 65536 with 1- and 2-bit stations and a band shift that is a
// multiple of C: clusters of C/2 CTAs, each owning a mirror pair of rows
// (corr_pair.cu); FFT 16384 (C = 2) with 1- and 2-bit stations and an odd
// band shift: both rows in one CTA.  Partials [clusters][4][H].
bool corr_pair_supported(uint32_t n, const CorrParams& p);
int corr_pair_capacity(uint32_t n);
int corr_pair_count(uint32_t n, uint64_t nf);
cudaError_t launch_corr_pair(uint32_t n, const CorrParams& p, int clusters, cudaStream_t s);
cudaError_t launch_reduce(const double* part, int nblk, int h, double m11, double m22, double m12,
                          double* out, cudaStream_t s);
// FFT lengths above 8192 (N = c * 8192): global-memory four-step path.
struct LargeParams {
  StationParams st[2];
  const FrameInfo* finfo;  // records of every frame of the sector
  const float2* tw;        // W_N^j, j < N (launch_twiddle_table)
  int32_t n, c;
  int32_t a1s, a1e, a2s, grid;
  uint32_t products;
  uint32_t* err;           // device error word (ERR_*)
};
constexpr int kLargeGroups = 16;  // frame groups (partials) per sector
int large_batch_frames(uint32_t n);
cudaError_t launch_twiddle_table(int n, float2* tw, cudaStream_t s);
cudaError_t launch_large_fft(const LargeParams& p, uint64_t f0, uint64_t nb, float2* buf0,
                             float2* buf1, int sms, cudaStream_t s);
cudaError_t launch_large_acc(const LargeParams& p, const float2* Y, uint64_t f0, uint64_t nb,
                             int groups, int first_batch, double* part, cudaStream_t s);
// Phased synthesis for the batch whose spectra are in buf1 (f64 |cb|^2 into
// part[group][H]); with pp.want_raw also the inverse FFT (via buf0) and the
// packed .raw frames.
cudaError_t launch_large_phased(const LargeParams& p, const struct PhasedParams& pp, float2* buf0,
                                float2* buf1, uint64_t f0, uint64_t nb, int groups,
                                int first_batch, double* part, int sms, cudaStream_t s);
cudaError_t launch_large_decode(const LargeParams& p, uint64_t f0, uint64_t nb, float* x1,
                                float* x2, int sms, cudaStream_t s);
cudaError_t launch_large_split(const LargeParams& p, const float2* Y, uint64_t f0, uint64_t nb,
                               float2* s1, float2* s2, int sms, cudaStream_t s);

// ------------------------------------------------------------ batched sectors
//
// One launch per FFT length runs the sectors of many scans: a persistent grid
// takes work items (a frame range of one sector) by an atomic ticket, each CTA
// reloading the item's scan tables; every item writes its own f64 partials,
// summed per sector in item order by one reduction over the whole batch.

// Batch groups: the kernels a batch may launch, one per FFT length (16384 =
// the two-row kernel, even band shifts only), then the phased kernels of
// FFT 1024..8192.
enum {
  BG_1024 = 0, BG_2048 = 1, BG_4096 = 2, BG_8192 = 3, BG_16384 = 4,
  BG_PHASED_1024 = 5, BG_PHASED_2048 = 6, BG_PHASED_4096 = 7, BG_PHASED_8192 = 8,
  BG_PHASED_16384 = 9, kCorrGroups = 5, kBatchGroups = 10
};

// Frames [f0, f1) of the sector of scan `scan` (for the two-row kernel, the
// bins of parity `row`), accumulated into partials + part ([4][H] f64).
struct BatchItem {
  uint32_t scan, row;
  uint64_t f0, f1;
  uint64_t part;
};

struct BatchScan {
  CorrParams p;         // the sector: raw words, tables, frame records, error word
                        // (a phased sector: its delay model and frame records only)
  PhasedParams pp;      // a phased sector (phased != 0): the phased kernels' parameters
  double* acc;          // [5][H] output (acf11, acf22, xcf re/im, phased power)
  double m11, m22, m12; // reduction multipliers (two-for-one 2x, level scaling)
  uint64_t part;        // partials offset of the sector's first item
  uint64_t fi0;         // first frame of the sector in the batch's frame numbering
  uint64_t bin0;        // first bin of the sector in the batch's bin numbering
  uint32_t nparts;      // partial slots (items; two-row items share one per row pair)
  uint32_t n, h;        // FFT length, bins
  uint32_t phased;      // 1: items hold [H] phased power partials instead of [4][H]
};

// Device-resident description of one batch: the kernels read every count and
// table address from it, so that a captured graph serves every batch of the
// same group set.
struct BatchHeader {
  const BatchScan* scans;  // the batch's tables (after the header in the arena)
  const BatchItem* items;
  uint32_t nscans;
  uint32_t ticket[kBatchGroups];  // reset before each launch
  uint32_t nitems[kBatchGroups];
  uint32_t item0[kBatchGroups];
  uint32_t pad;
  uint64_t nframes;  // frames of all sectors
  uint64_t nbins;    // bins of all sectors
};

struct BatchArgs {
  BatchHeader* hdr;
  double* partials;
};

// Batch kernel variants: group g with `fpc` frame pairs per CTA iteration
// (FFT 1024: 1, 2, 4; 2048: 1, 2, 4; 4096: 1, 2; the fold kernels of FFT
// 8192 / 16384 take fpc = 1).  batch_prepare sets the variant's shared-memory
// limit (once, before any launch or capture); batch_group_ctas_per_sm is its
// occupancy (0: no such variant); launch_batch_group runs `grid` persistent CTAs.
cudaError_t batch_prepare(int g, int fpc);
int batch_group_ctas_per_sm(int g, int fpc);
cudaError_t launch_batch_group(int g, int fpc, const BatchArgs& a, int grid, cudaStream_t s);
// Frame records of every sector of the batch; the fixed-order reduction of
// every sector's partials into its acc (grid-stride, any grid size).
cudaError_t launch_batch_frame_info(const BatchArgs& a, int grid, cudaStream_t s);
// Phased batch groups (phased_kernels.cu): FFT n in 1024..8192, frames per CTA
// iteration as the single-scan phased kernel; n = 16384 the two-row kernel's.
cudaError_t phased_batch_prepare(uint32_t n);
int phased_batch_ctas_per_sm(uint32_t n);
int phased_frames_per_cta_iter(uint32_t n);
cudaError_t launch_phased_batch(uint32_t n, const BatchArgs& a, int grp, int grid, cudaStream_t s);
cudaError_t launch_batch_reduce(const BatchArgs& a, int grid, cudaStream_t s);

cudaError_t launch_phased(uint32_t n, const PhasedParams& p, int grid, cudaStream_t s);
// FFT 16384 phased products (1- to 8-bit stations): one CTA per frame pair,
// both rows in shared memory (phased_pair.cu); partials [grid][H].
bool phased_pair_supported(uint32_t n, const PhasedParams& p);
int phased_pair_grid(int sms, uint64_t nf);
cudaError_t launch_phased_pair(const PhasedParams& p, int grid, cudaStream_t s);
// Its persistent batch form (group BG_PHASED_16384, sectors that
// phased_pair_supported accepts, any mix of bit depths): shared-memory
// limit, occupancy, launch.
cudaError_t phased_pair_batch_prepare();
int phased_pair_batch_ctas_per_sm();
cudaError_t launch_phased_pair_batch(const BatchArgs& a, int grp, int grid, cudaStream_t s);
// FFT 32768 / 65536 phased products with 1- and 2-bit stations and a band
// shift that is a multiple of C: clusters of C/2 CTAs in the correlation pair
// kernel's row layout (phased_cpair.cu); partials [clusters][H]; the .raw
// words are ORed together by the cluster's CTAs (zero them first).
bool phased_cpair_supported(uint32_t n, const PhasedParams& p);
int phased_cpair_count(uint32_t n, uint64_t nf);
cudaError_t launch_phased_cpair(uint32_t n, const PhasedParams& p, int clusters, cudaStream_t s);
cudaError_t launch_reduce_phased(const double* part, int nblk, int h, double* out, cudaStream_t s);
cudaError_t launch_frame_info(const DelayParams& p, uint64_t first, uint64_t nf, int n,
                              double df_hz, int a1s, int a2s, FrameInfo* out, cudaStream_t s);
cudaError_t launch_delay_entries(const DelayParams& p, uint64_t first, uint64_t nf,
                                 fxc_frame_delay_dev* out, cudaStream_t s);

}  // namespace fxc
