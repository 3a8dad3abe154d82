// api.cu — the C ABI of libfxc (include/fxc.h): engine, scans, per-sector
// submission on host buffers, device-resident sector calls, stage entry
// points and host helpers.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "fxc.h"
#include "fxc_internal.h"
#include "fxc_kernels.h"

using namespace fxc;

namespace {

thread_local std::string g_err;

// failure injection (fxc_debug_inject_wait_timeout)
std::atomic<uint32_t> g_dbg_polls{0}, g_dbg_flags{0};

fxc_status fail(fxc_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return s;
}

#define CK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? FXC_ENOMEM : FXC_ECUDA, "%s: %s", \
                  #call, cudaGetErrorString(e_));                                      \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

struct fxc_engine {
  int device = 0;
  int sm_count = 0;
  int max_inflight = 2;
  uint64_t budget = 0;
  uint64_t in_use = 0;
  std::mutex mu;
  std::vector<fxc_scan*> scans;  // open scans, closed by fxc_engine_destroy
  std::vector<fxc_server*> servers;  // live servers, destroyed first by fxc_engine_destroy
  std::vector<fxc_batch*> batches;   // live batches, destroyed next
};

struct SectorSlot {
  uint8_t* d_raw1 = nullptr;
  uint8_t* d_raw2 = nullptr;
  uint64_t cap1 = 0, cap2 = 0;
  double* d_acc = nullptr;
  uint8_t* d_rawout = nullptr;
  uint64_t cap_out = 0;
  double* h_acc = nullptr;     // pinned: 5H doubles + error word
  uint8_t* h_rawout = nullptr; // pinned
  uint64_t hcap_out = 0;
  cudaEvent_t ev_h2d = nullptr, ev_done = nullptr;
  uint64_t id = 0;
  uint64_t nf = 0;
  bool busy = false;
};

struct fxc_scan {
  fxc_engine* eng = nullptr;
  fxc_scan_cfg cfg{};
  uint32_t n = 0, h = 0;
  uint32_t bpf1 = 0, bpf2 = 0, bpfo = 0;
  int shkind[2] = {0, 0};
  float scale[2] = {1.0f, 1.0f};  // exact powers of two (see level_scale)
  double* d_table = nullptr;
  uint64_t table_cap = 0;        // doubles
  bool table_bound = false;      // the bound configuration has a geometric table
  uint8_t* h_tab = nullptr;      // pinned staging of the uploaded tables
  uint64_t h_tab_cap = 0;
  uint32_t* d_lut = nullptr;     // [2][1024]
  float* d_levels = nullptr;     // [2][256]
  uint8_t* d_shuffle_out = nullptr;
  float* d_qlevels = nullptr;     // levels1 as f32 for the phased re-quantiser
  uint32_t* d_enc_lut = nullptr;  // [4][256] byte LUTs of ant1's output shuffle
  int qmonotonic = 0;
  double* d_partials = nullptr;
  uint64_t partials_elems = 0;
  uint64_t partials_cap = 0;     // elements allocated
  uint64_t big_cap = 0;          // float2 elements allocated per batch buffer
  uint32_t acc_cap = 0;          // H the sector slots' d_acc / h_acc hold
  FrameInfo* d_finfo = nullptr;  // per-frame delay records of the sector in flight
  uint64_t finfo_cap = 0;
  float2* d_big[2] = {nullptr, nullptr};  // FFT lengths > 8192: batch scratch
  float2* d_twl = nullptr;                // FFT lengths > 8192: W_N^j, j < N
  uint64_t twl_cap = 0;                   // entries allocated
  uint64_t big_frames = 0;                // frames per batch
  uint32_t* d_err = nullptr;
  cudaStream_t stream = nullptr;     // compute
  cudaStream_t copy_stream = nullptr;
  std::vector<SectorSlot> slots;
  uint64_t next_id = 1;
  uint64_t hbm_bytes = 0;
  // kernel timing (fxc_scan_set_profiling)
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
  size_t prof_used = 0;
  uint64_t kernel_launches = 0;
  uint64_t all_launches = 0;
};

namespace {

int shuffle_kind(const uint8_t sh[32]) {
  bool ident = true, pair = true;
  for (int i = 0; i < 32; ++i) {
    if (sh[i] != i) ident = false;
    if (sh[i] != (i ^ 1)) pair = false;
  }
  return ident ? SH_IDENTITY : (pair ? SH_PAIRSWAP : SH_GENERIC);
}

// Byte LUTs for a generic 32-bit shuffle: out bit o takes word bit sh[o].
void build_lut(const uint8_t sh[32], uint32_t* lut) {
  std::memset(lut, 0, 1024 * sizeof(uint32_t));
  for (int o = 0; o < 32; ++o) {
    const int in = sh[o];
    const int byte = in >> 3, bit = in & 7;
    for (int v = 0; v < 256; ++v)
      if ((v >> bit) & 1) lut[byte * 256 + v] |= (1u << o);
  }
}

// Power of two nearest 1/RMS of a level table.  Both stations share one
// complex FFT (z = x1 + i x2), so rounding error scales with the stronger
// station; equalising the RMS by an exact power of two keeps the weaker
// station's spectrum at full f32 relative precision and is undone exactly.
float level_scale(const double* lv, uint32_t n) {
  double p = 0.0;
  for (uint32_t i = 0; i < n; ++i) p += lv[i] * lv[i];
  p /= (double)n;
  if (!(p > 0.0) || !std::isfinite(p)) return 1.0f;
  const int e = (int)std::lround(0.5 * std::log2(p));
  return std::ldexp(1.0f, -e);
}

DelayParams delay_params(const fxc_scan* s) {
  const fxc_delay_cfg& c = s->cfg.delay;
  DelayParams p;
  p.frame_dt = c.frame_dt;
  p.fs = c.fs;
  p.time_offset_s = c.time_offset_s;
  p.table = s->table_bound ? s->d_table : nullptr;
  p.table_len = s->table_bound ? c.geom_len : 0;
  p.coarse = c.coarse_delay_s;
  p.user_samples = c.delay_user_samples;
  p.extra_rate = c.extra_delay_rate_sps;
  p.c1d = c.clock1_delay_s;
  p.c1r = c.clock1_rate_sps;
  p.c2d = c.clock2_delay_s;
  p.c2r = c.clock2_rate_sps;
  p.d_seek = c.d_seek;
  p.d1 = c.net_d1_base;
  p.r1 = c.total_rate1_base;
  p.a1 = c.total_accel1_base;
  p.d2 = c.net_d2_base;
  p.r2 = c.total_rate2_base;
  p.a2 = c.total_accel2_base;
  p.lo1 = c.lo1_hz;
  p.lo2 = c.lo2_hz;
  return p;
}

void station_params(const fxc_scan* s, const uint8_t* r1, const uint8_t* r2, StationParams st[2]) {
  st[0].raw = r1;
  st[1].raw = r2;
  for (int k = 0; k < 2; ++k) {
    st[k].shlut = s->d_lut + 1024 * k;
    st[k].levels = s->d_levels + 256 * k;
    st[k].bpf = k ? s->bpf2 : s->bpf1;
    st[k].bits = (int)(k ? s->cfg.bits2 : s->cfg.bits1);
    st[k].lsb = k ? s->cfg.lsb2 : s->cfg.lsb1;
    st[k].shkind = s->shkind[k];
    st[k].scale = s->scale[k];
    std::memcpy(st[k].perm, k ? s->cfg.shuffle2 : s->cfg.shuffle1, 32);
  }
}

int corr_grid(const fxc_scan* s, uint64_t nf) {
  const uint64_t fpc = (uint64_t)corr_frames_per_cta_iter(s->n);
  const uint64_t iters = (nf + fpc - 1) / fpc;
  const uint64_t maxg = (uint64_t)s->eng->sm_count * (uint64_t)corr_ctas_per_sm(s->n);
  return (int)std::max<uint64_t>(1, std::min(iters, maxg));
}

CorrParams corr_params(const fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                       uint64_t first) {
  CorrParams p{};
  station_params(s, r1, r2, p.st);
  p.dl = delay_params(s);
  p.nf = nf;
  p.first_frame = first;
  p.a1s = (int32_t)s->cfg.a1s;
  p.a1e = (int32_t)s->cfg.a1e;
  p.a2s = (int32_t)s->cfg.a2s;
  p.grid = s->cfg.grid;
  p.products = s->cfg.products;
  const int fpc = corr_frames_per_cta_iter(s->n);
  p.stage_bytes = (uint32_t)fpc * (s->bpf1 + s->bpf2);
  p.flush_every = (uint32_t)std::max(1, 32 / fpc);
  p.df_hz = s->cfg.fs_hz / (double)s->n;
  p.partials = s->d_partials;
  p.finfo = s->d_finfo;
  p.err = s->d_err;
  internal_debug_settings(&p.wait_polls, &p.debug_flags);
  return p;
}

// Room for nf frame records in the scan's record buffer.
fxc_status grow_frame_info(fxc_scan* s, uint64_t nf) {
  if (nf > s->finfo_cap) {
    // growing frees the old buffer; cudaFree waits for the work that reads it
    cudaFree(s->d_finfo);
    s->d_finfo = nullptr;
    s->finfo_cap = 0;
    const uint64_t cap = std::max<uint64_t>(nf, 1u << 17);
    CK(cudaMalloc(&s->d_finfo, cap * sizeof(FrameInfo)));
    s->finfo_cap = cap;
  }
  return FXC_OK;
}

// Per-frame delay records for nf frames starting at `first` (FP64 delay model,
// one thread per frame) into the scan's record buffer, on stream st.
fxc_status stage_frame_info(fxc_scan* s, uint64_t first, uint64_t nf, cudaStream_t st) {
  const fxc_status g = grow_frame_info(s, nf);
  if (g != FXC_OK) return g;
  CK(launch_frame_info(delay_params(s), first, nf, (int)s->n, s->cfg.fs_hz / (double)s->n,
                       (int)s->cfg.a1s, (int)s->cfg.a2s, s->d_finfo, st));
  return FXC_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

fxc_status check_device_inputs(const fxc_scan* s, const uint8_t* r1, const uint8_t* r2) {
  if (!s) return fail(FXC_EINVAL, "scan is NULL");
  if (!r1 || !r2) return fail(FXC_EINVAL, "device input pointer is NULL");
  if (!aligned16(r1) || !aligned16(r2))
    return fail(FXC_EINVAL, "device inputs must be 16-byte aligned");
  return FXC_OK;
}

fxc_status validate_cfg(const fxc_scan_cfg* c) {
  const uint32_t n = c->fft_len;
  if (!(n == 1024 || n == 2048 || n == 4096 || n == 8192 || n == 16384 || n == 32768 ||
        n == 65536))
    return fail(FXC_EUNSUPPORTED, "fft_len %u not supported (powers of two 1024..65536)", n);
  for (uint32_t b : {c->bits1, c->bits2})
    if (!(b == 1 || b == 2 || b == 4 || b == 8))
      return fail(FXC_EUNSUPPORTED, "bits %u not supported (1, 2, 4, 8)", b);
  if (c->nlevels1 != (1u << c->bits1) || c->nlevels2 != (1u << c->bits2))
    return fail(FXC_EINVAL, "Expected %u / %u levels, received %u / %u", 1u << c->bits1,
                1u << c->bits2, c->nlevels1, c->nlevels2);
  if (c->bits_out != std::max(c->bits1, c->bits2))
    return fail(FXC_EINVAL, "bits_out must be max(bits1, bits2)");
  for (int k = 0; k < 2; ++k) {
    const uint8_t* sh = k ? c->shuffle2 : c->shuffle1;
    uint32_t seen = 0;
    for (int i = 0; i < 32; ++i) {
      if (sh[i] > 31) return fail(FXC_EINVAL, "Shuffle map must be a permutation of 0..31");
      seen |= 1u << sh[i];
    }
    if (seen != 0xFFFFFFFFu) return fail(FXC_EINVAL, "Shuffle map must be a permutation of 0..31");
  }
  const uint32_t h = n / 2 + 1;
  if (c->a1e <= c->a1s) return fail(FXC_EINVAL, "No band overlap");
  if (c->a1e > h || c->a2s + (c->a1e - c->a1s) > h)
    return fail(FXC_EINVAL, "band alignment outside the spectrum");
  if ((int64_t)c->a2s - (int64_t)c->a1s != (int64_t)c->shift_bins)
    return fail(FXC_EINVAL, "a2s must equal a1s + shift_bins");
  if (c->grid != 0 && c->grid != 1) return fail(FXC_EINVAL, "grid must be 0 (ant1) or 1 (ant2)");
  if (!(c->fs_hz > 0.0) || !(c->delay.fs > 0.0)) return fail(FXC_EINVAL, "sample rate must be > 0");
  if (c->delay.geom_table && c->delay.geom_len == 0)
    return fail(FXC_EINVAL, "geometric delay table is empty");
  if (c->products & ~31u) return fail(FXC_EINVAL, "unknown product flags");
  if ((c->products & (FXC_PROD_PHASED | FXC_PROD_RAW)) && !(c->w1 == c->w1 && c->w2 == c->w2))
    return fail(FXC_EINVAL, "phased weights must be numbers");
  return FXC_OK;
}

fxc_status grow_host(uint8_t** p, uint64_t* cap, uint64_t need) {
  if (*cap >= need) return FXC_OK;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  const uint64_t want = std::max<uint64_t>(need, 16);
  CK(cudaMallocHost(p, want));
  *cap = want;
  return FXC_OK;
}

fxc_status run_corr_stage(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                          uint64_t first, int grid, double* d_acc, cudaStream_t st);

LargeParams large_params(const fxc_scan* s, const uint8_t* r1, const uint8_t* r2) {
  LargeParams p{};
  station_params(s, r1, r2, p.st);
  p.finfo = s->d_finfo;
  p.tw = s->d_twl;
  p.n = (int32_t)s->n;
  p.c = (int32_t)(s->n / 8192);
  p.a1s = (int32_t)s->cfg.a1s;
  p.a1e = (int32_t)s->cfg.a1e;
  p.a2s = (int32_t)s->cfg.a2s;
  p.grid = s->cfg.grid;
  p.products = s->cfg.products;
  p.err = s->d_err;
  return p;
}

// The phased kernels' parameters of a sector (every phased kernel, per scan or
// batched).  The frame records of the sector must already be staged.
PhasedParams phased_params(const fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                           uint64_t first, uint8_t* d_raw_out) {
  PhasedParams p{};
  station_params(s, r1, r2, p.st);
  p.dl = delay_params(s);
  p.nf = nf;
  p.first_frame = first;
  p.a1s = (int32_t)s->cfg.a1s;
  p.a1e = (int32_t)s->cfg.a1e;
  p.a2s = (int32_t)s->cfg.a2s;
  p.grid = s->cfg.grid;
  const int fpc = corr_frames_per_cta_iter(s->n);
  p.stage_bytes = (uint32_t)fpc * (s->bpf1 + s->bpf2);
  p.flush_every = (uint32_t)std::max(1, 32 / fpc);
  p.bits_out = s->cfg.bits_out;
  p.bpf_out = s->bpfo;
  p.out_lsb = (s->cfg.lsb1 && s->cfg.lsb2) ? 1 : 0;  // output_lsb (main.rs:1093)
  p.want_raw = (s->cfg.products & FXC_PROD_RAW) && d_raw_out ? 1 : 0;
  p.w1 = (float)s->cfg.w1;
  p.w2 = (float)s->cfg.w2;
  p.qlevels = s->d_qlevels;
  p.nqlevels = s->cfg.nlevels1;
  p.qmonotonic = s->qmonotonic;
  p.enc_lut = s->d_enc_lut;
  p.finfo = s->d_finfo;
  p.partials = s->d_partials;
  p.raw_out = d_raw_out;
  p.err = s->d_err;
  return p;
}

// FFT lengths above 8192: per batch of frames one decode + four-step FFT,
// then the ACF/XCF accumulation and/or the phased synthesis (+ inverse FFT and
// re-quantisation) on the same spectra; fixed-order reductions at the end.
fxc_status run_large(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                     uint64_t first, double* d_acc, uint8_t* d_raw_out, bool corr, bool phased,
                     bool corr_done, cudaStream_t st) {
  if (!corr && !phased) return FXC_OK;
  const uint32_t h = s->h;
  const LargeParams p = large_params(s, r1, r2);
  PhasedParams pp{};
  if (phased) pp = phased_params(s, r1, r2, nf, first, d_raw_out);
  // frame groups of a batch (one f64 partial row each): as few as keep every
  // group within 32 frames, the f32 run length of the accumulation kernels
  const int groups = (int)std::max<uint64_t>(
      1, std::min<uint64_t>((uint64_t)kLargeGroups, (s->big_frames + 31) / 32));
  double* part_ph = s->d_partials + (uint64_t)kLargeGroups * 4 * h;
  bool first_batch = true;
  for (uint64_t f0 = 0; f0 < nf; f0 += s->big_frames) {
    const uint64_t nb = std::min(s->big_frames, nf - f0);
    CK(launch_large_fft(p, f0, nb, s->d_big[0], s->d_big[1], s->eng->sm_count, st));
    s->all_launches += 3;
    if (corr) {
      CK(launch_large_acc(p, s->d_big[1], f0, nb, groups, first_batch ? 1 : 0, s->d_partials, st));
      s->all_launches += 1;
    }
    if (phased) {
      CK(launch_large_phased(p, pp, s->d_big[0], s->d_big[1], f0, nb, groups, first_batch ? 1 : 0,
                             part_ph, s->eng->sm_count, st));
      s->all_launches += pp.want_raw ? 4 : 1;
    }
    first_batch = false;
  }
  if (corr) {
    const double u1 = 1.0 / s->scale[0], u2 = 1.0 / s->scale[1];
    CK(launch_reduce(s->d_partials, groups, (int)h, 0.25 * u1 * u1, 0.25 * u2 * u2,
                     0.25 * u1 * u2, d_acc, st));
    s->all_launches += 1;
    s->kernel_launches += 1;
  } else if (!corr_done) {
    CK(cudaMemsetAsync(d_acc, 0, sizeof(double) * 5 * h, st));
  }
  if (phased) {
    CK(launch_reduce_phased(part_ph, groups, (int)h, d_acc, st));
    s->all_launches += 1;
  }
  return FXC_OK;
}

fxc_status run_sector_device(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                             uint64_t first, double* d_acc, uint8_t* d_raw_out, cudaStream_t st) {
  const uint32_t h = s->h;
  const bool corr = (s->cfg.products & (FXC_PROD_ACF | FXC_PROD_XCF)) != 0;
  const bool phased = (s->cfg.products & (FXC_PROD_PHASED | FXC_PROD_RAW)) != 0;
  if (nf == 0 || !(corr || phased)) {
    CK(cudaMemsetAsync(d_acc, 0, sizeof(double) * 5 * h, st));
    return FXC_OK;
  }
  if ((s->cfg.products & FXC_PROD_RAW) && !d_raw_out)
    return fail(FXC_EINVAL, "the scan writes phased .raw frames but d_raw_out is NULL");
  const int grid = corr_grid(s, nf);
  fxc_status fst = stage_frame_info(s, first, nf, st);
  if (fst != FXC_OK) return fst;
  s->all_launches += 1;
  if (s->n > 8192) {
    // correlation: the two-row shared-memory kernel for FFT 16384 with an even
    // band shift, else the cluster kernel; the four-step path when neither
    // can run (and for the phased products)
    bool corr_done = false;
    if (corr && (corr_cluster_capacity(s->n) > 0 ||
                 (s->n == 16384 && corr_fold2_supported(corr_params(s, r1, r2, nf, first))))) {
      fst = run_corr_stage(s, r1, r2, nf, first, grid, d_acc, st);
      if (fst != FXC_OK) return fst;
      corr_done = true;
    }
    // phased products: the two-row kernel (FFT 16384, any bit depth) or, with
    // 1- and 2-bit stations, the cluster pair kernel (32768 / 65536, band
    // shift a multiple of C); else the four-step path
    if (phased) {
      const PhasedParams pp = phased_params(s, r1, r2, nf, first, d_raw_out);
      if (phased_pair_supported(s->n, pp)) {
        if (!corr) CK(cudaMemsetAsync(d_acc, 0, sizeof(double) * 5 * h, st));
        const int g = phased_pair_grid(s->eng->sm_count, nf);
        CK(launch_phased_pair(pp, g, st));
        CK(launch_reduce_phased(s->d_partials, g, (int)h, d_acc, st));
        s->all_launches += 2;
        return run_large(s, r1, r2, nf, first, d_acc, d_raw_out, corr && !corr_done, false, true,
                         st);
      }
      if (phased_cpair_supported(s->n, pp)) {
        if (!corr) CK(cudaMemsetAsync(d_acc, 0, sizeof(double) * 5 * h, st));
        if (pp.want_raw) CK(cudaMemsetAsync(d_raw_out, 0, (size_t)nf * s->bpfo, st));
        const int g = phased_cpair_count(s->n, nf);
        CK(launch_phased_cpair(s->n, pp, g, st));
        CK(launch_reduce_phased(s->d_partials, g, (int)h, d_acc, st));
        s->all_launches += 2;
        return run_large(s, r1, r2, nf, first, d_acc, d_raw_out, corr && !corr_done, false, true,
                         st);
      }
    }
    return run_large(s, r1, r2, nf, first, d_acc, d_raw_out, corr && !corr_done, phased, corr_done,
                     st);
  }
  if (!corr) {
    CK(cudaMemsetAsync(d_acc, 0, sizeof(double) * 5 * h, st));
  } else {
    fst = run_corr_stage(s, r1, r2, nf, first, grid, d_acc, st);
    if (fst != FXC_OK) return fst;
  }
  if (phased) {
    PhasedParams pp = phased_params(s, r1, r2, nf, first, d_raw_out);
    CK(launch_phased(s->n, pp, grid, st));
    CK(launch_reduce_phased(s->d_partials, grid, (int)h, d_acc, st));
    s->all_launches += 2;
  }
  return FXC_OK;
}

fxc_status run_corr_stage(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                          uint64_t first, int grid, double* d_acc, cudaStream_t st) {
  const uint32_t h = s->h;
  CorrParams p = corr_params(s, r1, r2, nf, first);
  std::pair<cudaEvent_t, cudaEvent_t>* ev = nullptr;
  if (s->profiling) {
    if (s->prof_used == s->prof_events.size()) {
      std::pair<cudaEvent_t, cudaEvent_t> pr;
      CK(cudaEventCreate(&pr.first));
      CK(cudaEventCreate(&pr.second));
      s->prof_events.push_back(pr);
    }
    ev = &s->prof_events[s->prof_used++];
    CK(cudaEventRecord(ev->first, st));
  }
  int nblk = grid;  // partial rows to reduce
  if (s->n > 8192 && corr_pair_supported(s->n, p)) {
    nblk = corr_pair_count(s->n, nf);
    CK(launch_corr_pair(s->n, p, nblk, st));
  } else if (s->n > 8192 && !(s->n == 16384 && corr_fold2_supported(p))) {
    nblk = corr_cluster_count(s->n, nf);
    if (nblk <= 0) return fail(FXC_EUNSUPPORTED, "no cluster of %d CTAs fits this GPU",
                               corr_cluster_size(s->n));
    CK(launch_corr_cluster(s->n, p, nblk, st));
  } else {
    CK(launch_corr(s->n, MODE_CORR, p, grid, st));
  }
  if (ev) CK(cudaEventRecord(ev->second, st));
  const double u1 = 1.0 / s->scale[0], u2 = 1.0 / s->scale[1];
  CK(launch_reduce(s->d_partials, nblk, (int)h, 0.25 * u1 * u1, 0.25 * u2 * u2, 0.25 * u1 * u2,
                   d_acc, st));
  s->kernel_launches += 1;
  s->all_launches += 2;
  return FXC_OK;
}

// Reserves `delta` more bytes of the engine's HBM budget for scan s.
fxc_status reserve(fxc_scan* s, uint64_t delta) {
  if (!delta) return FXC_OK;
  std::lock_guard<std::mutex> lk(s->eng->mu);
  if (s->eng->in_use + delta > s->eng->budget)
    return fail(FXC_EBUSY, "HBM budget exhausted (%llu + %llu > %llu bytes)",
                (unsigned long long)s->eng->in_use, (unsigned long long)delta,
                (unsigned long long)s->eng->budget);
  s->eng->in_use += delta;
  s->hbm_bytes += delta;
  return FXC_OK;
}

// Device buffer of at least `need` bytes, growth charged to the budget.
fxc_status grow_charged(fxc_scan* s, uint8_t** p, uint64_t* cap, uint64_t need) {
  if (*cap >= need) return FXC_OK;
  const uint64_t want = std::max<uint64_t>(need, 16);
  fxc_status st = reserve(s, want - *cap);
  if (st != FXC_OK) return st;
  const uint64_t old = *cap;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const cudaError_t e = cudaMalloc(p, want);
  if (e != cudaSuccess) {
    std::lock_guard<std::mutex> lk(s->eng->mu);
    s->eng->in_use -= std::min(s->eng->in_use, want);
    s->hbm_bytes -= std::min(s->hbm_bytes, want);
    (void)old;
    return fail(e == cudaErrorMemoryAllocation ? FXC_ENOMEM : FXC_ECUDA, "cudaMalloc: %s",
                cudaGetErrorString(e));
  }
  *cap = want;
  return FXC_OK;
}

// Takes a free sector slot of scan s and copies the sector's host inputs
// into its device buffers on the scan's copy stream (event ev_h2d after).
fxc_status stage_sector(fxc_scan* s, const uint8_t* raw1, uint64_t n1, const uint8_t* raw2,
                        uint64_t n2, uint64_t nf, SectorSlot** out) {
  if (nf && (!raw1 || !raw2)) return fail(FXC_EINVAL, "input buffer is NULL");
  const uint64_t need1 = nf * s->bpf1, need2 = nf * s->bpf2;
  if (n1 < need1 || n2 < need2)
    return fail(FXC_EINVAL, "input too short: need %llu / %llu bytes for %llu frames",
                (unsigned long long)need1, (unsigned long long)need2, (unsigned long long)nf);
  SectorSlot* sl = nullptr;
  for (auto& x : s->slots)
    if (!x.busy) {
      sl = &x;
      break;
    }
  if (!sl) return fail(FXC_EBUSY, "all %zu sector slots are in flight; wait for one first",
                       s->slots.size());
  fxc_status st;
  if ((st = grow_charged(s, &sl->d_raw1, &sl->cap1, need1)) != FXC_OK) return st;
  if ((st = grow_charged(s, &sl->d_raw2, &sl->cap2, need2)) != FXC_OK) return st;
  if (nf) {
    CK(cudaMemcpyAsync(sl->d_raw1, raw1, need1, cudaMemcpyHostToDevice, s->copy_stream));
    CK(cudaMemcpyAsync(sl->d_raw2, raw2, need2, cudaMemcpyHostToDevice, s->copy_stream));
  }
  const bool raw = (s->cfg.products & FXC_PROD_RAW) != 0;
  const uint64_t need_o = nf * s->bpfo;
  if (raw) {
    if ((st = grow_charged(s, &sl->d_rawout, &sl->cap_out, need_o)) != FXC_OK) return st;
    if ((st = grow_host(&sl->h_rawout, &sl->hcap_out, need_o)) != FXC_OK) return st;
  }
  CK(cudaEventRecord(sl->ev_h2d, s->copy_stream));
  sl->nf = nf;
  *out = sl;
  return FXC_OK;
}

// Device-to-host copies of a computed sector (ordered on the scan's compute
// stream), then ev_done; marks the slot in flight under a new id.
fxc_status collect_sector(fxc_scan* s, SectorSlot* sl) {
  const bool raw = (s->cfg.products & FXC_PROD_RAW) != 0;
  const uint64_t need_o = sl->nf * s->bpfo;
  CK(cudaMemcpyAsync(sl->h_acc, sl->d_acc, sizeof(double) * 5 * s->h, cudaMemcpyDeviceToHost,
                     s->stream));
  if (raw && need_o)
    CK(cudaMemcpyAsync(sl->h_rawout, sl->d_rawout, need_o, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(reinterpret_cast<uint8_t*>(sl->h_acc) + sizeof(double) * 5 * s->h, s->d_err,
                     4, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaEventRecord(sl->ev_done, s->stream));
  sl->busy = true;
  sl->id = s->next_id++;
  return FXC_OK;
}

}  // namespace

namespace fxc {

fxc_status sector_stage(fxc_scan* s, const uint8_t* raw1, uint64_t n1, const uint8_t* raw2,
                        uint64_t n2, uint64_t nf, StagedSector* out) {
  if (!s || !out) return fail(FXC_EINVAL, "NULL argument");
  DeviceGuard g(s->eng->device);
  SectorSlot* sl = nullptr;
  fxc_status st = stage_sector(s, raw1, n1, raw2, n2, nf, &sl);
  if (st != FXC_OK) return st;
  sl->busy = true;  // reserved until sector_collect
  out->slot = (uint32_t)(sl - s->slots.data());
  out->d_raw1 = sl->d_raw1;
  out->d_raw2 = sl->d_raw2;
  out->d_acc = sl->d_acc;
  out->d_raw_out = (s->cfg.products & FXC_PROD_RAW) ? sl->d_rawout : nullptr;
  out->h2d = sl->ev_h2d;
  return FXC_OK;
}

fxc_status sector_collect(fxc_scan* s, const StagedSector& ss, cudaEvent_t computed,
                          uint64_t* sector_id) {
  DeviceGuard g(s->eng->device);
  SectorSlot* sl = &s->slots[ss.slot];
  sl->busy = false;
  if (computed) CK(cudaStreamWaitEvent(s->stream, computed, 0));
  const fxc_status st = collect_sector(s, sl);
  if (st != FXC_OK) return st;
  *sector_id = sl->id;
  return FXC_OK;
}

void sector_release(fxc_scan* s, const StagedSector& ss) {
  DeviceGuard g(s->eng->device);
  SectorSlot* sl = &s->slots[ss.slot];
  cudaEventSynchronize(sl->ev_h2d);  // its copies may still be in flight
  sl->busy = false;
}

fxc_status upload_tables(fxc_scan* s, const fxc_scan_cfg* cfg, uint64_t tlen);

// Binds scan s to cfg: derived sizes, buffers grown (and charged to the HBM
// budget) where the new configuration needs more, tables uploaded on the
// scan's compute stream from pinned staging.  Rebinding an idle scan to
// another configuration is the serving loop's way of reusing the device
// state of a finished job; nothing is freed until the scan closes.
fxc_status scan_bind(fxc_scan* s, const fxc_scan_cfg* cfg) {
  fxc_status st = validate_cfg(cfg);
  if (st != FXC_OK) return st;
  for (const auto& sl : s->slots)
    if (sl.busy) return fail(FXC_EBUSY, "scan has sectors in flight");
  fxc_engine* e = s->eng;
  DeviceGuard g(e->device);
  const uint32_t n = cfg->fft_len, h = n / 2 + 1;
  const uint64_t maxg = n > 8192 ? (uint64_t)kLargeGroups
                                 : (uint64_t)e->sm_count * (uint64_t)corr_ctas_per_sm(n);
  // N > 8192: [group][4][H] correlation partials, then [group][H] phased partials;
  // also the two-row kernel's [CTA][4][H] (N = 16384) and the cluster
  // kernel's [cluster][4][H]
  uint64_t pel = maxg * (n > 8192 ? 5 : 4) * h;
  if (n == 16384) pel = std::max<uint64_t>(pel, (uint64_t)e->sm_count * 4 * h);
  if (n > 8192) {
    // clusters of C CTAs, or of C/2 (two rows per CTA) at FFT 32768 / 65536
    const uint64_t c = (uint64_t)corr_cluster_size(n) / (n > 16384 ? 2 : 1);
    pel = std::max<uint64_t>(pel, ((uint64_t)e->sm_count + c - 1) / c * 4 * h);
  }
  const uint64_t bigf = n > 8192 ? (uint64_t)large_batch_frames(n) : 0;
  const uint64_t bige = bigf * (uint64_t)n;
  const uint64_t tlen = cfg->delay.geom_table ? cfg->delay.geom_len : 0;
  // the previous configuration's work must be done before buffers are reused
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaStreamSynchronize(s->copy_stream));
  if (pel > s->partials_cap) {
    uint8_t* p = reinterpret_cast<uint8_t*>(s->d_partials);
    uint64_t cap = s->partials_cap * 8;
    if ((st = grow_charged(s, &p, &cap, pel * 8)) != FXC_OK) return st;
    s->d_partials = reinterpret_cast<double*>(p);
    s->partials_cap = cap / 8;
  }
  if (bige > s->big_cap) {
    for (int b = 0; b < 2; ++b) {
      uint8_t* p = reinterpret_cast<uint8_t*>(s->d_big[b]);
      uint64_t cap = s->big_cap * sizeof(float2);
      if ((st = grow_charged(s, &p, &cap, bige * sizeof(float2))) != FXC_OK) return st;
      s->d_big[b] = reinterpret_cast<float2*>(p);
    }
    s->big_cap = bige;
  }
  if (n > 8192 && n > s->twl_cap) {
    uint8_t* p = reinterpret_cast<uint8_t*>(s->d_twl);
    uint64_t cap = s->twl_cap * sizeof(float2);
    if ((st = grow_charged(s, &p, &cap, (uint64_t)n * sizeof(float2))) != FXC_OK) return st;
    s->d_twl = reinterpret_cast<float2*>(p);
    s->twl_cap = cap / sizeof(float2);
  }
  if (n > 8192) CK(launch_twiddle_table((int)n, s->d_twl, s->stream));
  if (tlen > s->table_cap) {
    uint8_t* p = reinterpret_cast<uint8_t*>(s->d_table);
    uint64_t cap = s->table_cap * 8;
    if ((st = grow_charged(s, &p, &cap, tlen * 8)) != FXC_OK) return st;
    s->d_table = reinterpret_cast<double*>(p);
    s->table_cap = cap / 8;
  }
  if (h > s->acc_cap) {
    for (auto& sl : s->slots) {
      uint8_t* p = reinterpret_cast<uint8_t*>(sl.d_acc);
      uint64_t cap = (uint64_t)s->acc_cap * 5 * 8;
      if ((st = grow_charged(s, &p, &cap, (uint64_t)h * 5 * 8)) != FXC_OK) return st;
      sl.d_acc = reinterpret_cast<double*>(p);
      if (sl.h_acc) cudaFreeHost(sl.h_acc);
      sl.h_acc = nullptr;
      CK(cudaMallocHost(&sl.h_acc, sizeof(double) * 5 * h + 16));
    }
    s->acc_cap = h;
  }
  // the decode tables of a scan rebound to the same levels and shuffles are
  // already on the device (the serving loop's common case)
  const bool reuse = s->n != 0 && tlen == 0 && cfg->nlevels1 == s->cfg.nlevels1 &&
                     cfg->nlevels2 == s->cfg.nlevels2 &&
                     !std::memcmp(cfg->levels1, s->cfg.levels1, 8 * cfg->nlevels1) &&
                     !std::memcmp(cfg->levels2, s->cfg.levels2, 8 * cfg->nlevels2) &&
                     !std::memcmp(cfg->shuffle1, s->cfg.shuffle1, 32) &&
                     !std::memcmp(cfg->shuffle2, s->cfg.shuffle2, 32);
  if (!reuse && (st = upload_tables(s, cfg, tlen)) != FXC_OK) return st;

  s->cfg = *cfg;
  s->cfg.delay.geom_table = nullptr;  // the host pointer is not kept
  s->table_bound = tlen != 0;
  s->n = n;
  s->h = h;
  s->bpf1 = (uint32_t)fxc_bytes_per_frame(n, cfg->bits1);
  s->bpf2 = (uint32_t)fxc_bytes_per_frame(n, cfg->bits2);
  s->bpfo = (uint32_t)fxc_bytes_per_frame(n, cfg->bits_out);
  s->shkind[0] = shuffle_kind(cfg->shuffle1);
  s->shkind[1] = shuffle_kind(cfg->shuffle2);
  s->scale[0] = level_scale(cfg->levels1, cfg->nlevels1);
  s->scale[1] = level_scale(cfg->levels2, cfg->nlevels2);
  s->partials_elems = pel;
  s->big_frames = bigf;
  return FXC_OK;
}

// Decode / re-quantiser tables and the geometric table into pinned staging,
// then one async upload each on the scan's compute stream.
fxc_status upload_tables(fxc_scan* s, const fxc_scan_cfg* cfg, uint64_t tlen) {
  fxc_status st;
  constexpr uint64_t kLut = 0, kLv = 8192, kSh = kLv + 2048, kQl = kSh + 32, kEnc = kQl + 1024,
                     kTab = kEnc + 4096;
  if ((st = grow_host(&s->h_tab, &s->h_tab_cap, kTab + tlen * 8)) != FXC_OK) return st;
  uint32_t* lut = reinterpret_cast<uint32_t*>(s->h_tab + kLut);
  float* lv = reinterpret_cast<float*>(s->h_tab + kLv);
  float* ql = reinterpret_cast<float*>(s->h_tab + kQl);
  uint32_t* enc = reinterpret_cast<uint32_t*>(s->h_tab + kEnc);
  build_lut(cfg->shuffle1, lut);
  build_lut(cfg->shuffle2, lut + 1024);
  for (int i = 0; i < 512; ++i) lv[i] = 0.0f;
  for (uint32_t i = 0; i < cfg->nlevels1; ++i) lv[i] = (float)cfg->levels1[i];
  for (uint32_t i = 0; i < cfg->nlevels2; ++i) lv[256 + i] = (float)cfg->levels2[i];
  std::memcpy(s->h_tab + kSh, cfg->shuffle1, 32);
  // phased re-quantiser: ant1's levels as f32 (quantise_frame compares
  // |x - lv as f32|) and the encode LUT of ant1's shuffle: packed bit pos
  // goes to bit shuffle1[pos] (utils.rs:395)
  std::memcpy(ql, lv, 256 * sizeof(float));
  std::memset(enc, 0, 1024 * sizeof(uint32_t));
  for (int pos = 0; pos < 32; ++pos)
    for (int v = 0; v < 256; ++v)
      if ((v >> (pos & 7)) & 1) enc[(pos >> 3) * 256 + v] |= 1u << cfg->shuffle1[pos];
  bool up = true, down = true;
  for (uint32_t i = 1; i < cfg->nlevels1; ++i) {
    if (!(lv[i] > lv[i - 1])) up = false;
    if (!(lv[i] < lv[i - 1])) down = false;
  }
  if (tlen) std::memcpy(s->h_tab + kTab, cfg->delay.geom_table, tlen * 8);
  CK(cudaMemcpyAsync(s->d_lut, lut, 8192, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->d_levels, lv, 2048, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->d_shuffle_out, s->h_tab + kSh, 32, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->d_qlevels, ql, 1024, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->d_enc_lut, enc, 4096, cudaMemcpyHostToDevice, s->stream));
  if (tlen)
    CK(cudaMemcpyAsync(s->d_table, s->h_tab + kTab, tlen * 8, cudaMemcpyHostToDevice, s->stream));
  // the copy stream's first transfer of a sector must not overtake the uploads
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, s->stream));
  CK(cudaStreamWaitEvent(s->copy_stream, ev, 0));
  cudaEventDestroy(ev);
  s->qmonotonic = up ? 1 : (down ? -1 : 0);
  return FXC_OK;
}


}  // namespace fxc

// ======================================================================= ABI

extern "C" {

int32_t fxc_abi_version(void) { return FXC_ABI_VERSION; }

const char* fxc_status_string(fxc_status s) {
  switch (s) {
    case FXC_OK: return "ok";
    case FXC_EINVAL: return "invalid argument";
    case FXC_ENOMEM: return "out of memory";
    case FXC_ECUDA: return "CUDA error";
    case FXC_ETIMEDOUT: return "timed out";
    case FXC_ENOTFOUND: return "not found";
    case FXC_EBUSY: return "busy";
    case FXC_EUNSUPPORTED: return "unsupported";
    case FXC_EDEVICE: return "device-reported error";
    default: return "unknown status";
  }
}

const char* fxc_last_error(void) { return g_err.c_str(); }

fxc_status fxc_engine_create(const fxc_device_opts* opts, fxc_engine** out) {
  if (!out) return fail(FXC_EINVAL, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  const int dev = opts ? opts->device : 0;
  if (dev < 0 || dev >= ndev) return fail(FXC_EINVAL, "device %d out of range (0..%d)", dev, ndev - 1);
  DeviceGuard g(dev);
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major < 10)
    return fail(FXC_EUNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a", dev,
                prop.major, prop.minor);
  auto* e = new fxc_engine();
  e->device = dev;
  e->sm_count = prop.multiProcessorCount;
  e->max_inflight = (opts && opts->max_inflight > 0) ? opts->max_inflight : 2;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  e->budget = (opts && opts->hbm_budget_bytes) ? opts->hbm_budget_bytes : (uint64_t)(0.8 * free_b);
  *out = e;
  return FXC_OK;
}

fxc_status fxc_engine_destroy(fxc_engine* e) {
  if (!e) return FXC_OK;
  std::vector<fxc_server*> live;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    live = e->servers;
  }
  for (fxc_server* sv : live) fxc_server_destroy(sv);
  std::vector<fxc_batch*> bl;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    bl = e->batches;
  }
  for (fxc_batch* b : bl) fxc_batch_destroy(b);
  std::vector<fxc_scan*> open;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    open = e->scans;
  }
  for (fxc_scan* s : open) fxc_scan_close(s);
  delete e;
  return FXC_OK;
}

fxc_status fxc_scan_open(fxc_engine* e, const fxc_scan_cfg* cfg, fxc_scan** out) {
  if (!e || !cfg || !out) return fail(FXC_EINVAL, "NULL argument");
  *out = nullptr;
  fxc_status st = validate_cfg(cfg);
  if (st != FXC_OK) return st;
  DeviceGuard g(e->device);
  auto* s = new fxc_scan();
  s->eng = e;
  auto cleanup = [&](fxc_status r) {
    fxc_scan_close(s);
    return r;
  };
#define CKS(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return cleanup(fail(e_ == cudaErrorMemoryAllocation ? FXC_ENOMEM : FXC_ECUDA, "%s: %s", \
                          #call, cudaGetErrorString(e_)));                                 \
  } while (0)
  CKS(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  CKS(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
  CKS(cudaMalloc(&s->d_lut, 2 * 1024 * sizeof(uint32_t)));
  CKS(cudaMalloc(&s->d_levels, 2 * 256 * sizeof(float)));
  CKS(cudaMalloc(&s->d_shuffle_out, 32));
  CKS(cudaMalloc(&s->d_qlevels, 256 * sizeof(float)));
  CKS(cudaMalloc(&s->d_enc_lut, 1024 * sizeof(uint32_t)));
  CKS(cudaMalloc(&s->d_err, 16));
  CKS(cudaMemset(s->d_err, 0, 16));
  s->slots.resize((size_t)e->max_inflight);
  for (auto& sl : s->slots) {
    CKS(cudaEventCreateWithFlags(&sl.ev_h2d, cudaEventDisableTiming));
    // a waiting host thread sleeps until the sector is done instead of polling
    CKS(cudaEventCreateWithFlags(&sl.ev_done, cudaEventDisableTiming | cudaEventBlockingSync));
  }
#undef CKS
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->scans.push_back(s);
  }
  st = scan_bind(s, cfg);
  if (st != FXC_OK) {
    const std::string msg = g_err;
    fxc_scan_close(s);
    g_err = msg;
    return st;
  }
  CK(cudaStreamSynchronize(s->stream));
  *out = s;
  return FXC_OK;
}

fxc_status fxc_scan_close(fxc_scan* s) {
  if (!s) return FXC_OK;
  DeviceGuard g(s->eng->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
  for (auto& sl : s->slots) {
    cudaFree(sl.d_raw1);
    cudaFree(sl.d_raw2);
    cudaFree(sl.d_acc);
    cudaFree(sl.d_rawout);
    cudaFreeHost(sl.h_acc);
    cudaFreeHost(sl.h_rawout);
    if (sl.ev_h2d) cudaEventDestroy(sl.ev_h2d);
    if (sl.ev_done) cudaEventDestroy(sl.ev_done);
  }
  for (auto& pr : s->prof_events) {
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  cudaFree(s->d_partials);
  cudaFree(s->d_big[0]);
  cudaFree(s->d_big[1]);
  cudaFree(s->d_twl);
  cudaFree(s->d_finfo);
  cudaFree(s->d_lut);
  cudaFree(s->d_levels);
  cudaFree(s->d_shuffle_out);
  cudaFree(s->d_qlevels);
  cudaFree(s->d_enc_lut);
  cudaFree(s->d_err);
  cudaFree(s->d_table);
  cudaFreeHost(s->h_tab);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  {
    std::lock_guard<std::mutex> lk(s->eng->mu);
    s->eng->in_use -= std::min(s->eng->in_use, s->hbm_bytes);
    auto& v = s->eng->scans;
    v.erase(std::remove(v.begin(), v.end(), s), v.end());
  }
  delete s;
  return FXC_OK;
}

fxc_status fxc_sector_run_device(fxc_scan* s, const uint8_t* d_raw1, const uint8_t* d_raw2,
                                 uint64_t nf, uint64_t first_frame, double* d_acc,
                                 uint8_t* d_raw_out, void* stream) {
  (void)d_raw_out;
  fxc_status st = check_device_inputs(s, d_raw1, d_raw2);
  if (st != FXC_OK) return st;
  if (!d_acc) return fail(FXC_EINVAL, "d_acc is NULL");
  DeviceGuard g(s->eng->device);
  return run_sector_device(s, d_raw1, d_raw2, nf, first_frame, d_acc, d_raw_out,
                           (cudaStream_t)stream);
}

fxc_status fxc_scan_check(fxc_scan* s) {
  if (!s) return fail(FXC_EINVAL, "scan is NULL");
  DeviceGuard g(s->eng->device);
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaDeviceSynchronize());
  uint32_t err = 0;
  CK(cudaMemcpy(&err, s->d_err, 4, cudaMemcpyDeviceToHost));
  CK(cudaMemset(s->d_err, 0, 4));
  return internal_device_error(err);
}

fxc_status fxc_debug_inject_wait_timeout(uint32_t wait_polls, int32_t withhold_copies) {
  g_dbg_polls.store(wait_polls);
  g_dbg_flags.store(withhold_copies ? DBG_WITHHOLD_COPIES : 0u);
  return FXC_OK;
}

fxc_status fxc_scan_set_profiling(fxc_scan* s, int32_t enable) {
  if (!s) return fail(FXC_EINVAL, "scan is NULL");
  s->profiling = enable != 0;
  return FXC_OK;
}

fxc_status fxc_scan_profile(fxc_scan* s, double* kernel_ms, uint64_t* kernel_launches,
                            uint64_t* all_launches, int32_t reset) {
  if (!s) return fail(FXC_EINVAL, "scan is NULL");
  DeviceGuard g(s->eng->device);
  double total = 0.0;
  for (size_t i = 0; i < s->prof_used; ++i) {
    CK(cudaEventSynchronize(s->prof_events[i].second));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s->prof_events[i].first, s->prof_events[i].second));
    total += ms;
  }
  if (kernel_ms) *kernel_ms = total;
  if (kernel_launches) *kernel_launches = s->kernel_launches;
  if (all_launches) *all_launches = s->all_launches;
  if (reset) {
    s->prof_used = 0;
    s->kernel_launches = 0;
    s->all_launches = 0;
  }
  return FXC_OK;
}

fxc_status fxc_delay_entries_device(fxc_scan* s, uint64_t first_frame, uint64_t nf,
                                    fxc_frame_delay* d_out, void* stream) {
  if (!s || (!d_out && nf)) return fail(FXC_EINVAL, "NULL argument");
  DeviceGuard g(s->eng->device);
  CK(launch_delay_entries(delay_params(s), first_frame, nf,
                          reinterpret_cast<fxc_frame_delay_dev*>(d_out), (cudaStream_t)stream));
  return FXC_OK;
}

fxc_status fxc_decode_device(fxc_scan* s, const uint8_t* d_raw1, const uint8_t* d_raw2,
                             uint64_t nf, uint64_t first_frame, float* d_x1, float* d_x2,
                             void* stream) {
  fxc_status st = check_device_inputs(s, d_raw1, d_raw2);
  if (st != FXC_OK) return st;
  if (nf == 0) return FXC_OK;
  if (!d_x1 || !d_x2) return fail(FXC_EINVAL, "output pointer is NULL");
  DeviceGuard g(s->eng->device);
  st = stage_frame_info(s, first_frame, nf, (cudaStream_t)stream);
  if (st != FXC_OK) return st;
  if (s->n > 8192) {
    CK(launch_large_decode(large_params(s, d_raw1, d_raw2), 0, nf, d_x1, d_x2,
                           s->eng->sm_count, (cudaStream_t)stream));
    return FXC_OK;
  }
  CorrParams p = corr_params(s, d_raw1, d_raw2, nf, first_frame);
  p.out_a = d_x1;
  p.out_b = d_x2;
  if (s->n == 8192) {
    // the FFT-8192 correlation kernel's decode path (fold_inputs)
    const int grid = (int)std::min<uint64_t>(nf, (uint64_t)s->eng->sm_count * 4);
    CK(launch_fold_decode(p, grid, (cudaStream_t)stream));
    return FXC_OK;
  }
  CK(launch_corr(s->n, MODE_DECODE, p, corr_grid(s, nf), (cudaStream_t)stream));
  return FXC_OK;
}

fxc_status fxc_spectra_device(fxc_scan* s, const uint8_t* d_raw1, const uint8_t* d_raw2,
                              uint64_t nf, uint64_t first_frame, float* d_s1, float* d_s2,
                              void* stream) {
  fxc_status st = check_device_inputs(s, d_raw1, d_raw2);
  if (st != FXC_OK) return st;
  if (nf == 0) return FXC_OK;
  if (!d_s1 || !d_s2) return fail(FXC_EINVAL, "output pointer is NULL");
  DeviceGuard g(s->eng->device);
  st = stage_frame_info(s, first_frame, nf, (cudaStream_t)stream);
  if (st != FXC_OK) return st;
  if (s->n > 8192) {
    const LargeParams lp = large_params(s, d_raw1, d_raw2);
    for (uint64_t f0 = 0; f0 < nf; f0 += s->big_frames) {
      const uint64_t nb = std::min(s->big_frames, nf - f0);
      CK(launch_large_fft(lp, f0, nb, s->d_big[0], s->d_big[1], s->eng->sm_count,
                          (cudaStream_t)stream));
      CK(launch_large_split(lp, s->d_big[1], f0, nb, reinterpret_cast<float2*>(d_s1),
                            reinterpret_cast<float2*>(d_s2), s->eng->sm_count,
                            (cudaStream_t)stream));
    }
    return FXC_OK;
  }
  CorrParams p = corr_params(s, d_raw1, d_raw2, nf, first_frame);
  p.out_a = d_s1;
  p.out_b = d_s2;
  CK(launch_corr(s->n, MODE_SPECTRA, p, corr_grid(s, nf), (cudaStream_t)stream));
  return FXC_OK;
}

fxc_status fxc_sector_submit(fxc_scan* s, const uint8_t* raw1, uint64_t n1, const uint8_t* raw2,
                             uint64_t n2, uint64_t nf, uint64_t first_frame, uint64_t* sector_id) {
  if (!s || !sector_id) return fail(FXC_EINVAL, "NULL argument");
  DeviceGuard g(s->eng->device);
  SectorSlot* sl = nullptr;
  fxc_status st = stage_sector(s, raw1, n1, raw2, n2, nf, &sl);
  if (st != FXC_OK) return st;
  const bool raw = (s->cfg.products & FXC_PROD_RAW) != 0;
  CK(cudaStreamWaitEvent(s->stream, sl->ev_h2d, 0));
  st = run_sector_device(s, sl->d_raw1, sl->d_raw2, nf, first_frame, sl->d_acc,
                         raw ? sl->d_rawout : nullptr, s->stream);
  if (st != FXC_OK) return st;
  if ((st = collect_sector(s, sl)) != FXC_OK) return st;
  *sector_id = sl->id;
  return FXC_OK;
}

fxc_status fxc_sector_wait(fxc_scan* s, uint64_t sector_id, int32_t timeout_ms,
                           fxc_sector_out* out) {
  if (!s) return fail(FXC_EINVAL, "scan is NULL");
  SectorSlot* sl = nullptr;
  for (auto& x : s->slots)
    if (x.busy && x.id == sector_id) sl = &x;
  if (!sl) return fail(FXC_ENOTFOUND, "sector id %llu is not in flight", (unsigned long long)sector_id);
  DeviceGuard g(s->eng->device);
  const auto t0 = std::chrono::steady_clock::now();
  if (timeout_ms < 0) {
    const cudaError_t q = cudaEventSynchronize(sl->ev_done);
    if (q != cudaSuccess) return fail(FXC_ECUDA, "sector failed: %s", cudaGetErrorString(q));
  }
  for (;;) {
    cudaError_t q = cudaEventQuery(sl->ev_done);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) return fail(FXC_ECUDA, "sector failed: %s", cudaGetErrorString(q));
    if (timeout_ms >= 0 &&
        std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(timeout_ms))
      return fail(FXC_ETIMEDOUT, "sector %llu not done after %d ms", (unsigned long long)sector_id,
                  timeout_ms);
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  sl->busy = false;
  const uint32_t h = s->h;
  uint32_t err = 0;
  std::memcpy(&err, reinterpret_cast<uint8_t*>(sl->h_acc) + sizeof(double) * 5 * h, 4);
  if (out) {
    if (out->acf11) std::memcpy(out->acf11, sl->h_acc, sizeof(double) * h);
    if (out->acf22) std::memcpy(out->acf22, sl->h_acc + h, sizeof(double) * h);
    if (out->xcf) std::memcpy(out->xcf, sl->h_acc + 2 * h, sizeof(double) * 2 * h);
    if (out->phased) std::memcpy(out->phased, sl->h_acc + 4 * h, sizeof(double) * h);
    out->frames_failed = 0;
    if (out->raw_out && (s->cfg.products & FXC_PROD_RAW)) {
      const uint64_t need_o = sl->nf * s->bpfo;
      if (out->raw_out_len < need_o)
        return fail(FXC_EINVAL, "raw_out_len %llu < %llu bytes of phased frames",
                    (unsigned long long)out->raw_out_len, (unsigned long long)need_o);
      if (need_o) std::memcpy(out->raw_out, sl->h_rawout, need_o);
    }
  }
  if (err) {
    cudaMemsetAsync(s->d_err, 0, 4, s->stream);
    return internal_device_error(err);
  }
  return FXC_OK;
}

// ---------------------------------------------------------------- helpers

fxc_status fxc_host_alloc(uint64_t bytes, void** out) {
  if (!out) return fail(FXC_EINVAL, "out is NULL");
  *out = nullptr;
  CK(cudaMallocHost(out, std::max<uint64_t>(bytes, 16)));
  return FXC_OK;
}

fxc_status fxc_host_free(void* p) {
  if (p) CK(cudaFreeHost(p));
  return FXC_OK;
}

fxc_status fxc_host_register(void* p, uint64_t bytes) {
  if (!p || !bytes) return fail(FXC_EINVAL, "fxc_host_register: NULL or empty buffer");
  const cudaError_t e = cudaHostRegister(p, bytes, cudaHostRegisterDefault);
  if (e == cudaErrorHostMemoryAlreadyRegistered) {
    cudaGetLastError();  // not sticky; the buffer is page-locked already
    return FXC_OK;
  }
  if (e != cudaSuccess) return fail(FXC_ECUDA, "cudaHostRegister: %s", cudaGetErrorString(e));
  return FXC_OK;
}

fxc_status fxc_host_unregister(void* p) {
  if (!p) return fail(FXC_EINVAL, "fxc_host_unregister: NULL buffer");
  const cudaError_t e = cudaHostUnregister(p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorHostMemoryNotRegistered ? FXC_EINVAL : FXC_ECUDA,
                "cudaHostUnregister: %s", cudaGetErrorString(e));
  }
  return FXC_OK;
}

uint64_t fxc_bytes_per_frame(uint32_t fft, uint32_t bits) {
  return ((uint64_t)fft * bits + 7) / 8;
}

fxc_status fxc_parse_shuffle(const int32_t ext[32], uint8_t internal[32]) {
  // args.rs:202-210
  if (!ext || !internal) return fail(FXC_EINVAL, "NULL argument");
  uint32_t seen = 0;
  for (int i = 0; i < 32; ++i) {
    if (ext[i] < 0 || ext[i] > 31 || ((seen >> ext[i]) & 1u))
      return fail(FXC_EINVAL, "Shuffle map must be a permutation of 0..31");
    seen |= 1u << ext[i];
  }
  for (int idx = 0; idx < 32; ++idx) internal[31 - idx] = (uint8_t)ext[idx];
  return FXC_OK;
}

fxc_status fxc_band_alignment(uint32_t fft, double fs, double c1, double c2, double bw1,
                              double bw2, int64_t out[4]) {
  // main.rs:363-372
  if (!out || fft == 0 || !(fs > 0.0)) return fail(FXC_EINVAL, "invalid argument");
  const double df = fs / (double)fft;
  const uint64_t h = fft / 2 + 1;
  const uint64_t lim = (fft % 2 == 0) ? h - 1 : h;
  const double q1 = std::floor((bw1 * 1e6) / df), q2 = std::floor((bw2 * 1e6) / df);
  uint64_t v1 = (q1 > 0.0 ? (uint64_t)q1 : 0) + 1, v2 = (q2 > 0.0 ? (uint64_t)q2 : 0) + 1;
  v1 = std::min(v1, lim);
  v2 = std::min(v2, lim);
  const double sr = (c1 * 1e6 - c2 * 1e6) / df;
  const int64_t sb = (int64_t)std::llround(sr);
  const int64_t a1s = std::max<int64_t>(0, -sb);
  const int64_t a1e = std::min<int64_t>((int64_t)v1, (int64_t)v2 - sb);
  if (a1e <= a1s) return fail(FXC_EINVAL, "No band overlap");
  out[0] = sb;
  out[1] = a1s;
  out[2] = a1e;
  out[3] = a1s + sb;
  return FXC_OK;
}

fxc_status fxc_level_power(const double* levels, uint32_t n, double* out) {
  // main.rs:378-387
  if (!levels || !out || n == 0) return fail(FXC_EINVAL, "levels are empty");
  double s = 0.0;
  for (uint32_t i = 0; i < n; ++i) s += levels[i] * levels[i];
  const double p = s / (double)n;
  if (!std::isfinite(p) || p <= 0.0) return fail(FXC_EINVAL, "mean-square level is invalid: %g", p);
  *out = p;
  return FXC_OK;
}

fxc_status fxc_normalize(uint32_t fft, uint64_t nf, double level_power, const double* acc_real,
                         const double* acc_cplx, float* out) {
  // main.rs:2645-2683
  if (!out || (!acc_real && !acc_cplx)) return fail(FXC_EINVAL, "NULL argument");
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
  return FXC_OK;
}

}  // extern "C"

// Internal helpers shared with noalloc.cu (no allocation, host only).
namespace fxc {

fxc_status internal_fail(fxc_status s, const char* msg) { return fail(s, "%s", msg); }

void internal_debug_settings(uint32_t* wait_polls, uint32_t* debug_flags) {
  *wait_polls = g_dbg_polls.load();
  *debug_flags = g_dbg_flags.load();
}

fxc_status internal_device_error(uint32_t err) {
  if (err & ERR_WAIT_TIMEOUT) return fail(FXC_ETIMEDOUT, "a bounded device-side wait gave up");
  if (err) return fail(FXC_EDEVICE, "kernel error word 0x%x", err);
  return FXC_OK;
}

int engine_sm_count(const fxc_engine* e) { return e->sm_count; }
int engine_device(const fxc_engine* e) { return e->device; }
fxc_engine* scan_engine(const fxc_scan* s) { return s->eng; }

fxc_status engine_reserve(fxc_engine* e, uint64_t bytes) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (e->in_use + bytes > e->budget)
    return fail(FXC_EBUSY, "HBM budget exhausted (%llu + %llu > %llu bytes)",
                (unsigned long long)e->in_use, (unsigned long long)bytes,
                (unsigned long long)e->budget);
  e->in_use += bytes;
  return FXC_OK;
}

void engine_release(fxc_engine* e, uint64_t bytes) {
  std::lock_guard<std::mutex> lk(e->mu);
  e->in_use -= std::min(e->in_use, bytes);
}

fxc_status batch_describe(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                          uint64_t first, double* d_acc, uint8_t* d_raw_out, BatchScan* out,
                          int* group) {
  *group = -1;
  if (!d_acc) return fail(FXC_EINVAL, "d_acc is NULL");
  fxc_status st = nf ? check_device_inputs(s, r1, r2) : FXC_OK;
  if (st != FXC_OK) return st;
  const bool corr = (s->cfg.products & (FXC_PROD_ACF | FXC_PROD_XCF)) != 0;
  const bool phased = (s->cfg.products & (FXC_PROD_PHASED | FXC_PROD_RAW)) != 0;
  if ((s->cfg.products & FXC_PROD_RAW) && nf && !d_raw_out)
    return fail(FXC_EINVAL, "the scan writes phased .raw frames but its raw output is NULL");
  if (nf == 0 || (corr && phased)) return FXC_OK;  // the per-scan path
  if (phased) {
    // phased sectors of FFT 1024..8192 run in the phased batch kernels, FFT
    // 16384 in the two-row kernel's batch group
    if (s->n > 16384) return FXC_OK;
    const PhasedParams pp = phased_params(s, r1, r2, nf, first, d_raw_out);
    if (s->n == 16384 && !phased_pair_supported(s->n, pp)) return FXC_OK;
    if ((st = grow_frame_info(s, nf)) != FXC_OK) return st;
    BatchScan b{};
    b.p = corr_params(s, r1, r2, nf, first);  // delay model and frame records
    b.p.finfo = s->d_finfo;
    b.p.partials = nullptr;
    b.pp = pp;
    b.pp.finfo = s->d_finfo;
    b.pp.partials = nullptr;  // the batch's
    b.acc = d_acc;
    b.n = s->n;
    b.h = s->h;
    b.phased = 1;
    *out = b;
    *group = s->n == 1024 ? BG_PHASED_1024 : s->n == 2048 ? BG_PHASED_2048
           : s->n == 4096 ? BG_PHASED_4096 : s->n == 8192 ? BG_PHASED_8192 : BG_PHASED_16384;
    return FXC_OK;
  }
  if (s->n > 16384) return FXC_OK;
  CorrParams p = corr_params(s, r1, r2, nf, first);
  if (s->n == 16384 && !corr_fold2_supported(p)) return FXC_OK;
  if ((st = grow_frame_info(s, nf)) != FXC_OK) return st;
  p.finfo = s->d_finfo;
  p.partials = nullptr;  // the batch's
  BatchScan b{};
  b.p = p;
  b.acc = d_acc;
  const double u1 = 1.0 / s->scale[0], u2 = 1.0 / s->scale[1];
  b.m11 = 0.25 * u1 * u1;
  b.m22 = 0.25 * u2 * u2;
  b.m12 = 0.25 * u1 * u2;
  b.n = s->n;
  b.h = s->h;
  *out = b;
  *group = s->n == 1024 ? BG_1024 : s->n == 2048 ? BG_2048 : s->n == 4096 ? BG_4096
         : s->n == 8192 ? BG_8192 : BG_16384;
  return FXC_OK;
}

fxc_status run_sector_internal(fxc_scan* s, const uint8_t* r1, const uint8_t* r2, uint64_t nf,
                               uint64_t first, double* d_acc, uint8_t* d_raw_out,
                               cudaStream_t st) {
  const fxc_status c = nf ? check_device_inputs(s, r1, r2) : FXC_OK;
  if (c != FXC_OK) return c;
  if (!d_acc) return fail(FXC_EINVAL, "d_acc is NULL");
  if ((s->cfg.products & FXC_PROD_RAW) && nf && !d_raw_out)
    return fail(FXC_EINVAL, "the scan writes phased .raw frames but its raw output is NULL");
  return run_sector_device(s, r1, r2, nf, first, d_acc, d_raw_out, st);
}

void engine_track_batch(fxc_engine* e, fxc_batch* b, bool add) {
  std::lock_guard<std::mutex> lk(e->mu);
  auto& v = e->batches;
  if (add) v.push_back(b);
  else v.erase(std::remove(v.begin(), v.end(), b), v.end());
}

void engine_track_server(fxc_engine* e, fxc_server* sv, bool add) {
  std::lock_guard<std::mutex> lk(e->mu);
  auto& v = e->servers;
  if (add) v.push_back(sv);
  else v.erase(std::remove(v.begin(), v.end(), sv), v.end());
}

fxc_status internal_prepare_tables(const fxc_scan_cfg* c, uint32_t* lut2048, float* lv512,
                                   float scale[2], int kind[2]) {
  const fxc_status st = validate_cfg(c);
  if (st != FXC_OK) return st;
  build_lut(c->shuffle1, lut2048);
  build_lut(c->shuffle2, lut2048 + 1024);
  for (int i = 0; i < 512; ++i) lv512[i] = 0.0f;
  for (uint32_t i = 0; i < c->nlevels1; ++i) lv512[i] = (float)c->levels1[i];
  for (uint32_t i = 0; i < c->nlevels2; ++i) lv512[256 + i] = (float)c->levels2[i];
  scale[0] = level_scale(c->levels1, c->nlevels1);
  scale[1] = level_scale(c->levels2, c->nlevels2);
  kind[0] = shuffle_kind(c->shuffle1);
  kind[1] = shuffle_kind(c->shuffle2);
  return FXC_OK;
}

}  // namespace fxc
