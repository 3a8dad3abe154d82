// noalloc.cu — a correlation entry point that allocates no memory.
//
// Some callers cannot call cudaMalloc at the point where they correlate: a
// real-time streaming loop must not pay cudaMalloc/cudaFree's implicit device
// synchronisation (it stalls every other stream on the GPU mid-observation),
// and a host application whose memory manager owns all device memory forbids
// allocations outside it.  fxc_sector_run_device_noalloc serves them: it runs
// the same correlation kernels as fxc_sector_run_device, but the scratch those
// kernels need (per-frame delay records, decode tables, the geometric delay
// table, per-CTA f64 partials and the error word) lives in the file-scope
// array below.  The caller still provides the inputs and the output block.
//
// The array is 24 MiB.  Every GPU that loads this library holds it until the
// process exits.  Its device address is looked up once per device, on the
// first call made with that device current.  Every call shares the array and
// it keeps the last call's contents: the kernels rewrite every partial they
// read and the error word is cleared per call, so results never depend on
// earlier calls, but calls whose work overlaps on the GPU (different streams,
// or different host threads, on one device) race on the array.
//
// A bounded device-side wait that gives up sets the array's error word; the
// call then fills its output block with NaN (a last small kernel on the same
// stream), and fxc_sector_noalloc_check reads the word back, without
// allocating, as FXC_ETIMEDOUT / FXC_EDEVICE.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "fxc.h"
#include "fxc_internal.h"
#include "fxc_kernels.h"

using namespace fxc;

namespace {

// Layout of the array (byte offsets).
constexpr size_t kRecBytes = (size_t)FXC_NOALLOC_MAX_FRAMES * sizeof(FrameInfo);  // 1.5 MiB
constexpr size_t kOffTables = kRecBytes;
constexpr size_t kOffLut = kOffTables;                                  // 2 x 1024 u32
constexpr size_t kOffLevels = kOffLut + 2048 * sizeof(uint32_t);       // 2 x 256 f32
constexpr size_t kOffGeom = kOffLevels + 512 * sizeof(float);          // geometric table
constexpr size_t kOffErr = kOffGeom + FXC_NOALLOC_MAX_GEOM * sizeof(double);
constexpr size_t kOffPartials = (kOffErr + 256 + 65535) & ~(size_t)65535;
constexpr size_t kScratchBytes = (size_t)FXC_NOALLOC_SCRATCH_MIB << 20;
static_assert(kOffPartials < kScratchBytes, "scratch layout");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[64] = {};  // device address of the array, per device ordinal

// Device address of the array on device `dev` (looked up once per device).
fxc_status scratch_base(int dev, unsigned char** base) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      char msg[256];
      snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the scratch array failed: %s",
               cudaGetErrorString(e));
      return internal_fail(FXC_ECUDA, msg);
    }
    g_scratch_addr[dev] = p;
  }
  *base = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return FXC_OK;
}

// The current device, and that `stream` (NULL: the default stream) belongs to it.
fxc_status current_device(void* stream, int* dev) {
  if (cudaGetDevice(dev) != cudaSuccess || *dev < 0 || *dev >= 64)
    return internal_fail(FXC_ECUDA, "no current CUDA device");
  if (stream) {
    int sd = -1;
    if (cudaStreamGetDevice((cudaStream_t)stream, &sd) != cudaSuccess)
      return internal_fail(FXC_EINVAL, "stream is not a valid CUDA stream");
    if (sd != *dev)
      return internal_fail(FXC_EINVAL,
                           "stream belongs to another device than the current one; make the "
                           "stream's device current before the call");
  }
  return FXC_OK;
}

// After the reduction: a call whose bounded wait gave up leaves NaN in every
// output value instead of short sums.
__global__ void noalloc_poison_kernel(const uint32_t* err, double* acc, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && *err != 0u) acc[i] = __longlong_as_double(0x7ff8000000000000ll);
}

}  // namespace

extern "C" fxc_status fxc_sector_run_device_noalloc(const fxc_scan_cfg* cfg,
                                                    const uint8_t* d_raw1, const uint8_t* d_raw2,
                                                    uint64_t nf, uint64_t first_frame,
                                                    double* d_acc, void* stream) {
  if (!cfg || !d_raw1 || !d_raw2 || !d_acc)
    return internal_fail(FXC_EINVAL, "fxc_sector_run_device_noalloc: NULL argument");
  if ((reinterpret_cast<uintptr_t>(d_raw1) | reinterpret_cast<uintptr_t>(d_raw2)) & 15u)
    return internal_fail(FXC_EINVAL, "device inputs must be 16-byte aligned");
  if (cfg->fft_len > 8192)
    return internal_fail(FXC_EUNSUPPORTED,
                         "fxc_sector_run_device_noalloc: fft_len above 8192 needs "
                         "fxc_sector_run_device (its scratch exceeds the fixed array)");
  if (cfg->products & (FXC_PROD_PHASED | FXC_PROD_RAW))
    return internal_fail(FXC_EUNSUPPORTED,
                         "fxc_sector_run_device_noalloc computes ACF/XCF products only");
  if (nf > FXC_NOALLOC_MAX_FRAMES)
    return internal_fail(FXC_EINVAL,
                         "fxc_sector_run_device_noalloc: nf exceeds FXC_NOALLOC_MAX_FRAMES "
                         "(32768); split the sector into several calls and add the results");
  if (cfg->delay.geom_table && cfg->delay.geom_len > FXC_NOALLOC_MAX_GEOM)
    return internal_fail(FXC_EINVAL,
                         "fxc_sector_run_device_noalloc: geometric delay table longer than "
                         "FXC_NOALLOC_MAX_GEOM (4096) entries");
  uint32_t lut[2048];
  float lv[512];
  float scale[2];
  int kind[2];
  fxc_status st = internal_prepare_tables(cfg, lut, lv, scale, kind);
  if (st != FXC_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t n = cfg->fft_len, h = n / 2 + 1;
  if (nf == 0) {
    if (cudaMemsetAsync(d_acc, 0, sizeof(double) * 5 * h, s) != cudaSuccess)
      return internal_fail(FXC_ECUDA, "cudaMemsetAsync failed");
    return FXC_OK;
  }

  int dev = 0;
  st = current_device(stream, &dev);
  if (st != FXC_OK) return st;
  unsigned char* base = nullptr;
  st = scratch_base(dev, &base);
  if (st != FXC_OK) return st;
  FrameInfo* rec = reinterpret_cast<FrameInfo*>(base);
  uint32_t* d_lut = reinterpret_cast<uint32_t*>(base + kOffLut);
  float* d_lv = reinterpret_cast<float*>(base + kOffLevels);
  double* d_geom = reinterpret_cast<double*>(base + kOffGeom);
  uint32_t* d_err = reinterpret_cast<uint32_t*>(base + kOffErr);
  double* part = reinterpret_cast<double*>(base + kOffPartials);

#define NA_CK(call)                                                              \
  do {                                                                           \
    const cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) return internal_fail(FXC_ECUDA, cudaGetErrorString(e_)); \
  } while (0)
  // tables from host memory into the array (pageable copies: no allocation)
  NA_CK(cudaMemcpyAsync(d_lut, lut, sizeof lut, cudaMemcpyHostToDevice, s));
  NA_CK(cudaMemcpyAsync(d_lv, lv, sizeof lv, cudaMemcpyHostToDevice, s));
  if (cfg->delay.geom_table)
    NA_CK(cudaMemcpyAsync(d_geom, cfg->delay.geom_table, cfg->delay.geom_len * sizeof(double),
                          cudaMemcpyHostToDevice, s));
  NA_CK(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), s));

  const fxc_delay_cfg& c = cfg->delay;
  DelayParams dl;
  dl.frame_dt = c.frame_dt;
  dl.fs = c.fs;
  dl.time_offset_s = c.time_offset_s;
  dl.table = c.geom_table ? d_geom : nullptr;
  dl.table_len = c.geom_table ? c.geom_len : 0;
  dl.coarse = c.coarse_delay_s;
  dl.user_samples = c.delay_user_samples;
  dl.extra_rate = c.extra_delay_rate_sps;
  dl.c1d = c.clock1_delay_s;
  dl.c1r = c.clock1_rate_sps;
  dl.c2d = c.clock2_delay_s;
  dl.c2r = c.clock2_rate_sps;
  dl.d_seek = c.d_seek;
  dl.d1 = c.net_d1_base;
  dl.r1 = c.total_rate1_base;
  dl.a1 = c.total_accel1_base;
  dl.d2 = c.net_d2_base;
  dl.r2 = c.total_rate2_base;
  dl.a2 = c.total_accel2_base;
  dl.lo1 = c.lo1_hz;
  dl.lo2 = c.lo2_hz;
  const double df = cfg->fs_hz / (double)n;
  NA_CK(launch_frame_info(dl, first_frame, nf, (int)n, df, (int)cfg->a1s, (int)cfg->a2s, rec, s));
  if (!(cfg->products & (FXC_PROD_ACF | FXC_PROD_XCF))) {
    NA_CK(cudaMemsetAsync(d_acc, 0, sizeof(double) * 5 * h, s));
    return FXC_OK;
  }

  CorrParams p{};
  const uint8_t* raw[2] = {d_raw1, d_raw2};
  for (int k = 0; k < 2; ++k) {
    p.st[k].raw = raw[k];
    p.st[k].shlut = d_lut + 1024 * k;
    p.st[k].levels = d_lv + 256 * k;
    p.st[k].bits = (int)(k ? cfg->bits2 : cfg->bits1);
    p.st[k].bpf = (uint32_t)fxc_bytes_per_frame(n, (uint32_t)p.st[k].bits);
    p.st[k].lsb = k ? cfg->lsb2 : cfg->lsb1;
    p.st[k].shkind = kind[k];
    p.st[k].scale = scale[k];
    std::memcpy(p.st[k].perm, k ? cfg->shuffle2 : cfg->shuffle1, 32);
  }
  p.dl = dl;
  p.nf = nf;
  p.first_frame = first_frame;
  p.a1s = (int32_t)cfg->a1s;
  p.a1e = (int32_t)cfg->a1e;
  p.a2s = (int32_t)cfg->a2s;
  p.grid = cfg->grid;
  p.products = cfg->products;
  const int fpc = corr_frames_per_cta_iter(n);
  p.stage_bytes = (uint32_t)fpc * (p.st[0].bpf + p.st[1].bpf);
  p.flush_every = (uint32_t)std::max(1, 32 / fpc);
  p.df_hz = df;
  p.partials = part;
  p.finfo = rec;
  p.err = d_err;
  internal_debug_settings(&p.wait_polls, &p.debug_flags);
  int sms = 0;
  NA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint64_t iters = (nf + fpc - 1) / fpc;
  const uint64_t fit = (kScratchBytes - kOffPartials) / (4ull * h * sizeof(double));
  const uint64_t grid = std::max<uint64_t>(
      1, std::min<uint64_t>({iters, (uint64_t)sms * corr_ctas_per_sm(n), fit}));
  NA_CK(launch_corr(n, MODE_CORR, p, (int)grid, s));
  const double u1 = 1.0 / scale[0], u2 = 1.0 / scale[1];
  NA_CK(launch_reduce(part, (int)grid, (int)h, 0.25 * u1 * u1, 0.25 * u2 * u2, 0.25 * u1 * u2,
                      d_acc, s));
  noalloc_poison_kernel<<<(5 * h + 255) / 256, 256, 0, s>>>(d_err, d_acc, 5 * h);
  NA_CK(cudaGetLastError());
#undef NA_CK
  return FXC_OK;
}

extern "C" fxc_status fxc_sector_noalloc_check(void* stream) {
  int dev = 0;
  fxc_status st = current_device(stream, &dev);
  if (st != FXC_OK) return st;
  unsigned char* base = nullptr;
  st = scratch_base(dev, &base);
  if (st != FXC_OK) return st;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  uint32_t err = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&err, base + kOffErr, sizeof err, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return internal_fail(FXC_ECUDA, cudaGetErrorString(e));
  return internal_device_error(err);
}
