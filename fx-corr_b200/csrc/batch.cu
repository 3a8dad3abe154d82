// batch.cu — batched sectors of many scans (include/fxc.h, fxc_batch_*).
//
// A call describes each scan's sector (BatchScan: the scan's tables, frame
// record buffer, raw words and output; correlation or phased products),
// splits every sector into work items
// of `item_frames` frames (at most one per persistent CTA), uploads the
// tables in one copy and runs
//   batch_frame_info_kernel  the FP64 delay records of every frame,
//   one persistent kernel per FFT length present (tickets over its items),
//   batch_reduce_kernel      every sector's partials in item order,
// either launched directly or as a CUDA graph captured once per set of FFT
// lengths (the kernels read every count from the uploaded header, so one
// graph serves every batch of that set).  The autotuner times each kernel
// variant (frames per CTA iteration) and item size on a synthetic batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "fxc.h"
#include "fxc_internal.h"
#include "fxc_kernels.h"

using namespace fxc;

namespace {

#define BCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      char m_[256];                                                                        \
      snprintf(m_, sizeof m_, "%s: %s", #call, cudaGetErrorString(e_));                    \
      return internal_fail(e_ == cudaErrorMemoryAllocation ? FXC_ENOMEM : FXC_ECUDA, m_); \
    }                                                                                      \
  } while (0)

constexpr uint32_t kGroupN[kBatchGroups] = {1024, 2048, 4096, 8192, 16384,
                                            1024, 2048, 4096, 8192, 16384};
// kernel variants (frame pairs per CTA iteration) of each group; the phased
// groups have one variant each (the single-scan phased kernel's)
const std::vector<int> kGroupFpc[kBatchGroups] = {{1, 2, 4}, {1, 2, 4}, {1, 2}, {1}, {1},
                                                  {4}, {2}, {1}, {1}, {1}};
// single-scan defaults: the frames per iteration of corr_kernel / phased_kernel
constexpr int kDefaultFpc[kBatchGroups] = {4, 2, 1, 1, 1, 4, 2, 1, 1, 1};

bool phased_group(int g) { return g >= kCorrGroups; }
// Default frames per item (the tuner replaces a correlation group's).  Items
// of the FFT-16384 phased group take ~0.8 ms at 32 frames: larger ones leave
// SMs idle for up to an item's time after the last tickets of a call.
constexpr uint32_t kDefaultItems[kBatchGroups] = {128, 128, 128, 128, 128, 128, 128, 128, 128, 32};
const uint32_t kItemCandidates[] = {32, 64, 128, 256, 512};

// The correlation group of FFT length n (-1: none).
int group_of(uint32_t n) {
  for (int g = 0; g < kCorrGroups; ++g)
    if (kGroupN[g] == n) return g;
  return -1;
}

uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

struct Shape {
  int fpc = 1;
  uint32_t item_frames = 128;
  int ctas = 0;  // resident CTAs per SM of the variant
  double gsps = 0.0;
  bool tuned = false;
};

}  // namespace

struct fxc_batch {
  fxc_engine* eng = nullptr;
  int device = 0, sms = 0;
  bool graphs = false, autotune = false;
  uint32_t item_override = 0;
  Shape shape[kBatchGroups];
  bool tuning[kBatchGroups] = {};  // the tuner's own batches run untuned
  bool prepared[kBatchGroups][5] = {};
  // two device arenas [header][scans][items], each mirroring its pinned
  // staging, used by alternate calls: a call need not wait for the previous
  // call's upload (queued behind that call's inputs) before staging its own
  struct Arena {
    uint8_t* d = nullptr;
    uint64_t cap = 0;
    uint8_t* h = nullptr;
    uint64_t hcap = 0;
    cudaEvent_t staged = nullptr;  // this staging's last upload has been read
  } arena[2];
  int next_arena = 0;
  double* d_part = nullptr;
  uint64_t part_cap = 0;  // doubles
  uint64_t charged = 0;
  cudaEvent_t ev_done = nullptr;    // the last call's device work
  cudaStream_t cap_stream = nullptr;
  std::map<uint64_t, cudaGraphExec_t> execs;  // by group set and variants
  std::mutex mu;
  uint64_t launches = 0;
};

namespace {

struct DeviceGuardB {
  int prev = -1;
  explicit DeviceGuardB(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuardB() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

void drop_graphs(fxc_batch* b) {
  if (b->execs.empty()) return;
  cudaEventSynchronize(b->ev_done);  // no replay of them in flight
  for (auto& kv : b->execs) cudaGraphExecDestroy(kv.second);
  b->execs.clear();
}

fxc_status prepare_variant(fxc_batch* b, int g, int fpc) {
  if (!b->prepared[g][fpc]) {
    if (phased_group(g)) BCK(phased_batch_prepare(kGroupN[g]));
    else BCK(batch_prepare(g, fpc));
    b->prepared[g][fpc] = true;
  }
  return FXC_OK;
}

fxc_status set_shape(fxc_batch* b, int g, int fpc, uint32_t item_frames) {
  fxc_status st = prepare_variant(b, g, fpc);
  if (st != FXC_OK) return st;
  const int ctas = phased_group(g) ? phased_batch_ctas_per_sm(kGroupN[g])
                                   : batch_group_ctas_per_sm(g, fpc);
  if (ctas <= 0) return internal_fail(FXC_ECUDA, "batch kernel variant does not fit an SM");
  if (b->shape[g].fpc != fpc || b->shape[g].ctas != ctas) drop_graphs(b);
  b->shape[g].fpc = fpc;
  b->shape[g].item_frames = item_frames;
  b->shape[g].ctas = ctas;
  return FXC_OK;
}

// Grows the device arena / partials (waiting for the previous call's work,
// whose graphs point at the old buffers) and the pinned staging.
fxc_status grow(fxc_batch* b, fxc_batch::Arena& A, uint64_t arena_bytes, uint64_t part_elems) {
  if (arena_bytes > A.cap || part_elems > b->part_cap) {
    BCK(cudaEventSynchronize(b->ev_done));
    drop_graphs(b);
  }
  if (arena_bytes > A.cap) {
    const uint64_t want = std::max<uint64_t>(arena_bytes, 2 * A.cap);
    fxc_status st = engine_reserve(b->eng, want);
    if (st != FXC_OK) return st;
    cudaFree(A.d);
    engine_release(b->eng, A.cap);
    b->charged -= std::min(b->charged, A.cap);
    A.d = nullptr;
    A.cap = 0;
    const cudaError_t e = cudaMalloc(&A.d, want);
    if (e != cudaSuccess) {
      engine_release(b->eng, want);
      BCK(e);
    }
    A.cap = want;
    b->charged += want;
  }
  if (part_elems > b->part_cap) {
    const uint64_t want = std::max<uint64_t>(part_elems, b->part_cap + b->part_cap / 2);
    fxc_status st = engine_reserve(b->eng, want * 8);
    if (st != FXC_OK) return st;
    cudaFree(b->d_part);
    engine_release(b->eng, b->part_cap * 8);
    b->charged -= std::min(b->charged, b->part_cap * 8);
    b->d_part = nullptr;
    b->part_cap = 0;
    const cudaError_t e = cudaMalloc(&b->d_part, want * 8);
    if (e != cudaSuccess) {
      engine_release(b->eng, want * 8);
      BCK(e);
    }
    b->part_cap = want;
    b->charged += want * 8;
  }
  if (arena_bytes > A.hcap) {
    BCK(cudaEventSynchronize(A.staged));
    if (A.h) cudaFreeHost(A.h);
    A.h = nullptr;
    A.hcap = 0;
    BCK(cudaMallocHost(&A.h, A.cap));
    A.hcap = A.cap;
  }
  return FXC_OK;
}

struct Entry {
  uint32_t idx;  // position in the caller's arrays
  int group;
  BatchScan bs;
};

// Frames per item of a sector: the group's item size, enlarged so that a
// sector has at most one item per resident CTA, rounded to whole CTA iterations.
uint64_t item_len(const Shape& sh, int sms, uint64_t nf) {
  const uint64_t maxn = (uint64_t)std::max(1, sms * sh.ctas);
  uint64_t per = sh.item_frames;
  if ((nf + per - 1) / per > maxn) per = (nf + maxn - 1) / maxn;
  return align_up(per, (uint64_t)sh.fpc);
}

fxc_status run_batch(fxc_batch* b, fxc_scan* const* scans, const uint8_t* const* r1,
                     const uint8_t* const* r2, const uint64_t* nf, const uint64_t* first,
                     double* const* acc, uint8_t* const* raw_out, uint32_t count,
                     cudaStream_t stream, bool allow_graph);

// Times every variant x item size of group g on a synthetic batch and keeps
// the fastest.  The caller holds b->mu.
fxc_status autotune_locked(fxc_batch* b, int g) {
  if (b->tuning[g]) return FXC_OK;
  struct Flag {
    bool& f;
    explicit Flag(bool& x) : f(x) { f = true; }
    ~Flag() { f = false; }
  } flag(b->tuning[g]);
  const Shape saved = b->shape[g];
  const uint32_t fft_len = kGroupN[g];
  // synthetic batch: 16 scans of 2-bit stations, 2^25 samples per sector each
  // (a few items per CTA, as in a serving batch)
  constexpr int kScans = 16;
  const uint64_t frames = (1ull << 25) / fft_len;
  const uint64_t bpf = fxc_bytes_per_frame(fft_len, 2);
  const double fs = 1024e6;
  fxc_scan_cfg cfg{};
  cfg.fft_len = fft_len;
  cfg.bits1 = cfg.bits2 = cfg.bits_out = 2;
  cfg.fs_hz = fs;
  const double lv[4] = {-3.0, -1.0, 1.0, 3.0};
  for (int i = 0; i < 4; ++i) cfg.levels1[i] = cfg.levels2[i] = lv[i];
  cfg.nlevels1 = cfg.nlevels2 = 4;
  for (int i = 0; i < 32; ++i) cfg.shuffle1[i] = cfg.shuffle2[i] = (uint8_t)i;
  cfg.a1s = 0;
  cfg.a1e = fft_len / 2;
  cfg.a2s = 0;
  cfg.products = FXC_PROD_ACF | FXC_PROD_XCF;
  cfg.w1 = cfg.w2 = 1.0;
  cfg.delay.frame_dt = fft_len / fs;
  cfg.delay.fs = fs;
  cfg.delay.net_d1_base = 3.1e-7;
  cfg.delay.total_rate1_base = 2e-9;
  cfg.delay.lo1_hz = cfg.delay.lo2_hz = 8.4e9;
  std::vector<fxc_scan*> scans(kScans, nullptr);
  uint8_t* d_raw = nullptr;
  double* d_acc = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  fxc_status result = FXC_OK;
  const uint64_t raw_bytes = (uint64_t)kScans * 2 * frames * bpf;
  const uint64_t h = fft_len / 2 + 1;
  auto cleanup = [&]() {
    if (st) cudaStreamSynchronize(st);
    for (fxc_scan* s : scans) fxc_scan_close(s);
    cudaFree(d_raw);
    cudaFree(d_acc);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
  };
  do {
    for (auto& s : scans)
      if ((result = fxc_scan_open(b->eng, &cfg, &s)) != FXC_OK) break;
    if (result != FXC_OK) break;
    if (cudaMalloc(&d_raw, raw_bytes) != cudaSuccess ||
        cudaMalloc(&d_acc, (size_t)kScans * 5 * h * 8) != cudaSuccess ||
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      result = internal_fail(FXC_ENOMEM, "autotune: device allocation failed");
      break;
    }
    {
      std::vector<uint8_t> hr(raw_bytes);
      std::mt19937_64 rng(0x5eed + fft_len);
      for (uint64_t i = 0; i < raw_bytes; i += 8) {
        const uint64_t v = rng();
        std::memcpy(hr.data() + i, &v, std::min<uint64_t>(8, raw_bytes - i));
      }
      if (cudaMemcpy(d_raw, hr.data(), raw_bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
        result = internal_fail(FXC_ECUDA, "autotune: upload failed");
        break;
      }
    }
    std::vector<const uint8_t*> r1(kScans), r2(kScans);
    std::vector<uint64_t> nfs(kScans, frames), firsts(kScans);
    std::vector<double*> accs(kScans);
    for (int k = 0; k < kScans; ++k) {
      r1[k] = d_raw + (uint64_t)(2 * k) * frames * bpf;
      r2[k] = d_raw + (uint64_t)(2 * k + 1) * frames * bpf;
      firsts[k] = (uint64_t)k * frames;
      accs[k] = d_acc + (uint64_t)k * 5 * h;
    }
    Shape best;
    double best_ms = 1e30;
    std::vector<uint32_t> items;
    if (b->item_override) items.push_back(b->item_override);
    else items.assign(std::begin(kItemCandidates), std::end(kItemCandidates));
    for (int fpc : kGroupFpc[g]) {
      for (uint32_t itf : items) {
        if ((result = set_shape(b, g, fpc, itf)) != FXC_OK) break;
        float best_c = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {
          if (cudaEventRecord(e0, st) != cudaSuccess) break;
          result = run_batch(b, scans.data(), r1.data(), r2.data(), nfs.data(), firsts.data(),
                             accs.data(), nullptr, kScans, st, false);
          if (result != FXC_OK) break;
          float ms = 0.f;
          if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
              cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            result = internal_fail(FXC_ECUDA, "autotune: timing failed");
            break;
          }
          if (rep > 0) best_c = std::min(best_c, ms);  // the first run warms up
        }
        if (result != FXC_OK) break;
        if (best_c < best_ms) {
          best_ms = best_c;
          best = b->shape[g];
        }
      }
      if (result != FXC_OK) break;
    }
    if (result != FXC_OK) break;
    result = set_shape(b, g, best.fpc, best.item_frames);
    b->shape[g].tuned = true;
    b->shape[g].gsps = (double)kScans * frames * 2.0 * fft_len / (best_ms * 1e-3) / 1e9;
  } while (false);
  cleanup();
  if (result != FXC_OK) {
    // keep the shape the length had before (the candidates may have replaced it)
    const std::string msg = fxc_last_error();
    if (set_shape(b, g, saved.fpc, saved.item_frames) == FXC_OK) {
      b->shape[g].tuned = saved.tuned;
      b->shape[g].gsps = saved.gsps;
    }
    internal_fail(result, msg.c_str());
  }
  return result;
}

fxc_status run_batch(fxc_batch* b, fxc_scan* const* scans, const uint8_t* const* r1,
                     const uint8_t* const* r2, const uint64_t* nf, const uint64_t* first,
                     double* const* acc, uint8_t* const* raw_out, uint32_t count,
                     cudaStream_t stream, bool allow_graph) {
  std::vector<Entry> ents;
  std::vector<uint32_t> others;
  ents.reserve(count);
  {
    std::vector<const fxc_scan*> seen(scans, scans + count);
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end())
      return internal_fail(FXC_EINVAL, "a scan appears twice in one batch");
  }
  for (uint32_t i = 0; i < count; ++i) {
    if (!scans[i]) return internal_fail(FXC_EINVAL, "scan is NULL");
    if (scan_engine(scans[i]) != b->eng)
      return internal_fail(FXC_EINVAL, "scan belongs to another engine");
    Entry e{};
    e.idx = i;
    fxc_status st = batch_describe(scans[i], r1[i], r2[i], nf[i], first[i], acc[i],
                                   raw_out ? raw_out[i] : nullptr, &e.bs, &e.group);
    if (st != FXC_OK) return st;
    if (e.group < 0) others.push_back(i);
    else ents.push_back(e);
  }
  // tuning and variants of the groups present
  uint32_t mask = 0;
  for (const Entry& e : ents) mask |= 1u << e.group;
  for (int g = 0; g < kBatchGroups; ++g) {
    if (!(mask & (1u << g))) continue;
    if (phased_group(g)) b->shape[g].tuned = true;  // one variant, default item size
    if (b->autotune && !b->shape[g].tuned && !b->tuning[g]) {
      // first use: tune; if the tuner cannot run (e.g. no HBM for its
      // synthetic batch) the length keeps its default shape
      if (autotune_locked(b, g) != FXC_OK) {
        b->shape[g].tuned = true;
        b->shape[g].gsps = 0.0;
      }
    }
    if (b->shape[g].ctas == 0) {
      fxc_status st = set_shape(b, g, b->shape[g].fpc, b->shape[g].item_frames);
      if (st != FXC_OK) return st;
    }
  }
  // table order: by group, then call order; items follow the same order
  std::stable_sort(ents.begin(), ents.end(),
                   [](const Entry& a, const Entry& c) { return a.group < c.group; });
  BatchHeader hdr{};
  hdr.nscans = (uint32_t)ents.size();
  std::vector<BatchItem> items;
  uint64_t fi = 0, bins = 0, part = 0;
  for (int g = 0; g < kBatchGroups; ++g) {
    hdr.item0[g] = (uint32_t)items.size();
    for (Entry& e : ents) {
      if (e.group != g) continue;
      const Shape& sh = b->shape[g];
      const uint64_t n = e.bs.p.nf;
      const uint64_t per = item_len(sh, b->sms, n);
      const uint32_t nparts = (uint32_t)((n + per - 1) / per);
      const uint64_t h = e.bs.h;
      const uint64_t slot = phased_group(g) ? h : 4 * h;  // partial doubles per item
      e.bs.part = part;
      e.bs.nparts = nparts;
      e.bs.fi0 = fi;
      e.bs.bin0 = bins;
      const uint32_t si = (uint32_t)(&e - ents.data());
      for (uint32_t k = 0; k < nparts; ++k) {
        const uint64_t f0 = k * per, f1 = std::min(n, f0 + per);
        for (uint32_t row = 0; row < (g == BG_16384 ? 2u : 1u); ++row)
          items.push_back(BatchItem{si, row, f0, f1, part + (uint64_t)k * slot});
      }
      part += (uint64_t)nparts * slot;
      fi += n;
      bins += h;
    }
    hdr.nitems[g] = (uint32_t)items.size() - hdr.item0[g];
  }
  hdr.nframes = fi;
  hdr.nbins = bins;

  BCK(cudaStreamWaitEvent(stream, b->ev_done, 0));
  if (!ents.empty()) {
    const uint64_t off_scans = align_up(sizeof(BatchHeader), 256);
    const uint64_t off_items = off_scans + align_up(ents.size() * sizeof(BatchScan), 256);
    const uint64_t bytes = off_items + items.size() * sizeof(BatchItem);
    const int ai = b->next_arena;
    b->next_arena ^= 1;
    fxc_batch::Arena& A = b->arena[ai];
    fxc_status st = grow(b, A, bytes, std::max<uint64_t>(part, 1));
    if (st != FXC_OK) return st;
    BCK(cudaEventSynchronize(A.staged));  // the call before the previous one
    hdr.scans = reinterpret_cast<const BatchScan*>(A.d + off_scans);
    hdr.items = reinterpret_cast<const BatchItem*>(A.d + off_items);
    std::memcpy(A.h, &hdr, sizeof hdr);
    for (size_t k = 0; k < ents.size(); ++k)
      std::memcpy(A.h + off_scans + k * sizeof(BatchScan), &ents[k].bs, sizeof(BatchScan));
    std::memcpy(A.h + off_items, items.data(), items.size() * sizeof(BatchItem));
    BCK(cudaMemcpyAsync(A.d, A.h, bytes, cudaMemcpyHostToDevice, stream));
    BCK(cudaEventRecord(A.staged, stream));

    BatchArgs a;
    a.hdr = reinterpret_cast<BatchHeader*>(A.d);
    a.partials = b->d_part;
    // the graph's kernels take the header and partials addresses as
    // arguments: graphs are dropped whenever either moves (grow)
    uint64_t key = mask;  // kBatchGroups bits
    for (int g = 0; g < kCorrGroups; ++g) key |= (uint64_t)b->shape[g].fpc << (16 + 4 * g);
    key |= (uint64_t)ai << 40;
    const int grid_aux = b->sms * 8;
    auto enqueue = [&](cudaStream_t s, bool full) -> fxc_status {
      const uint64_t fgrid = full ? (uint64_t)grid_aux
                                  : std::min<uint64_t>((uint64_t)grid_aux, (hdr.nframes + 127) / 128);
      BCK(launch_batch_frame_info(a, (int)std::max<uint64_t>(fgrid, 1), s));
      for (int g = 0; g < kBatchGroups; ++g) {
        if (!(mask & (1u << g))) continue;
        const Shape& sh = b->shape[g];
        uint64_t grid = (uint64_t)b->sms * sh.ctas;
        if (!full) grid = std::min<uint64_t>(grid, hdr.nitems[g]);
        if (phased_group(g))
          BCK(launch_phased_batch(kGroupN[g], a, g, (int)std::max<uint64_t>(grid, 1), s));
        else
          BCK(launch_batch_group(g, sh.fpc, a, (int)std::max<uint64_t>(grid, 1), s));
      }
      const uint64_t rgrid = full ? (uint64_t)grid_aux
                                  : std::min<uint64_t>((uint64_t)grid_aux, (hdr.nbins + 255) / 256);
      BCK(launch_batch_reduce(a, (int)std::max<uint64_t>(rgrid, 1), s));
      return FXC_OK;
    };
    const uint64_t kernels = 2 + (uint64_t)__builtin_popcount(mask);
    if (b->graphs && allow_graph) {
      auto it = b->execs.find(key);
      if (it == b->execs.end()) {
        BCK(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
        const fxc_status cst = enqueue(b->cap_stream, true);
        cudaGraph_t graph = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(b->cap_stream, &graph);
        if (cst != FXC_OK) {
          if (graph) cudaGraphDestroy(graph);
          return cst;
        }
        BCK(ee);
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        BCK(ie);
        it = b->execs.emplace(key, exec).first;
      }
      BCK(cudaGraphLaunch(it->second, stream));
    } else {
      st = enqueue(stream, false);
      if (st != FXC_OK) return st;
    }
    b->launches += kernels;
  }
  for (uint32_t i : others) {
    fxc_status st = run_sector_internal(scans[i], r1[i], r2[i], nf[i], first[i], acc[i],
                                        raw_out ? raw_out[i] : nullptr, stream);
    if (st != FXC_OK) return st;
  }
  BCK(cudaEventRecord(b->ev_done, stream));
  return FXC_OK;
}

}  // namespace

namespace fxc {

void batch_release(fxc_batch* b) {
  if (!b) return;
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuardB dg(b->device);
  cudaEventSynchronize(b->ev_done);
  drop_graphs(b);
  for (auto& A : b->arena) {
    if (A.staged) cudaEventSynchronize(A.staged);
    cudaFree(A.d);
    if (A.h) cudaFreeHost(A.h);
    A.d = nullptr;
    A.h = nullptr;
    A.cap = 0;
    A.hcap = 0;
  }
  cudaFree(b->d_part);
  b->d_part = nullptr;
  b->part_cap = 0;
  engine_release(b->eng, b->charged);
  b->charged = 0;
}

}  // namespace fxc

extern "C" {

fxc_status fxc_batch_create(fxc_engine* e, const fxc_batch_opts* opts, fxc_batch** out) {
  if (!e || !out) return internal_fail(FXC_EINVAL, "NULL argument");
  *out = nullptr;
  auto* b = new fxc_batch();
  b->eng = e;
  b->device = engine_device(e);
  b->sms = engine_sm_count(e);
  b->graphs = opts && opts->use_graphs;
  b->autotune = opts && opts->autotune;
  b->item_override = opts ? opts->item_frames : 0;
  for (int g = 0; g < kBatchGroups; ++g) {
    b->shape[g].fpc = kDefaultFpc[g];
    b->shape[g].item_frames = b->item_override ? b->item_override : kDefaultItems[g];
  }
  DeviceGuardB dg(b->device);
  auto bail = [&](cudaError_t err) {
    fxc_batch_destroy(b);
    char m[256];
    snprintf(m, sizeof m, "fxc_batch_create: %s", cudaGetErrorString(err));
    return internal_fail(FXC_ECUDA, m);
  };
  cudaError_t err;
  if ((err = cudaEventCreateWithFlags(&b->arena[0].staged, cudaEventDisableTiming)) != cudaSuccess ||
      (err = cudaEventCreateWithFlags(&b->arena[1].staged, cudaEventDisableTiming)) != cudaSuccess ||
      (err = cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming)) != cudaSuccess ||
      (err = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(err);
  engine_track_batch(e, b, true);
  *out = b;
  return FXC_OK;
}

fxc_status fxc_batch_destroy(fxc_batch* b) {
  if (!b) return FXC_OK;
  engine_track_batch(b->eng, b, false);
  DeviceGuardB dg(b->device);
  if (b->ev_done) cudaEventSynchronize(b->ev_done);
  drop_graphs(b);
  for (auto& A : b->arena) {
    cudaFree(A.d);
    if (A.h) cudaFreeHost(A.h);
    if (A.staged) cudaEventDestroy(A.staged);
  }
  cudaFree(b->d_part);
  engine_release(b->eng, b->charged);
  if (b->ev_done) cudaEventDestroy(b->ev_done);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  delete b;
  return FXC_OK;
}

fxc_status fxc_batch_run_device(fxc_batch* b, fxc_scan* const* scans, const uint8_t* const* d_raw1,
                                const uint8_t* const* d_raw2, const uint64_t* nf,
                                const uint64_t* first_frame, double* const* d_acc, uint32_t count,
                                void* stream) {
  if (!b) return internal_fail(FXC_EINVAL, "batch is NULL");
  if (count == 0) return FXC_OK;
  if (!scans || !d_raw1 || !d_raw2 || !nf || !first_frame || !d_acc)
    return internal_fail(FXC_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuardB dg(b->device);
  return run_batch(b, scans, d_raw1, d_raw2, nf, first_frame, d_acc, nullptr, count,
                   (cudaStream_t)stream, true);
}

fxc_status fxc_batch_run_device_raw(fxc_batch* b, fxc_scan* const* scans,
                                    const uint8_t* const* d_raw1, const uint8_t* const* d_raw2,
                                    const uint64_t* nf, const uint64_t* first_frame,
                                    double* const* d_acc, uint8_t* const* d_raw_out,
                                    uint32_t count, void* stream) {
  if (!b) return internal_fail(FXC_EINVAL, "batch is NULL");
  if (count == 0) return FXC_OK;
  if (!scans || !d_raw1 || !d_raw2 || !nf || !first_frame || !d_acc || !d_raw_out)
    return internal_fail(FXC_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuardB dg(b->device);
  return run_batch(b, scans, d_raw1, d_raw2, nf, first_frame, d_acc, d_raw_out, count,
                   (cudaStream_t)stream, true);
}

fxc_status fxc_batch_shape(fxc_batch* b, uint32_t fft_len, int32_t* fpc, uint32_t* item_frames,
                           int32_t* ctas_per_sm, double* gsps) {
  if (!b) return internal_fail(FXC_EINVAL, "batch is NULL");
  const int g = group_of(fft_len);
  if (g < 0) return internal_fail(FXC_EUNSUPPORTED, "batches take FFT lengths 1024..16384");
  std::lock_guard<std::mutex> lk(b->mu);
  if (b->shape[g].ctas == 0) {
    DeviceGuardB dg(b->device);
    fxc_status st = set_shape(b, g, b->shape[g].fpc, b->shape[g].item_frames);
    if (st != FXC_OK) return st;
  }
  if (fpc) *fpc = b->shape[g].fpc;
  if (item_frames) *item_frames = b->shape[g].item_frames;
  if (ctas_per_sm) *ctas_per_sm = b->shape[g].ctas;
  if (gsps) *gsps = b->shape[g].tuned ? b->shape[g].gsps : 0.0;
  return FXC_OK;
}

fxc_status fxc_batch_autotune(fxc_batch* b, uint32_t fft_len) {
  if (!b) return internal_fail(FXC_EINVAL, "batch is NULL");
  const int g = group_of(fft_len);
  if (g < 0) return internal_fail(FXC_EUNSUPPORTED, "batches take FFT lengths 1024..16384");
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuardB dg(b->device);
  return autotune_locked(b, g);
}

fxc_status fxc_batch_set_shape(fxc_batch* b, uint32_t fft_len, int32_t fpc,
                               uint32_t item_frames) {
  if (!b) return internal_fail(FXC_EINVAL, "batch is NULL");
  const int g = group_of(fft_len);
  if (g < 0) return internal_fail(FXC_EUNSUPPORTED, "batches take FFT lengths 1024..16384");
  const auto& v = kGroupFpc[g];
  if (std::find(v.begin(), v.end(), (int)fpc) == v.end())
    return internal_fail(FXC_EINVAL, "no kernel variant with that many frames per iteration");
  if (item_frames == 0 || item_frames % 32 != 0)
    return internal_fail(FXC_EINVAL, "item_frames must be a positive multiple of 32");
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuardB dg(b->device);
  fxc_status st = set_shape(b, g, fpc, item_frames);
  if (st != FXC_OK) return st;
  b->shape[g].tuned = true;  // pinned: the first-use tuner leaves it
  b->shape[g].gsps = 0.0;
  return FXC_OK;
}

uint64_t fxc_batch_launches(fxc_batch* b) { return b ? b->launches : 0; }

}  // extern "C"
