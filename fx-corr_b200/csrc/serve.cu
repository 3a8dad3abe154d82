// serve.cu — the serving loop: continuous batching of correlation jobs over
// a fixed set of device contexts (include/fxc.h, fxc_server_*).
//
// Each slot is a worker thread that owns one scan (streams, partials, frame
// records, sector staging buffers, tables).  A worker takes the oldest queued
// job, rebinds its scan to the job's configuration (scan_bind reuses the
// buffers and grows them within the engine's HBM budget), and streams the
// job's sectors through fxc_sector_submit / fxc_sector_wait with the engine's
// sectors-in-flight depth: host-to-device copies on the scan's copy stream
// overlap the previous sector's kernels, and the slots' streams overlap each
// other on the device.  A job whose buffers do not fit the budget waits for
// another job to finish, and fails with FXC_EBUSY only when no other job is
// running to free memory.
//
// Batched mode (opts.batch): a worker only stages its sectors (host-to-device
// copies into its scan's sector slots) and posts them; one dispatcher thread
// takes every posted sector (one per scan) and computes them together with one
// fxc_batch_run_device call on its own stream, keeping at most two batches in
// flight so that the next batch gathers the sectors posted meanwhile; each
// worker then queues its sector's device-to-host copies behind that batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fxc.h"
#include "fxc_internal.h"

namespace {

uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Job {
  uint64_t id = 0;
  fxc_scan_cfg cfg{};
  std::vector<double> table;  // the geometric table, copied at submit
  fxc_job job{};
  fxc_job_stats stats{};
  std::string error;
  bool done = false;
};

// A staged sector waiting for, or computed by, a dispatcher batch.
struct Posted {
  fxc_scan* s = nullptr;
  std::condition_variable* cv = nullptr;  // the posting worker's (woken alone)
  fxc::StagedSector ss{};
  uint64_t nf = 0, first = 0;
  cudaEvent_t done = nullptr;  // recorded after the batch that computed it
  bool launched = false;
  fxc_status st = FXC_OK;
  std::string err;
};

constexpr int kBatchEvents = 4;  // batches in flight at most, plus slack
constexpr uint32_t kMaxBatch = 1024;

}  // namespace

struct fxc_server {
  fxc_engine* eng = nullptr;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> queue;
  std::unordered_map<uint64_t, Job*> jobs;  // submitted, not yet waited
  std::vector<std::thread> workers;
  uint64_t next_id = 1;
  int running = 0;       // jobs on a slot
  int idle_holding = 0;  // idle slots that still hold device buffers
  bool pressure = false; // a job waits for HBM: idle slots release theirs
  bool stopping = false;
  // batched mode
  fxc_batch* batch = nullptr;
  std::thread dispatcher;
  std::deque<Posted*> posted;
  std::condition_variable cv_post;
  bool disp_stop = false;
  cudaStream_t disp_stream = nullptr;
  cudaEvent_t ev[kBatchEvents] = {};
};

namespace {

// Streams one job's sectors through scan s (opened on first use).
fxc_status run_job(fxc_server* sv, fxc_scan** sp, Job* J) {
  fxc_scan_cfg cfg = J->cfg;
  cfg.delay.geom_table = J->table.empty() ? nullptr : J->table.data();
  // admission: bind the slot's scan within the budget, or wait for memory
  bool batch_released = false;
  for (;;) {
    fxc_status st = *sp ? fxc::scan_bind(*sp, &cfg) : fxc_scan_open(sv->eng, &cfg, sp);
    if (st != FXC_EBUSY) {
      if (st != FXC_OK) return st;
      break;
    }
    if (*sp) {  // this slot's own buffers have the wrong shape: release them first
      fxc_scan_close(*sp);
      *sp = nullptr;
      continue;
    }
    std::unique_lock<std::mutex> lk(sv->mu);
    if (sv->running <= 1 && sv->idle_holding == 0) {
      // no other job holds memory; the batch's tables and partials (grown
      // by earlier batches) are the last thing to give back
      if (sv->batch && !batch_released) {
        lk.unlock();
        fxc::batch_release(sv->batch);
        batch_released = true;
        continue;
      }
      return st;  // nothing can free memory
    }
    sv->pressure = true;
    sv->cv_work.notify_all();
    sv->cv_done.wait_for(lk, std::chrono::milliseconds(2));
  }
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->pressure = false;
  }
  fxc_scan* s = *sp;
  const fxc_job& j = J->job;
  const uint64_t h = cfg.fft_len / 2 + 1;
  const uint64_t b1 = fxc_bytes_per_frame(cfg.fft_len, cfg.bits1);
  const uint64_t b2 = fxc_bytes_per_frame(cfg.fft_len, cfg.bits2);
  const uint64_t bo = fxc_bytes_per_frame(cfg.fft_len, cfg.bits_out);
  const bool raw = (cfg.products & FXC_PROD_RAW) && j.raw_out;
  const uint64_t sf = j.sector_frames ? j.sector_frames : std::max<uint64_t>(j.nf, 1);
  const uint64_t nsec = j.nf ? (j.nf + sf - 1) / sf : 1;
  struct Pending {
    uint64_t id, sec, f0, nfs;
  };
  std::deque<Pending> inflight;
  fxc_status result = FXC_OK;
  auto finish_one = [&]() -> fxc_status {
    const Pending p = inflight.front();
    inflight.pop_front();
    double* base = j.out + p.sec * 5 * h;
    fxc_sector_out o{};
    o.acf11 = base;
    o.acf22 = base + h;
    o.xcf = base + 2 * h;
    o.phased = base + 4 * h;
    if (raw) {
      o.raw_out = j.raw_out + p.f0 * bo;
      o.raw_out_len = p.nfs * bo;
    }
    const fxc_status st = fxc_sector_wait(s, p.id, -1, &o);
    if (st == FXC_OK) J->stats.sectors += 1;
    return st;
  };
  if (sv->batch) {
    // batched: stage, post to the dispatcher, collect behind its batch
    std::deque<std::pair<Posted, uint64_t>> posts;  // (post, sector index)
    std::condition_variable cv_mine;  // the dispatcher wakes this worker only
    auto finish_posted = [&]() -> fxc_status {
      Posted& p = posts.front().first;
      const uint64_t sec = posts.front().second;
      {
        std::unique_lock<std::mutex> lk(sv->mu);
        cv_mine.wait(lk, [&] { return p.launched; });
      }
      fxc_status st = p.st;
      uint64_t id = 0;
      if (st == FXC_OK) st = fxc::sector_collect(s, p.ss, p.done, &id);
      else fxc::sector_release(s, p.ss);
      if (st == FXC_OK) {
        const uint64_t f0 = sec * sf;
        inflight.push_back({id, sec, f0, p.nf});
        st = finish_one();
      } else if (!p.err.empty()) {
        fxc::internal_fail(st, p.err.c_str());
      }
      posts.pop_front();
      return st;
    };
    for (uint64_t sec = 0; sec < nsec && result == FXC_OK; ++sec) {
      const uint64_t f0 = sec * sf;
      const uint64_t nfs = j.nf ? std::min(sf, j.nf - f0) : 0;
      Posted np;
      np.s = s;
      np.cv = &cv_mine;
      np.nf = nfs;
      np.first = j.first_frame + f0;
      fxc_status st;
      for (;;) {
        st = fxc::sector_stage(s, j.raw1 + f0 * b1, nfs * b1, j.raw2 + f0 * b2, nfs * b2, nfs,
                               &np.ss);
        if (st != FXC_EBUSY || posts.empty()) break;
        // every sector slot in flight: finish the oldest
        if ((st = finish_posted()) != FXC_OK) break;
      }
      if (st != FXC_OK) {
        result = st;
        break;
      }
      posts.emplace_back(np, sec);
      {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->posted.push_back(&posts.back().first);
      }
      sv->cv_post.notify_one();
    }
    while (!posts.empty()) {
      const fxc_status st = finish_posted();
      if (result == FXC_OK) result = st;
    }
    return result;
  }
  // sectors in flight: as many as the scan's sector slots (the engine's
  // max_inflight) take; a submit that finds them all busy drains the oldest
  for (uint64_t sec = 0; sec < nsec && result == FXC_OK; ++sec) {
    const uint64_t f0 = sec * sf;
    const uint64_t nfs = j.nf ? std::min(sf, j.nf - f0) : 0;
    uint64_t id = 0;
    fxc_status st;
    for (;;) {
      st = fxc_sector_submit(s, j.raw1 + f0 * b1, nfs * b1, j.raw2 + f0 * b2, nfs * b2, nfs,
                             j.first_frame + f0, &id);
      if (st != FXC_EBUSY || inflight.empty()) break;
      // all sector slots busy, or staging memory over budget: drain one
      if ((st = finish_one()) != FXC_OK) break;
    }
    if (st != FXC_OK) {
      result = st;
      break;
    }
    inflight.push_back({id, sec, f0, nfs});
  }
  while (!inflight.empty()) {
    const fxc_status st = finish_one();
    if (result == FXC_OK) result = st;
  }
  return result;
}

void worker(fxc_server* sv) {
  fxc_scan* scan = nullptr;  // this slot's device context, kept between jobs
  std::unique_lock<std::mutex> lk(sv->mu);
  for (;;) {
    if (scan) sv->idle_holding += 1;
    sv->cv_work.wait(lk, [&] {
      return sv->stopping || !sv->queue.empty() || (sv->pressure && scan);
    });
    if (scan) sv->idle_holding -= 1;
    if (sv->queue.empty() && !sv->stopping) {
      // another slot waits for HBM: give this idle slot's buffers back
      fxc_scan* s = scan;
      scan = nullptr;
      lk.unlock();
      fxc_scan_close(s);
      lk.lock();
      sv->cv_done.notify_all();
      continue;
    }
    if (sv->queue.empty()) break;  // stopping, nothing left
    if (sv->stopping) {
      // shutting down: a job that has not started fails at once
      for (Job* Q : sv->queue) {
        Q->stats.status = FXC_EBUSY;
        Q->stats.t_start_ns = Q->stats.t_done_ns = now_ns();
        Q->error = "the server was destroyed before the job started";
        Q->done = true;
      }
      sv->queue.clear();
      sv->cv_done.notify_all();
      break;
    }
    Job* J = sv->queue.front();
    sv->queue.pop_front();
    sv->running += 1;
    lk.unlock();
    J->stats.t_start_ns = now_ns();
    const fxc_status st = run_job(sv, &scan, J);
    std::string err = st == FXC_OK ? std::string() : std::string(fxc_last_error());
    lk.lock();
    J->stats.status = st;
    J->stats.t_done_ns = now_ns();
    J->error = err;
    J->done = true;
    sv->running -= 1;
    sv->cv_done.notify_all();
  }
  lk.unlock();
  if (scan) fxc_scan_close(scan);
}

// Batched mode: computes every posted sector (one per scan and batch) with
// one fxc_batch_run_device call; at most two batches in flight.
void dispatcher(fxc_server* sv) {
  const int dev = fxc::engine_device(sv->eng);
  cudaSetDevice(dev);
  std::deque<int> inflight;  // event indices of batches in flight
  int next_ev = 0;
  std::vector<Posted*> take;
  std::vector<Posted*> later;
  std::vector<fxc_scan*> scans;
  std::vector<const uint8_t*> r1, r2;
  std::vector<uint64_t> nfs, firsts;
  std::vector<double*> accs;
  std::vector<uint8_t*> raws;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv_post.wait(lk, [&] { return sv->disp_stop || !sv->posted.empty(); });
      if (sv->posted.empty()) break;  // stopping, nothing left
    }
    // the previous batch but one must be done: the next one gathers meanwhile
    while ((int)inflight.size() >= 2) {
      cudaEventSynchronize(sv->ev[inflight.front()]);
      inflight.pop_front();
    }
    take.clear();
    later.clear();
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      std::vector<fxc_scan*> seen;
      while (!sv->posted.empty() && take.size() < kMaxBatch) {
        Posted* p = sv->posted.front();
        sv->posted.pop_front();
        if (std::find(seen.begin(), seen.end(), p->s) != seen.end()) {
          later.push_back(p);  // a scan's next sector waits for the next batch
          continue;
        }
        seen.push_back(p->s);
        take.push_back(p);
      }
      for (auto it = later.rbegin(); it != later.rend(); ++it) sv->posted.push_front(*it);
    }
    scans.clear();
    r1.clear();
    r2.clear();
    nfs.clear();
    firsts.clear();
    accs.clear();
    raws.clear();
    for (Posted* p : take) {
      cudaStreamWaitEvent(sv->disp_stream, p->ss.h2d, 0);
      scans.push_back(p->s);
      r1.push_back(p->ss.d_raw1);
      r2.push_back(p->ss.d_raw2);
      nfs.push_back(p->nf);
      firsts.push_back(p->first);
      accs.push_back(p->ss.d_acc);
      raws.push_back(p->ss.d_raw_out);
    }
    fxc_status st = fxc_batch_run_device_raw(sv->batch, scans.data(), r1.data(), r2.data(),
                                             nfs.data(), firsts.data(), accs.data(), raws.data(),
                                             (uint32_t)take.size(), sv->disp_stream);
    std::string err;
    if (st == FXC_EBUSY || st == FXC_ENOMEM) {
      // no room for the batch's tables: each sector on its scan's own buffers
      st = FXC_OK;
      for (Posted* p : take) {
        const fxc_status s1 = fxc::run_sector_internal(p->s, p->ss.d_raw1, p->ss.d_raw2, p->nf,
                                                       p->first, p->ss.d_acc, p->ss.d_raw_out,
                                                       sv->disp_stream);
        if (s1 != FXC_OK) {
          st = s1;
          break;
        }
      }
    }
    if (st != FXC_OK) err = fxc_last_error();
    const int e = next_ev;
    next_ev = (next_ev + 1) % kBatchEvents;
    cudaEventRecord(sv->ev[e], sv->disp_stream);
    inflight.push_back(e);
    {
      // notified under the lock: a worker cannot run on (and drop its post)
      // before the dispatcher is done with it
      std::lock_guard<std::mutex> lk(sv->mu);
      for (Posted* p : take) {
        p->done = sv->ev[e];
        p->st = st;
        p->err = err;
        p->launched = true;
        p->cv->notify_one();
      }
    }
  }
  cudaStreamSynchronize(sv->disp_stream);
}

}  // namespace

extern "C" {

fxc_status fxc_server_create(fxc_engine* e, const fxc_server_opts* opts, fxc_server** out) {
  if (!e || !out) return fxc::internal_fail(FXC_EINVAL, "NULL argument");
  *out = nullptr;
  const int slots = (opts && opts->slots > 0) ? opts->slots : 4;
  if (slots > 256) return fxc::internal_fail(FXC_EINVAL, "at most 256 slots");
  auto* sv = new fxc_server();
  sv->eng = e;
  if (opts && opts->batch) {
    fxc_batch_opts bo{};
    bo.use_graphs = 1;
    bo.autotune = opts->batch == 1 ? 1 : 0;  // 2: fixed shapes, timing-independent products
    fxc_status st = fxc_batch_create(e, &bo, &sv->batch);
    if (st != FXC_OK) {
      delete sv;
      return st;
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(fxc::engine_device(e));
    bool ok = cudaStreamCreateWithFlags(&sv->disp_stream, cudaStreamNonBlocking) == cudaSuccess;
    for (int k = 0; k < kBatchEvents && ok; ++k)
      ok = cudaEventCreateWithFlags(&sv->ev[k], cudaEventDisableTiming | cudaEventBlockingSync) ==
           cudaSuccess;
    cudaSetDevice(prev);
    if (!ok) {
      for (auto& ev : sv->ev)
        if (ev) cudaEventDestroy(ev);
      if (sv->disp_stream) cudaStreamDestroy(sv->disp_stream);
      fxc_batch_destroy(sv->batch);
      delete sv;
      return fxc::internal_fail(FXC_ECUDA, "server: dispatcher stream or events");
    }
    sv->dispatcher = std::thread(dispatcher, sv);
  }
  for (int k = 0; k < slots; ++k) sv->workers.emplace_back(worker, sv);
  fxc::engine_track_server(e, sv, true);
  *out = sv;
  return FXC_OK;
}

fxc_status fxc_server_submit(fxc_server* sv, const fxc_job* job, uint64_t* job_id) {
  if (!sv || !job || !job_id || !job->cfg || !job->out)
    return fxc::internal_fail(FXC_EINVAL, "NULL argument");
  if (job->nf && (!job->raw1 || !job->raw2))
    return fxc::internal_fail(FXC_EINVAL, "input buffer is NULL");
  auto* J = new Job();
  J->cfg = *job->cfg;
  if (job->cfg->delay.geom_table && job->cfg->delay.geom_len)
    J->table.assign(job->cfg->delay.geom_table,
                    job->cfg->delay.geom_table + job->cfg->delay.geom_len);
  J->cfg.delay.geom_table = nullptr;
  J->job = *job;
  J->job.cfg = nullptr;
  J->stats.t_submit_ns = now_ns();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stopping) {
      delete J;
      return fxc::internal_fail(FXC_EINVAL, "server is shutting down");
    }
    J->id = sv->next_id++;
    sv->jobs[J->id] = J;
    sv->queue.push_back(J);
    *job_id = J->id;
  }
  sv->cv_work.notify_one();
  return FXC_OK;
}

fxc_status fxc_server_wait(fxc_server* sv, uint64_t job_id, int32_t timeout_ms,
                           fxc_job_stats* stats) {
  if (!sv) return fxc::internal_fail(FXC_EINVAL, "server is NULL");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(job_id);
  if (it == sv->jobs.end()) return fxc::internal_fail(FXC_ENOTFOUND, "job id not pending");
  Job* J = it->second;
  auto ready = [&] { return J->done; };
  if (timeout_ms < 0) {
    sv->cv_done.wait(lk, ready);
  } else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return fxc::internal_fail(FXC_ETIMEDOUT, "job not done within the timeout");
  }
  sv->jobs.erase(it);
  lk.unlock();
  if (stats) *stats = J->stats;
  const fxc_status st = (fxc_status)J->stats.status;
  const std::string err = J->error;
  delete J;
  if (st != FXC_OK) return fxc::internal_fail(st, err.c_str());
  return FXC_OK;
}

fxc_status fxc_server_destroy(fxc_server* sv) {
  if (!sv) return FXC_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stopping = true;
  }
  sv->cv_work.notify_all();
  for (auto& t : sv->workers) t.join();
  if (sv->dispatcher.joinable()) {
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->disp_stop = true;
    }
    sv->cv_post.notify_all();
    sv->dispatcher.join();
  }
  if (sv->batch) {
    for (auto& ev : sv->ev)
      if (ev) cudaEventDestroy(ev);
    if (sv->disp_stream) cudaStreamDestroy(sv->disp_stream);
    fxc_batch_destroy(sv->batch);
  }
  for (auto& kv : sv->jobs) delete kv.second;
  fxc::engine_track_server(sv->eng, sv, false);
  delete sv;
  return FXC_OK;
}

}  // extern "C"
