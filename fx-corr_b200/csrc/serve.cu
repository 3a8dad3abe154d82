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
};

namespace {

// Streams one job's sectors through scan s (opened on first use).
fxc_status run_job(fxc_server* sv, fxc_scan** sp, Job* J) {
  fxc_scan_cfg cfg = J->cfg;
  cfg.delay.geom_table = J->table.empty() ? nullptr : J->table.data();
  // admission: bind the slot's scan within the budget, or wait for memory
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
    if (sv->running <= 1 && sv->idle_holding == 0) return st;  // nothing can free memory
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

}  // namespace

extern "C" {

fxc_status fxc_server_create(fxc_engine* e, const fxc_server_opts* opts, fxc_server** out) {
  if (!e || !out) return fxc::internal_fail(FXC_EINVAL, "NULL argument");
  *out = nullptr;
  const int slots = (opts && opts->slots > 0) ? opts->slots : 4;
  if (slots > 64) return fxc::internal_fail(FXC_EINVAL, "at most 64 slots");
  auto* sv = new fxc_server();
  sv->eng = e;
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
  for (auto& kv : sv->jobs) delete kv.second;
  fxc::engine_track_server(sv->eng, sv, false);
  delete sv;
  return FXC_OK;
}

}  // extern "C"
