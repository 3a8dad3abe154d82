// yi_main.cpp — the yi-acf / yi-xcf / yi-corr / yi-phasedarray tools on the
// B200 engine: the reference's command line, XML schedule merge, input seek,
// sector plan, .cor / phased .raw outputs (fx-corr src/main.rs:889-1013 main,
// 1013-2772 run_once), with every sector correlated by libfxc
// (fxc_sector_submit / fxc_sector_wait) while a reader thread streams the next
// sectors from the .raw files into page-locked buffers.
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdarg>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <exception>
#include <mutex>
#include <set>
#include <optional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "args.h"
#include "cor_writer.h"
#include "fxc.h"
#include "geom.h"
#include "schedule.h"

namespace yi {
namespace {

enum class Mode { Acf, Xcf, PhasedArray, Corr };

const char* mode_label(Mode m) {  // main.rs:254-262
  switch (m) {
    case Mode::Acf: return "yi_acf";
    case Mode::Xcf: return "yi-xcf";
    case Mode::PhasedArray: return "yi-phasedarray";
    default: return "yi-corr";
  }
}

// detect_run_mode_from_argv0 (main.rs:265-278)
Mode mode_from_argv0(const char* argv0) {
  std::string p = argv0 ? argv0 : "";
  const size_t sl = p.find_last_of('/');
  if (sl != std::string::npos) p = p.substr(sl + 1);
  const size_t dot = p.find_last_of('.');
  if (dot != std::string::npos && dot > 0) p = p.substr(0, dot);
  for (auto& c : p) c = (char)std::tolower((unsigned char)c);
  if (p == "yi_acf" || p == "yi-acf") return Mode::Acf;
  if (p == "yi-xcf" || p == "yi_xcf") return Mode::Xcf;
  if (p == "yi_phasedarray" || p == "yi-phasedarray") return Mode::PhasedArray;
  return Mode::Corr;
}

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// An error the reference raises as std::io::Error::other(String): its main
// prints the Debug form `Custom { kind: Other, error: "..." }`.
struct IoFail : Fail {
  using Fail::Fail;
};

// A string's Debug form: quoted, with quotes and backslashes escaped.
std::string debug_quoted(const std::string& m) {
  std::string q = "\"";
  for (char c : m) {
    if (c == '"' || c == '\\') q += '\\';
    if (c == '\n') {
      q += "\\n";
      continue;
    }
    q += c;
  }
  return q + "\"";
}

// std::io::Error's Display of an OS error: "<strerror> (os error <n>)".
std::string os_error(int e) { return std::string(std::strerror(e)) + " (os error " + std::to_string(e) + ")"; }

// ------------------------------------------------------------------ logging
// println! of the reference, optionally teed to ./stdout/stdout_<tag>.log
// (main.rs:36-108, yi-corr only).
FILE* g_tee = nullptr;
std::mutex g_log_mu;

// Output files held by the processes running at once (--jobs): two
// processes that would write the same file take turns, as they would one
// after another.
std::mutex g_out_mu;
std::condition_variable g_out_cv;
std::set<std::string> g_out_busy;

struct OutputClaim {
  std::vector<std::string> paths;
  explicit OutputClaim(std::vector<std::string> p) : paths(std::move(p)) {
    std::unique_lock<std::mutex> lk(g_out_mu);
    g_out_cv.wait(lk, [&] {
      for (const auto& x : paths)
        if (g_out_busy.count(x)) return false;
      return true;
    });
    for (const auto& x : paths) g_out_busy.insert(x);
  }
  ~OutputClaim() {
    {
      std::lock_guard<std::mutex> lk(g_out_mu);
      for (const auto& x : paths) g_out_busy.erase(x);
    }
    g_out_cv.notify_all();
  }
};

void logf(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
void logf(const char* fmt, ...) {
  char buf[4096];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  std::lock_guard<std::mutex> lk(g_log_mu);
  std::fputs(buf, stdout);
  std::fputc('\n', stdout);
  std::fflush(stdout);
  if (g_tee) {
    std::fputs(buf, g_tee);
    std::fputc('\n', g_tee);
    std::fflush(g_tee);
  }
}

void mkdir_p(const std::string& d) {
  std::string cur;
  for (size_t i = 0; i < d.size(); ++i) {
    cur += d[i];
    if (d[i] == '/' || i + 1 == d.size()) {
      if (cur == "/") continue;
      if (::mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST)
        throw Fail("failed to create directory " + cur + ": " + std::strerror(errno));
    }
  }
}

bool file_exists(const std::string& p) {
  struct stat st;
  return ::stat(p.c_str(), &st) == 0;
}

uint64_t file_size(const std::string& p) {
  struct stat st;
  if (::stat(p.c_str(), &st) != 0)
    throw Fail("No such file or directory (os error 2): " + p);
  return (uint64_t)st.st_size;
}

std::string cwd() {
  char b[4096];
  if (!::getcwd(b, sizeof b)) throw Fail("getcwd failed");
  return b;
}

std::string join(const std::string& d, const std::string& f) {
  if (d.empty()) return f;
  return d.back() == '/' ? d + f : d + "/" + f;
}

// sanitize_file_token (main.rs:561-576)
std::string sanitize(const std::string& raw) {
  std::string out;
  for (unsigned char c : raw) out += (std::isalnum(c) || c == '-' || c == '_') ? (char)c : '_';
  size_t a = 0, b = out.size();
  while (a < b && out[a] == '_') ++a;
  while (b > a && out[b - 1] == '_') --b;
  out = out.substr(a, b - a);
  return out.empty() ? "unknown" : out;
}

std::pair<int64_t, std::string> epoch_tag(const std::string& ep) {
  const int64_t u = epoch_to_unix_seconds(ep);
  return {u, unix_seconds_to_yyyydddhhmmss(u)};
}

double level_power(const std::vector<double>& lv, const char* label) {  // main.rs:378-387
  if (lv.empty()) throw Fail(std::string(label) + " levels are empty");
  double p = 0.0;
  for (double v : lv) p += v * v;
  p /= (double)lv.size();
  if (!std::isfinite(p) || p <= 0.0)
    throw Fail(std::string(label) + " mean-square level is invalid: " + std::to_string(p));
  return p;
}

void ck(fxc_status s, const char* what) {
  if (s != FXC_OK) throw Fail(std::string(what) + ": " + fxc_last_error());
}

// ------------------------------------------------------------- raw reader
// PackedSampleReader at a word-aligned start (bit offset 0) with zero padding
// of short reads (main.rs:445-503, 1578-1616).
class RawReader {
 public:
  // label: "ant1" / "ant2", for the reference's read-error message
  RawReader(const std::string& path, uint64_t start_byte, const char* label)
      : path_(path), label_(label) {
    f_ = std::fopen(path.c_str(), "rb");
    if (!f_) throw Fail("failed to open/seek " + path + ": " + os_error(errno));
    if (fseeko(f_, (off_t)start_byte, SEEK_SET) != 0)
      throw Fail("failed to open/seek " + path + ": " + os_error(errno));
#ifdef POSIX_FADV_SEQUENTIAL
    posix_fadvise(fileno(f_), 0, 0, POSIX_FADV_SEQUENTIAL);
    posix_fadvise(fileno(f_), 0, 0, POSIX_FADV_WILLNEED);
#endif
  }
  ~RawReader() {
    if (f_) std::fclose(f_);
  }
  RawReader(const RawReader&) = delete;
  RawReader& operator=(const RawReader&) = delete;
  // read_with_padding (main.rs:445-456): a short read leaves the tail zero
  void read_padded(uint8_t* out, size_t n) {
    size_t got = 0;
    while (got < n) {
      errno = 0;
      const size_t r = std::fread(out + got, 1, n - got, f_);
      if (r == 0) {
        if (std::ferror(f_)) {
          if (errno == EINTR) {
            std::clearerr(f_);
            continue;
          }
          throw Fail(std::string("failed reading ") + label_ + " input: " + os_error(errno));
        }
        break;
      }
      got += r;
    }
    if (got < n) std::memset(out + got, 0, n - got);
  }

 private:
  std::string path_;
  const char* label_;
  FILE* f_ = nullptr;
};

// Opens a station's reader; a failure is reported as the reference's reader
// thread reports it through its channel (main.rs:2110-2127, 2196-2210).
std::unique_ptr<RawReader> open_reader(const std::string& path, uint64_t start_byte,
                                       const char* label) {
  try {
    return std::make_unique<RawReader>(path, start_byte, label);
  } catch (const std::exception& e) {
    throw IoFail(std::string("synth reader error: ") + e.what());
  }
}

// One sector's packed bytes of both stations in page-locked memory.
struct SectorBuf {
  uint8_t* b1 = nullptr;
  uint8_t* b2 = nullptr;
  uint64_t cap1 = 0, cap2 = 0;
  uint64_t nf = 0;
  size_t index = 0;
};

// Reader thread: fills free buffers with consecutive sectors in order.
class SectorReader {
 public:
  SectorReader(const std::string& p1, uint64_t s1, const std::string& p2, uint64_t s2,
               std::vector<uint64_t> counts, uint64_t bpf1, uint64_t bpf2, int depth)
      : r1_(open_reader(p1, s1, "ant1")), r2_(open_reader(p2, s2, "ant2")),
        counts_(std::move(counts)), bpf1_(bpf1), bpf2_(bpf2) {
    uint64_t mx = 0;
    for (uint64_t c : counts_) mx = std::max(mx, c);
    for (int k = 0; k < depth; ++k) {
      auto b = std::make_unique<SectorBuf>();
      b->cap1 = std::max<uint64_t>(mx * bpf1, 16);
      b->cap2 = std::max<uint64_t>(mx * bpf2, 16);
      ck(fxc_host_alloc(b->cap1, reinterpret_cast<void**>(&b->b1)), "fxc_host_alloc");
      ck(fxc_host_alloc(b->cap2, reinterpret_cast<void**>(&b->b2)), "fxc_host_alloc");
      free_.push_back(b.get());
      owned_.push_back(std::move(b));
    }
    th_ = std::thread([this] { run(); });
  }
  ~SectorReader() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (th_.joinable()) th_.join();
    for (auto& b : owned_) {
      fxc_host_free(b->b1);
      fxc_host_free(b->b2);
    }
  }
  // Next filled sector in order (nullptr at the end); throws the reader's error.
  SectorBuf* next() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return !ready_.empty() || done_ || !err_.empty(); });
    if (!err_.empty()) throw IoFail("synth reader error: " + err_);
    if (ready_.empty()) return nullptr;
    SectorBuf* b = ready_.front();
    ready_.pop_front();
    return b;
  }
  void release(SectorBuf* b) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      free_.push_back(b);
    }
    cv_.notify_all();
  }
  uint64_t bytes_read() const { return bytes_.load(); }

 private:
  void run() {
    try {
      for (size_t i = 0; i < counts_.size(); ++i) {
        SectorBuf* b = nullptr;
        {
          std::unique_lock<std::mutex> lk(mu_);
          cv_.wait(lk, [&] { return stop_ || !free_.empty(); });
          if (stop_) return;
          b = free_.front();
          free_.pop_front();
        }
        b->nf = counts_[i];
        b->index = i;
        r1_->read_padded(b->b1, b->nf * bpf1_);
        r2_->read_padded(b->b2, b->nf * bpf2_);
        bytes_ += b->nf * (bpf1_ + bpf2_);
        {
          std::lock_guard<std::mutex> lk(mu_);
          ready_.push_back(b);
        }
        cv_.notify_all();
      }
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lk(mu_);
      err_ = e.what();
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      done_ = true;
    }
    cv_.notify_all();
  }
  std::unique_ptr<RawReader> r1_, r2_;
  std::vector<uint64_t> counts_;
  uint64_t bpf1_, bpf2_;
  std::vector<std::unique_ptr<SectorBuf>> owned_;
  std::deque<SectorBuf*> free_, ready_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::thread th_;
  std::atomic<uint64_t> bytes_{0};
  bool stop_ = false, done_ = false;
  std::string err_;
};

// ----------------------------------------------------------------- run_once

constexpr double kCorOneSidedPowerFactor = 0.5;  // main.rs:35
const int kDefaultShuffleIn[32] = {31, 30, 29, 28, 27, 26, 25, 24, 23, 22, 21, 20, 19, 18, 17, 16,
                                   15, 14, 13, 12, 11, 10, 9,  8,  7,  6,  5,  4,  3,  2,  1,  0};

std::string join_csv(const int* v, int n) {
  std::string s;
  for (int i = 0; i < n; ++i) s += (i ? "," : "") + std::to_string(v[i]);
  return s;
}

// With `server` (--jobs > 1) the sectors are submitted as one-dump jobs to
// a batched server shared by the processes running at once; otherwise they
// stream through a scan of this process.
void run_once(const Args& args, Mode mode, const std::optional<Schedule>& sch, fxc_engine* eng,
              fxc_server* server = nullptr) {
  const bool fringe_enabled = mode == Mode::PhasedArray && args.fringe;
  if (args.fringe && mode != Mode::PhasedArray) logf("[info] --fringe is ignored for this mode");
  if (fringe_enabled)
    logf("[info] --fringe: the whole-scan XCF delay diagnostic is not part of this build; "
         "phased products are written as usual");
  const bool write_raw = mode == Mode::PhasedArray;
  const bool write_acf_cor = mode == Mode::Acf || mode == Mode::Corr;
  const bool write_xcf_cor = mode == Mode::Xcf || mode == Mode::Corr;
  const bool write_phased_cor = mode == Mode::PhasedArray;

  std::optional<ProcessEntry> proc;
  if (sch) {
    if (args.process_index) {
      if (*args.process_index >= sch->processes.size())
        throw Fail("--process-index " + std::to_string(*args.process_index) +
                   " out of range (0.." +
                   std::to_string(sch->processes.empty() ? 0 : sch->processes.size() - 1) + ")");
      proc = sch->processes[*args.process_index];
      logf("[info] Selected process index %zu: epoch=%s skip=%g length=%s", *args.process_index,
           proc->epoch.c_str(), proc->skip_sec,
           proc->length_sec ? std::to_string(*proc->length_sec).c_str() : "-");
    } else if (!sch->processes.empty()) {
      proc = sch->processes.front();
    }
  }
  // configuration merge, with the reference's precedence (main.rs:1061-1110)
  size_t fft_len =
      args.fft == kDefaultFft ? (sch && sch->fft ? *sch->fft : args.fft) : args.fft;
  const std::vector<std::string> bit_a = args.bin.empty() ? std::vector<std::string>{"2"} : args.bin;
  auto bits = per_antenna_usize(bit_a, sch && sch->ant1_bit ? *sch->ant1_bit : 2);
  // this build's per-process extension: <fft>, <bit> (both stations) and
  // <level> inside <process> override the values above; a <bit> without a
  // <level> takes the uniform table of 2^b half-integer steps
  std::optional<std::string> proc_level;
  if (proc && proc->fft) fft_len = *proc->fft;
  if (proc && proc->bit) {
    bits = {*proc->bit, *proc->bit};
    proc_level = proc->level;
    if (!proc_level) {
      std::string d;
      const long n = 1L << *proc->bit;
      for (long i = 0; i < n; ++i) {
        char b[32];
        std::snprintf(b, sizeof b, "%s%.1f", i ? "," : "", (double)i - 0.5 * (double)(n - 1));
        d += b;
      }
      proc_level = d;
    }
  } else if (proc && proc->level) {
    proc_level = proc->level;
  }
  const size_t bit1 = bits.first, bit2 = bits.second, bit_out = std::max(bit1, bit2);
  const auto level_args = proc_level ? std::vector<std::string>{*proc_level}
                                     : normalize_level_args(args.level, bit1, bit2);
  const auto lv_s = per_antenna_str(
      level_args, sch && sch->ant1_level ? *sch->ant1_level : std::string("-1.5,-0.5,0.5,1.5"));
  const std::vector<double> levels1 = parse_levels(bit1, lv_s.first);
  const std::vector<double> levels2 = parse_levels(bit2, lv_s.second);
  const double lp1 = level_power(levels1, "ant1"), lp2 = level_power(levels2, "ant2");
  const auto shuffle_args = normalize_shuffle_args(args.shuffle_in);
  const auto sh_s = per_antenna_str(
      shuffle_args, sch && sch->ant1_shuffle ? *sch->ant1_shuffle : join_csv(kDefaultShuffleIn, 32));
  const std::vector<int> sh1 = parse_shuffle_internal(sh_s.first);
  const std::vector<int> sh2 = parse_shuffle_internal(sh_s.second);
  const auto sb_s = per_antenna_str(args.sideband.empty() ? std::vector<std::string>{"LSB"}
                                                          : args.sideband,
                                    sch && sch->ant1_sideband ? *sch->ant1_sideband : "LSB", true);
  const bool lsb1 = sb_s.first == "LSB", lsb2 = sb_s.second == "LSB";
  const auto tsys = per_antenna_f64(args.tsys, 1.0);
  const auto dia = per_antenna_f64(args.diameter, 0.0);
  const auto eta = per_antenna_f64(args.eta, 0.65);
  const auto gain = per_antenna_f64(args.gain, 1.0);
  const auto sefd = per_antenna_f64(args.sefd, 0.0);

  const double fs = sch && sch->sampling_hz ? *sch->sampling_hz : args.sampling * 1e6;
  const double obs_mhz = sch && sch->obsfreq_mhz ? *sch->obsfreq_mhz : args.obsfreq;
  std::string ep_i = "2000";
  if (args.epoch) ep_i = *args.epoch;
  else if (proc) ep_i = proc->epoch;
  else if (sch && sch->epoch) ep_i = *sch->epoch;

  // input files (main.rs:518-529)
  std::string a1p, a2p;
  if (args.ant1 && args.ant2) {
    epoch_tag(ep_i);
    a1p = *args.ant1;
    a2p = *args.ant2;
  } else {
    const std::string dir = args.raw_directory ? *args.raw_directory : ".";
    const std::string tag = epoch_tag(ep_i).second;
    std::vector<std::pair<std::string, std::string>> cand;
    if (sch && sch->ant1_station_name && sch->ant2_station_name)
      cand.push_back({*sch->ant1_station_name, *sch->ant2_station_name});
    cand.push_back({"YAMAGU32", "YAMAGU34"});
    bool found = false;
    for (const auto& c : cand) {
      const std::string p1 = join(dir, c.first + "_" + tag + ".raw");
      const std::string p2 = join(dir, c.second + "_" + tag + ".raw");
      if (file_exists(p1) && file_exists(p2)) {
        logf("[info] Auto-resolved inputs: %s / %s", p1.c_str(), p2.c_str());
        a1p = p1;
        a2p = p2;
        found = true;
        break;
      }
    }
    if (!found) throw Fail("Input files not found");
  }
  const int64_t c_unix_base = epoch_tag(ep_i).first;
  double ant1_ecef[3], ant2_ecef[3];
  for (int k = 0; k < 3; ++k) {
    ant1_ecef[k] = sch && sch->ant1_ecef_m ? (*sch->ant1_ecef_m)[k] : kYamagu32Ecef[k];
    ant2_ecef[k] = sch && sch->ant2_ecef_m ? (*sch->ant2_ecef_m)[k] : kYamagu34Ecef[k];
  }

  // geometry (main.rs:1101-1118): J2000 input, precessed to the epoch
  bool have_geom = false;
  double src_ra = 0.0, src_dec = 0.0, mjd0 = 0.0, gd0 = 0.0, gr0 = 0.0, ga0 = 0.0;
  std::optional<std::string> ra_in = args.ra, dec_in = args.dec;
  if (!ra_in && proc && proc->ra) ra_in = proc->ra;
  if (!dec_in && proc && proc->dec) dec_in = proc->dec;
  if (!ra_in && sch) ra_in = sch->ra;
  if (!dec_in && sch) dec_in = sch->dec;
  if (ra_in && dec_in) {
    const double ra_raw = parse_ra(*ra_in), dec_raw = parse_dec(*dec_in);
    mjd0 = parse_epoch_to_mjd(ep_i);
    precess_j2000_to_mean_of_date(ra_raw, dec_raw, mjd0, &src_ra, &src_dec);
    const GeomDelay g = geometric_delay_and_derivatives(ant1_ecef, ant2_ecef, src_ra, src_dec, mjd0);
    gd0 = g.delay;
    gr0 = g.rate;
    ga0 = g.accel;
    have_geom = true;
  }
  // clocks (main.rs:1119-1172)
  const double cd_rel = sch && sch->clock_delay_s ? *sch->clock_delay_s : 0.0;
  const double cr_rel = sch && sch->clock_rate_sps ? *sch->clock_rate_sps : 0.0;
  const double c1d_base = sch && sch->ant1_clock_delay_s ? *sch->ant1_clock_delay_s : 0.0;
  const double c2d_base = sch && sch->ant2_clock_delay_s ? *sch->ant2_clock_delay_s : c1d_base + cd_rel;
  const double c1r = sch && sch->ant1_clock_rate_sps ? *sch->ant1_clock_rate_sps : 0.0;
  const double c2r = sch && sch->ant2_clock_rate_sps ? *sch->ant2_clock_rate_sps : c1r + cr_rel;
  double c1_off = 0.0, c2_off = 0.0;
  if (sch && sch->ant1_clock_epoch) {
    try {
      c1_off = (double)(c_unix_base - epoch_to_unix_seconds(*sch->ant1_clock_epoch));
    } catch (const std::exception& e) {
      throw Fail("invalid ant1 clock epoch '" + *sch->ant1_clock_epoch + "': " + e.what());
    }
  }
  if (sch && sch->ant2_clock_epoch) {
    try {
      c2_off = (double)(c_unix_base - epoch_to_unix_seconds(*sch->ant2_clock_epoch));
    } catch (const std::exception& e) {
      throw Fail("invalid ant2 clock epoch '" + *sch->ant2_clock_epoch + "': " + e.what());
    }
  }
  const double c1d = c1d_base + c1r * c1_off;
  const double c2d = c2d_base + c2r * c2_off;
  const double clock_delay_s = c2d - c1d;
  const double clock_rate_sps = c2r - c1r;
  const double coarse_delay_s = args.coarse ? *args.coarse : 0.0;
  const double delay_user_samples = args.delay + args.resdelay;
  const double rate_user_hz = args.rate + args.resrate;
  const double net_d_rel_no_clock0 = gd0 + coarse_delay_s + delay_user_samples / fs;
  const double net_d0 = net_d_rel_no_clock0 + clock_delay_s;

  // rotations: XML, then --rotation (main.rs:1183-1205; in an ant1:/ant2:
  // entry, parts without a prefix are ignored)
  double rot1 = sch && sch->ant1_rotation_hz ? *sch->ant1_rotation_hz : 0.0;
  double rot2 = sch && sch->ant2_rotation_hz ? *sch->ant2_rotation_hz : 0.0;
  for (const auto& entry : args.rotation) {
    if (entry.find("ant1:") != std::string::npos || entry.find("ant2:") != std::string::npos) {
      std::string cur;
      std::vector<std::string> parts;
      for (char c : entry) {
        if (c == ',' || c == ' ') {
          if (!cur.empty()) parts.push_back(cur);
          cur.clear();
        } else {
          cur += c;
        }
      }
      if (!cur.empty()) parts.push_back(cur);
      for (const auto& part : parts) {
        if (part.rfind("ant1:", 0) == 0) rot1 = parse_f64(part.substr(5));
        else if (part.rfind("ant2:", 0) == 0) rot2 = parse_f64(part.substr(5));
      }
    } else {
      std::string t = entry;
      while (!t.empty() && std::isspace((unsigned char)t.back())) t.pop_back();
      while (!t.empty() && std::isspace((unsigned char)t.front())) t.erase(t.begin());
      rot1 = rot2 = parse_f64(t);
    }
  }
  const double bw = fs / 2e6;
  const double a1_low = obs_mhz + rot1 / 1e6, a2_low = obs_mhz + rot2 / 1e6;
  const double lo1_hz = a1_low * 1e6, lo2_hz = a2_low * 1e6;
  int64_t band[4];
  if (fxc_band_alignment((uint32_t)fft_len, fs, a1_low + 0.5 * bw, a2_low + 0.5 * bw, bw, bw,
                         band) != FXC_OK)
    throw Fail(fxc_last_error());
  const int grid = std::fabs(rot1) <= std::fabs(rot2) ? 0 : 1;

  const uint64_t bpf1 = (fft_len * bit1 + 7) / 8, bpf2 = (fft_len * bit2 + 7) / 8;
  const uint64_t bpf_o = (fft_len * bit_out + 7) / 8;
  if (args.chunk_frames && *args.chunk_frames == 0) throw Fail("--chunk-frames must be >= 1");
  if (args.pipeline_depth && *args.pipeline_depth == 0) throw Fail("--pipeline-depth must be >= 1");
  const uint64_t f1_len = file_size(a1p), f2_len = file_size(a2p);
  if (args.skip < 0.0) throw Fail("--skip must be >= 0");
  if (args.length && *args.length < 0.0) throw Fail("--length must be >= 0");
  const double xml_skip = proc ? proc->skip_sec : (sch && sch->process_skip_sec ? *sch->process_skip_sec : 0.0);
  std::optional<double> xml_length;
  if (proc && proc->length_sec) xml_length = proc->length_sec;
  else if (sch && sch->process_length_sec) xml_length = sch->process_length_sec;
  if (xml_skip < 0.0) throw Fail("XML process/skip must be >= 0");
  if (xml_length && *xml_length < 0.0) throw Fail("XML process/length must be >= 0");
  const double total_skip_sec = xml_skip + args.skip;
  const int64_t c_unix = c_unix_base + (int64_t)std::llround(total_skip_sec);
  const std::string c_tag = unix_seconds_to_yyyydddhhmmss(c_unix);
  // output layout (main.rs:531-545)
  std::string o_dir;
  if (mode == Mode::PhasedArray) {
    o_dir = cwd();
  } else {
    if (!args.cor_directory) throw Fail("--cor-directory is required for yi-acf/yi-xcf/yi-corr");
    o_dir = *args.cor_directory;
    mkdir_p(o_dir);
  }
  const std::string o_path = join(o_dir, "YAMAGU66_" + c_tag + ".raw");
  std::optional<double> window = args.length ? args.length : xml_length;

  // scan window (main.rs:1276-1304)
  const uint64_t total_samples1 = f1_len * 8 / bit1, total_samples2 = f2_len * 8 / bit2;
  const int64_t init_delay = (int64_t)std::llround(net_d0 * fs);
  const uint64_t seek1 = init_delay < 0 ? (uint64_t)(-init_delay) : 0;
  const uint64_t seek2 = init_delay > 0 ? (uint64_t)init_delay : 0;
  const uint64_t skip_samples = (uint64_t)std::llround(total_skip_sec * fs);
  const uint64_t start1 = seek1 + skip_samples, start2 = seek2 + skip_samples;
  const uint64_t avail1 = total_samples1 > start1 ? total_samples1 - start1 : 0;
  const uint64_t avail2 = total_samples2 > start2 ? total_samples2 - start2 : 0;
  const double available_sec = (double)std::min(avail1, avail2) / fs;
  const double requested_sec = window ? std::max(*window - total_skip_sec, 0.0) : available_sec;
  const double total_sec = std::min(requested_sec, available_sec);
  const uint64_t total_f = (uint64_t)std::floor(total_sec * fs / (double)fft_len);

  const double w1 = resolve_weight(tsys.first, gain.first,
                                   sefd.first > 0.0 ? std::optional<double>(sefd.first) : std::nullopt,
                                   dia.first > 0.0 ? std::optional<double>(dia.first) : std::nullopt,
                                   eta.first, "A1");
  const double w2 = resolve_weight(tsys.second, gain.second,
                                   sefd.second > 0.0 ? std::optional<double>(sefd.second) : std::nullopt,
                                   dia.second > 0.0 ? std::optional<double>(dia.second) : std::nullopt,
                                   eta.second, "A2");
  const std::string a1_name = sch && sch->ant1_station_name ? *sch->ant1_station_name : "YAMAGU32";
  const std::string a2_name = sch && sch->ant2_station_name ? *sch->ant2_station_name : "YAMAGU34";
  auto code_of = [](const std::optional<std::string>& key, const std::string& name, uint8_t d) {
    if (key && !key->empty()) return (uint8_t)(*key)[0];
    if (!name.empty()) return (uint8_t)name[0];
    return d;
  };
  const uint8_t a1_code = code_of(sch ? sch->ant1_station_key : std::nullopt, a1_name, '1');
  const uint8_t a2_code = code_of(sch ? sch->ant2_station_key : std::nullopt, a2_name, '2');

  // rates (main.rs:1316-1328)
  const double correction_sign = -1.0;
  const double geometric_rate_hz = correction_sign * gr0 * obs_mhz * 1e6;
  const double df_hz = fs / (double)fft_len;
  const double rotation_residual_hz = (rot1 - rot2) - (double)band[0] * df_hz;
  const double rotation_fringe_hz = -rotation_residual_hz;

  logf(mode == Mode::PhasedArray ? "Starting phased array processing with the following arguments:"
                                 : "Starting correlation processing with the following arguments:");
  logf("--------------------------------------------------");
  logf("  mode:       %s", mode_label(mode));
  logf("  %s:  %s (Size: %llu bytes)", a1_name.c_str(), a1p.c_str(), (unsigned long long)f1_len);
  logf("  %s:  %s (Size: %llu bytes)", a2_name.c_str(), a2p.c_str(), (unsigned long long)f2_len);
  logf("  fft:        %zu  sampling: %.3f Msps  bits: %zu/%zu  sideband: %s/%s", fft_len, fs / 1e6,
       bit1, bit2, sb_s.first.c_str(), sb_s.second.c_str());
  logf("  band-align: shift %lld bins, overlap [%lld..%lld), grid %s", (long long)band[0],
       (long long)band[1], (long long)band[2], grid == 0 ? a1_name.c_str() : a2_name.c_str());
  logf("  read-align delay: %.3f samples (%.3e s)", net_d0 * fs, net_d0);
  logf("  frames:     %llu (%.6f s)", (unsigned long long)total_f,
       (double)total_f * (double)fft_len / fs);
  logf("--------------------------------------------------");

  // word-aligned starts (main.rs:1577-1616)
  const uint64_t spw1 = 32 / bit1, spw2 = 32 / bit2;
  if (spw1 == 0 || spw2 == 0) throw Fail("invalid samples-per-word while aligning input start");
  const uint64_t start1_a = (start1 / spw1) * spw1, start2_a = (start2 / spw2) * spw2;
  const uint64_t start1_byte = start1_a * bit1 / 8, start2_byte = start2_a * bit2 / 8;
  const int64_t res1 = (int64_t)start1_a - (int64_t)start1, res2 = (int64_t)start2_a - (int64_t)start2;
  logf("[info] Input start ant1: desired sample %llu -> byte %llu + bit 0 (actual sample %llu, "
       "residual %lld sample)", (unsigned long long)start1, (unsigned long long)start1_byte,
       (unsigned long long)start1_a, (long long)res1);
  logf("[info] Input start ant2: desired sample %llu -> byte %llu + bit 0 (actual sample %llu, "
       "residual %lld sample)", (unsigned long long)start2, (unsigned long long)start2_byte,
       (unsigned long long)start2_a, (long long)res2);
  if (res1 != 0 || res2 != 0)
    logf("[info] Word-aligned seek residual: ant1=%lld sample(s), ant2=%lld sample(s)",
         (long long)res1, (long long)res2);
  const double d_seek = ((double)((int64_t)start2_a - (int64_t)start1_a)) / fs;

  // delay model (main.rs:1618-1673)
  const double frame_dt = (double)fft_len / fs;
  const double net_d1_base = net_d_rel_no_clock0 + clock_delay_s - d_seek;
  const double rate_rel_no_clock = (geometric_rate_hz + rotation_fringe_hz + rate_user_hz) / (obs_mhz * 1e6);
  const double total_rate1_base = rate_rel_no_clock + clock_rate_sps;
  const double total_accel1_base = correction_sign * ga0;
  std::vector<double> table;
  if (have_geom) {
    const double total_duration = (double)total_f * frame_dt;
    const size_t n_update = (size_t)std::max(std::ceil(total_duration), 1.0);
    for (size_t sec = 0; sec <= n_update; ++sec) {
      const double t_abs = total_skip_sec + (double)sec;
      table.push_back(baseline_delay(ant1_ecef, ant2_ecef, src_ra, src_dec, mjd0 + t_abs / 86400.0));
    }
    logf("[info] Delay model refinement: 1-second geometric-delay table enabled (process scope, "
         "%zu entries)", table.size());
  }
  const double extra_rate = (rotation_fringe_hz + rate_user_hz) / (obs_mhz * 1e6);

  std::string source_name = "UNKNOWN";
  if (proc && proc->object) source_name = *proc->object;
  else if (sch && sch->source) source_name = *sch->source;
  const std::string cor_label =
      sanitize(mode == Mode::PhasedArray ? std::string("phasedarray")
                                         : (sch && sch->stream_label ? *sch->stream_label
                                                                     : std::string("phasedarray")));
  const std::string n1f = sanitize(a1_name), n2f = sanitize(a2_name);
  if (total_f == 0) return;

  // sector plan (main.rs:2058-2072)
  const double total_duration = (double)total_f * frame_dt;
  uint64_t sector_count = (uint64_t)std::max(std::round(total_duration), 1.0);
  sector_count = std::min<uint64_t>(sector_count, std::max<uint64_t>(total_f, 1));
  std::vector<uint64_t> counts;
  for (uint64_t si = 0; si < sector_count; ++si) {
    const uint64_t nf = total_f / sector_count + (si < total_f % sector_count ? 1 : 0);
    if (nf) counts.push_back(nf);
  }

  // device scan
  fxc_scan_cfg cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.fft_len = (uint32_t)fft_len;
  cfg.bits1 = (uint32_t)bit1;
  cfg.bits2 = (uint32_t)bit2;
  cfg.bits_out = (uint32_t)bit_out;
  cfg.fs_hz = fs;
  for (size_t i = 0; i < levels1.size(); ++i) cfg.levels1[i] = levels1[i];
  for (size_t i = 0; i < levels2.size(); ++i) cfg.levels2[i] = levels2[i];
  cfg.nlevels1 = (uint32_t)levels1.size();
  cfg.nlevels2 = (uint32_t)levels2.size();
  for (int i = 0; i < 32; ++i) {
    cfg.shuffle1[i] = (uint8_t)sh1[i];
    cfg.shuffle2[i] = (uint8_t)sh2[i];
  }
  cfg.lsb1 = lsb1;
  cfg.lsb2 = lsb2;
  cfg.shift_bins = band[0];
  cfg.a1s = (uint32_t)band[1];
  cfg.a1e = (uint32_t)band[2];
  cfg.a2s = (uint32_t)band[3];
  cfg.grid = grid;
  if (mode == Mode::Acf) cfg.products = FXC_PROD_ACF | FXC_PROD_ACF_OVERLAP_ONLY;
  else if (mode == Mode::Xcf) cfg.products = FXC_PROD_XCF;
  else if (mode == Mode::Corr) cfg.products = FXC_PROD_ACF | FXC_PROD_XCF;
  else cfg.products = FXC_PROD_PHASED | FXC_PROD_RAW;
  cfg.w1 = w1;
  cfg.w2 = w2;
  fxc_delay_cfg& d = cfg.delay;
  d.frame_dt = frame_dt;
  d.fs = fs;
  d.time_offset_s = total_skip_sec;
  d.geom_table = table.empty() ? nullptr : table.data();
  d.geom_len = table.size();
  d.coarse_delay_s = coarse_delay_s;
  d.delay_user_samples = delay_user_samples;
  d.extra_delay_rate_sps = extra_rate;
  d.clock1_delay_s = c1d;
  d.clock1_rate_sps = c1r;
  d.clock2_delay_s = c2d;
  d.clock2_rate_sps = c2r;
  d.d_seek = d_seek;
  d.net_d1_base = net_d1_base;
  d.total_rate1_base = total_rate1_base;
  d.total_accel1_base = total_accel1_base;
  d.net_d2_base = 0.0;
  d.total_rate2_base = 0.0;
  d.total_accel2_base = 0.0;
  d.lo1_hz = lo1_hz;
  d.lo2_hz = lo2_hz;
  fxc_scan* scan = nullptr;
  if (!server) ck(fxc_scan_open(eng, &cfg, &scan), "fxc_scan_open");
  struct ScanCloser {
    fxc_scan* s;
    ~ScanCloser() {
      if (s) fxc_scan_close(s);
    }
  } closer{scan};

  // writers (main.rs:2074-2096)
  CorHeaderConfig hc;
  hc.sampling_speed_hz = (int32_t)std::lround(fs);
  hc.observing_frequency_hz = obs_mhz * 1e6;
  hc.fft_point = (int32_t)fft_len;
  hc.number_of_sector_hint = (int32_t)counts.size();
  hc.clock_reference_unix_sec = c_unix;
  hc.source_name = source_name;
  hc.source_ra_rad = have_geom ? src_ra : 0.0;
  hc.source_dec_rad = have_geom ? src_dec : 0.0;
  CorStation s1{a1_name, a1_code, {ant1_ecef[0], ant1_ecef[1], ant1_ecef[2]}};
  CorStation s2{a2_name, a2_code, {ant2_ecef[0], ant2_ecef[1], ant2_ecef[2]}};
  CorStation sm{"YAMAGU66", (uint8_t)'M', {ant1_ecef[0], ant1_ecef[1], ant1_ecef[2]}};
  std::unique_ptr<OutputClaim> claim;
  if (server) {
    std::vector<std::string> outs;
    if (write_phased_cor)
      outs.push_back(join(o_dir, "YAMAGU66_YAMAGU66_" + c_tag + "_" + cor_label + ".cor"));
    if (write_acf_cor) {
      outs.push_back(join(o_dir, n1f + "_" + n1f + "_" + c_tag + "_" + cor_label + ".cor"));
      outs.push_back(join(o_dir, n2f + "_" + n2f + "_" + c_tag + "_" + cor_label + ".cor"));
    }
    if (write_xcf_cor)
      outs.push_back(join(o_dir, n1f + "_" + n2f + "_" + c_tag + "_" + cor_label + ".cor"));
    if (write_raw) outs.push_back(o_path);
    claim = std::make_unique<OutputClaim>(std::move(outs));
  }
  std::unique_ptr<CorWriter> cw_ph, cw_11, cw_12, cw_22;
  if (write_phased_cor)
    cw_ph = std::make_unique<CorWriter>(
        join(o_dir, "YAMAGU66_YAMAGU66_" + c_tag + "_" + cor_label + ".cor"), hc, sm, sm);
  if (write_acf_cor)
    cw_11 = std::make_unique<CorWriter>(join(o_dir, n1f + "_" + n1f + "_" + c_tag + "_" + cor_label + ".cor"),
                                        hc, s1, s1);
  if (write_xcf_cor)
    cw_12 = std::make_unique<CorWriter>(join(o_dir, n1f + "_" + n2f + "_" + c_tag + "_" + cor_label + ".cor"),
                                        hc, s1, s2);
  if (write_acf_cor)
    cw_22 = std::make_unique<CorWriter>(join(o_dir, n2f + "_" + n2f + "_" + c_tag + "_" + cor_label + ".cor"),
                                        hc, s2, s2);
  FILE* raw_out = nullptr;
  if (write_raw) {
    raw_out = std::fopen(o_path.c_str(), "wb");
    if (!raw_out) throw Fail("failed to create " + o_path + ": " + std::strerror(errno));
  }
  logf(mode == Mode::PhasedArray ? "[info] Synthesising output..." : "[info] Integrating correlation sectors...");

  const int depth = args.pipeline_depth ? (int)std::max<size_t>(*args.pipeline_depth, 2) : 3;
  SectorReader reader(a1p, start1_byte, a2p, start2_byte, counts, bpf1, bpf2, depth);
  const size_t h = fft_len / 2 + 1;
  std::vector<double> acc11(h), acc22(h), xcf(2 * h), ph(h);
  std::vector<uint8_t> raw_frames;
  std::vector<float> spec(fft_len);  // fft/2 (re, im) pairs
  struct Inflight {
    uint64_t id;
    SectorBuf* buf;
    std::vector<double> out;    // server jobs: acf11 | acf22 | xcf | phased
    std::vector<uint8_t> raw;   // server jobs: phased .raw frames
  };
  std::deque<Inflight> inflight;
  // on an error, server jobs still reading this process's reader buffers
  // finish before the buffers are freed (declared after the reader, so
  // destroyed before it)
  struct DrainJobs {
    std::deque<Inflight>* q;
    fxc_server* sv;
    ~DrainJobs() {
      if (!sv) return;
      for (auto& in : *q) {
        fxc_job_stats js;
        fxc_server_wait(sv, in.id, -1, &js);
      }
    }
  } drain{&inflight, server};
  uint64_t emitted = 0;
  const auto t_start = std::chrono::steady_clock::now();
  auto finish = [&]() {
    Inflight in = std::move(inflight.front());
    inflight.pop_front();
    const uint64_t nf = in.buf->nf;
    const size_t si = in.buf->index;
    fxc_sector_out o;
    std::memset(&o, 0, sizeof o);
    o.acf11 = acc11.data();
    o.acf22 = acc22.data();
    o.xcf = xcf.data();
    o.phased = ph.data();
    if (write_raw) {
      raw_frames.resize(nf * bpf_o);
      o.raw_out = raw_frames.data();
      o.raw_out_len = raw_frames.size();
    }
    if (server) {
      fxc_job_stats js;
      ck(fxc_server_wait(server, in.id, -1, &js), "sector");
      std::memcpy(acc11.data(), in.out.data(), sizeof(double) * h);
      std::memcpy(acc22.data(), in.out.data() + h, sizeof(double) * h);
      std::memcpy(xcf.data(), in.out.data() + 2 * h, sizeof(double) * 2 * h);
      std::memcpy(ph.data(), in.out.data() + 4 * h, sizeof(double) * h);
      if (write_raw) raw_frames = std::move(in.raw);
    } else {
      ck(fxc_sector_wait(scan, in.id, -1, &o), "sector");
    }
    reader.release(in.buf);
    if (raw_out && !raw_frames.empty() &&
        std::fwrite(raw_frames.data(), 1, raw_frames.size(), raw_out) != raw_frames.size())
      throw Fail("failed writing " + o_path);
    emitted += nf;
    const float integ = (float)((double)nf * (double)fft_len / fs);
    const int64_t ts = c_unix + (int64_t)si;
    // normalisation + dump (main.rs:2645-2683)
    if (cw_ph) {
      ck(fxc_normalize((uint32_t)fft_len, nf, std::max(w1 * w1 * lp1 + w2 * w2 * lp2, 1e-12),
                       ph.data(), nullptr, spec.data()), "normalize");
      cw_ph->write_sector(ts, integ, spec.data());
    }
    if (cw_11) {
      ck(fxc_normalize((uint32_t)fft_len, nf, lp1, acc11.data(), nullptr, spec.data()), "normalize");
      cw_11->write_sector(ts, integ, spec.data());
    }
    if (cw_12) {
      ck(fxc_normalize((uint32_t)fft_len, nf, std::sqrt(lp1 * lp2), nullptr, xcf.data(), spec.data()),
         "normalize");
      cw_12->write_sector(ts, integ, spec.data());
    }
    if (cw_22) {
      ck(fxc_normalize((uint32_t)fft_len, nf, lp2, acc22.data(), nullptr, spec.data()), "normalize");
      cw_22->write_sector(ts, integ, spec.data());
    }
    if (!server) {  // processes running at once would overwrite each other's line
      std::printf("\r[info] %s second %zu/%zu (%.2f%%)",
                  mode == Mode::PhasedArray ? "Synthesised" : "Processed", si + 1, counts.size(),
                  100.0 * (double)emitted / (double)total_f);
      std::fflush(stdout);
    }
  };
  uint64_t first_frame = 0;
  for (;;) {
    // server jobs hold their reader buffers until done: leave the reader one
    if (server && (int)inflight.size() >= depth - 1) finish();
    SectorBuf* b = reader.next();
    if (!b) break;
    uint64_t id = 0;
    if (server) {
      Inflight in{0, b, std::vector<double>(5 * h), {}};
      if (write_raw) in.raw.resize(b->nf * bpf_o);
      fxc_job j;
      std::memset(&j, 0, sizeof j);
      j.cfg = &cfg;
      j.raw1 = b->b1;
      j.raw2 = b->b2;
      j.nf = b->nf;
      j.first_frame = first_frame;
      j.sector_frames = 0;
      j.out = in.out.data();
      j.raw_out = write_raw ? in.raw.data() : nullptr;
      ck(fxc_server_submit(server, &j, &in.id), "fxc_server_submit");
      first_frame += b->nf;
      inflight.push_back(std::move(in));
      continue;
    }
    for (;;) {
      const fxc_status st = fxc_sector_submit(scan, b->b1, b->nf * bpf1, b->b2, b->nf * bpf2, b->nf,
                                              first_frame, &id);
      if (st == FXC_EBUSY && !inflight.empty()) {
        finish();
        continue;
      }
      ck(st, "fxc_sector_submit");
      break;
    }
    first_frame += b->nf;
    inflight.push_back({id, b, {}, {}});
  }
  while (!inflight.empty()) finish();
  if (!counts.empty() && !server) std::printf("\n");
  const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  logf("[info] I/O reader summary: avg=%.1f MiB/s total=%.1f MiB, %.3f s",
       (double)reader.bytes_read() / (1024.0 * 1024.0) / std::max(el, 1e-9),
       (double)reader.bytes_read() / (1024.0 * 1024.0), el);
  if (raw_out) std::fclose(raw_out);
  for (auto* w : {cw_ph.get(), cw_11.get(), cw_12.get(), cw_22.get()})
    if (w) w->finalize();
  if (mode == Mode::PhasedArray)
    logf("[info] Phased-array spectrum plots are not produced by this build (presentation only)");
}

int real_main(int argc, char** argv) {
  const Mode mode = mode_from_argv0(argc > 0 ? argv[0] : "yi-corr");
  std::string prog = argc > 0 ? argv[0] : "yi-corr";
  {
    const size_t sl = prog.find_last_of('/');
    if (sl != std::string::npos) prog = prog.substr(sl + 1);
  }
  Args args;
  try {
    args = parse_args(argc, argv, prog);
  } catch (const ArgsExit& e) {
    std::fputs(e.what(), e.code == 0 ? stdout : stderr);
    std::fputc('\n', e.code == 0 ? stdout : stderr);
    return e.code;
  }
  if (args.mkxml) {
    write_example_xml("example.xml");
    logf("[info] Wrote example schedule XML: example.xml");
    return 0;
  }
  if (args.stdout_log && mode == Mode::Corr) {
    const int64_t now = (int64_t)std::time(nullptr);
    const std::string tag = unix_seconds_to_yyyydddhhmmss(now);
    const std::string dir = join(cwd(), "stdout");
    mkdir_p(dir);
    const std::string path = join(dir, "stdout_" + tag + ".log");
    g_tee = std::fopen(path.c_str(), "w");
    if (!g_tee) throw Fail("failed to create " + path);
    std::fprintf(g_tee, "# yi-corr stdout log started at %s\n", tag.c_str());
    logf("[info] stdout log dir: %s", dir.c_str());
    logf("[info] stdout log: %s", path.c_str());
  }
  if (mode == Mode::PhasedArray) {
    if (!args.schedule) throw Fail("--schedule is required for yi-phasedarray");
    if (!args.raw_directory) throw Fail("--raw-directory is required for yi-phasedarray");
  } else {
    if (!args.schedule) throw Fail("--schedule is required for yi-acf/yi-xcf/yi-corr");
    if (!args.raw_directory) throw Fail("--raw-directory is required for yi-acf/yi-xcf/yi-corr");
    if (!args.cor_directory) throw Fail("--cor-directory is required for yi-acf/yi-xcf/yi-corr");
  }
  if (args.cpu && *args.cpu == 0) throw Fail("--cpu must be >= 1");
  std::optional<Schedule> sch;
  if (args.schedule) {
    const std::string& p = *args.schedule;
    const size_t dot = p.find_last_of('.');
    std::string ext = dot == std::string::npos ? "" : p.substr(dot + 1);
    for (auto& c : ext) c = (char)std::tolower((unsigned char)c);
    if (ext != "xml" || p.find_last_of('/') + 1 == p.size())
      throw Fail("--schedule must point to a .xml file");
    sch = parse_xml_schedule(p);
  }
  fxc_device_opts dopts;
  std::memset(&dopts, 0, sizeof dopts);
  dopts.device = 0;
  dopts.max_inflight = 3;
  fxc_engine* eng = nullptr;
  ck(fxc_engine_create(&dopts, &eng), "fxc_engine_create");
  struct EngineCloser {
    fxc_engine* e;
    ~EngineCloser() { fxc_engine_destroy(e); }
  } ec{eng};
  const bool run_all = sch && sch->processes.size() > 1 && !args.process_index && !args.epoch &&
                       !args.ra && !args.dec && !args.length && args.skip == 0.0;
  if (run_all && args.jobs && *args.jobs > 1) {
    // this build's extension: up to --jobs processes at once, their sectors
    // computed together by a batched server (fixed kernel shapes, so the
    // products do not depend on timing)
    const size_t np = sch->processes.size();
    const size_t nj = std::min(*args.jobs, np);
    logf("[info] Processing all scans, %zu at a time: %zu process entries", nj, np);
    fxc_server_opts so;
    std::memset(&so, 0, sizeof so);
    so.slots = (int32_t)std::min<size_t>(256, std::max<size_t>(4, 2 * nj));
    so.batch = 2;
    fxc_server* sv = nullptr;
    ck(fxc_server_create(eng, &so, &sv), "fxc_server_create");
    struct ServerCloser {
      fxc_server* s;
      ~ServerCloser() { fxc_server_destroy(s); }
    } sc{sv};
    std::mutex mu;
    size_t next = 0;
    std::exception_ptr first_error;
    auto worker = [&]() {
      for (;;) {
        size_t idx;
        {
          std::lock_guard<std::mutex> lk(mu);
          if (next >= np || first_error) return;
          idx = next++;
        }
        const ProcessEntry& p = sch->processes[idx];
        logf("[info] process %zu/%zu: epoch=%s skip=%g length=%s", idx + 1, np, p.epoch.c_str(),
             p.skip_sec, p.length_sec ? std::to_string(*p.length_sec).c_str() : "-");
        Args ra = args;
        ra.process_index = idx;
        ra.compact_logs = true;
        const auto t0 = std::chrono::steady_clock::now();
        try {
          run_once(ra, mode, sch, eng, sv);
          logf("[info] process %zu/%zu elapsed: %.3fs", idx + 1, np,
               std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
        } catch (...) {
          logf("[error] process %zu/%zu failed after %.3fs", idx + 1, np,
               std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
          std::lock_guard<std::mutex> lk(mu);
          if (!first_error) first_error = std::current_exception();
        }
      }
    };
    std::vector<std::thread> ths;
    for (size_t k = 0; k < nj; ++k) ths.emplace_back(worker);
    for (auto& t : ths) t.join();
    if (first_error) std::rethrow_exception(first_error);
    return 0;
  }
  if (run_all) {
    const size_t np = sch->processes.size();
    logf("[info] Processing all scans sequentially: %zu process entries", np);
    for (size_t idx = 0; idx < np; ++idx) {
      const ProcessEntry& p = sch->processes[idx];
      logf("[info] process %zu/%zu: epoch=%s skip=%g length=%s", idx + 1, np, p.epoch.c_str(),
           p.skip_sec, p.length_sec ? std::to_string(*p.length_sec).c_str() : "-");
      Args ra = args;
      ra.process_index = idx;
      ra.compact_logs = idx > 0;
      const auto t0 = std::chrono::steady_clock::now();
      try {
        run_once(ra, mode, sch, eng);
      } catch (...) {
        logf("[error] process %zu/%zu failed after %.3fs", idx + 1, np,
             std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
        throw;
      }
      logf("[info] process %zu/%zu elapsed: %.3fs", idx + 1, np,
           std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }
    return 0;
  }
  run_once(args, mode, sch, eng);
  return 0;
}

}  // namespace
}  // namespace yi

int main(int argc, char** argv) {
  try {
    return yi::real_main(argc, argv);
  } catch (const yi::IoFail& e) {
    // an io::Error::other(String) returned from main: its Debug form
    std::fflush(stdout);
    std::fprintf(stderr, "Error: Custom { kind: Other, error: %s }\n",
                 yi::debug_quoted(e.what()).c_str());
    return 1;
  } catch (const std::exception& e) {
    // a Rust main returning Err prints the error's Debug form and exits 1
    std::fflush(stdout);
    std::fprintf(stderr, "Error: %s\n", yi::debug_quoted(e.what()).c_str());
    return 1;
  }
}
