// cor_writer.cpp — GICO3-compatible .cor writer (fx-corr src/cor.rs:1-326).
#include "cor_writer.h"

#include <cmath>
#include <cstring>
#include <ctime>
#include <stdexcept>

namespace yi {

namespace {

void put_i32(uint8_t* b, size_t off, int32_t v) { std::memcpy(b + off, &v, 4); }
void put_u32(uint8_t* b, size_t off, uint32_t v) { std::memcpy(b + off, &v, 4); }
void put_f32(uint8_t* b, size_t off, float v) { std::memcpy(b + off, &v, 4); }
void put_f64(uint8_t* b, size_t off, double v) { std::memcpy(b + off, &v, 8); }
void put_ascii(uint8_t* b, size_t off, size_t len, const std::string& s) {
  std::memset(b + off, 0, len);
  std::memcpy(b + off, s.data(), std::min(len, s.size()));
}

// split_sec_nsec (cor.rs:111-140)
void split_sec_nsec(int64_t unix_sec, double extra, uint32_t* sec_out, uint32_t* nsec_out) {
  if (!std::isfinite(extra)) throw std::runtime_error("non-finite sector time offset");
  double sec = (double)unix_sec + extra;
  double nsec = (sec - std::trunc(sec)) * 1e9;
  sec = std::floor(sec);
  if (nsec < 0.0) {
    nsec += 1e9;
    sec -= 1.0;
  } else if (nsec >= 1e9) {
    nsec -= 1e9;
    sec += 1.0;
  }
  int64_t s = (int64_t)sec;
  int64_t ns = (int64_t)std::llround(nsec);
  if (ns >= 1000000000) {
    s += 1;
    ns = 0;
  }
  if (s < 0 || s > 0xFFFFFFFFll) throw std::runtime_error("sector sec out of u32 range for .cor sector header");
  if (ns < 0 || ns > 0xFFFFFFFFll) throw std::runtime_error("sector nsec out of u32 range for .cor sector header");
  *sec_out = (uint32_t)s;
  *nsec_out = (uint32_t)ns;
}

}  // namespace

void build_cor_file_header(const CorHeaderConfig& cfg, const CorStation& st1,
                           const CorStation& st2, uint8_t out[256]) {
  if (cfg.fft_point <= 0 || (cfg.fft_point % 2) != 0)
    throw std::runtime_error("cor header fft_point must be positive even integer");
  if (cfg.number_of_sector_hint < 0)
    throw std::runtime_error("cor header number_of_sector_hint must be non-negative");
  if (cfg.clock_reference_unix_sec < 0 || cfg.clock_reference_unix_sec > 0xFFFFFFFFll)
    throw std::runtime_error("clock_reference_unix_sec out of u32 range for .cor header");
  const uint32_t clk = (uint32_t)cfg.clock_reference_unix_sec;
  std::memset(out, 0, 256);
  const uint8_t magic[4] = {0x83, 0xF9, 0xA2, 0x3E};
  std::memcpy(out, magic, 4);
  put_i32(out, 4, 0x01030000);
  put_i32(out, 8, 1);
  put_i32(out, 12, cfg.sampling_speed_hz);
  put_f64(out, 16, cfg.observing_frequency_hz);
  put_i32(out, 24, cfg.fft_point);
  put_i32(out, 28, cfg.number_of_sector_hint);
  put_ascii(out, 32, 16, st1.name);
  put_f64(out, 48, st1.ecef_m[0]);
  put_f64(out, 56, st1.ecef_m[1]);
  put_f64(out, 64, st1.ecef_m[2]);
  put_ascii(out, 72, 1, std::string(1, (char)st1.code));
  put_ascii(out, 80, 16, st2.name);
  put_f64(out, 96, st2.ecef_m[0]);
  put_f64(out, 104, st2.ecef_m[1]);
  put_f64(out, 112, st2.ecef_m[2]);
  put_ascii(out, 120, 1, std::string(1, (char)st2.code));
  put_ascii(out, 128, 16, cfg.source_name);
  put_f64(out, 144, cfg.source_ra_rad);
  put_f64(out, 152, cfg.source_dec_rad);
  put_u32(out, 160, clk);
  put_u32(out, 164, 0);
  put_u32(out, 208, clk);
  put_u32(out, 212, 0);
}

void build_cor_sector_header(int64_t ts, float integ, uint8_t out[128]) {
  if (ts < INT32_MIN || ts > INT32_MAX)
    throw std::runtime_error("timestamp out of i32 range for .cor sector header");
  std::memset(out, 0, 128);
  put_i32(out, 0, (int32_t)ts);
  uint32_t st_sec, st_nsec, et_sec, et_nsec;
  split_sec_nsec(ts, 0.0, &st_sec, &st_nsec);
  const double integ_sec = (std::isfinite(integ) && integ > 0.0f) ? (double)integ : 1.0;
  split_sec_nsec(ts, integ_sec, &et_sec, &et_nsec);
  put_u32(out, 4, st_nsec);
  put_u32(out, 8, et_sec);
  put_u32(out, 12, et_nsec);
  put_f32(out, 112, integ);
}

CorWriter::CorWriter(const std::string& path, const CorHeaderConfig& cfg, const CorStation& st1,
                     const CorStation& st2)
    : path_(path), fft_half_(cfg.fft_point / 2) {
  uint8_t hdr[256];
  build_cor_file_header(cfg, st1, st2, hdr);
  f_ = std::fopen(path.c_str(), "wb");
  if (!f_) throw std::runtime_error("cannot create " + path);
  if (std::fwrite(hdr, 1, 256, f_) != 256) throw std::runtime_error("write failed: " + path);
}

CorWriter::~CorWriter() {
  if (f_) std::fclose(f_);
}

void CorWriter::write_sector(int64_t ts, float integ, const float* spectrum) {
  uint8_t hdr[128];
  build_cor_sector_header(ts, integ, hdr);
  if (std::fwrite(hdr, 1, 128, f_) != 128 ||
      std::fwrite(spectrum, sizeof(float), 2 * (size_t)fft_half_, f_) != 2 * (size_t)fft_half_)
    throw std::runtime_error("write failed: " + path_);
  ++sectors_;
}

void CorWriter::finalize() {
  if (!f_) return;
  std::fflush(f_);
  std::fseek(f_, 28, SEEK_SET);
  std::fwrite(&sectors_, 4, 1, f_);
  std::fclose(f_);
  f_ = nullptr;
}

std::string unix_seconds_to_yyyydddhhmmss(int64_t unix_seconds) {
  const int64_t c = std::max<int64_t>(INT32_MIN, std::min<int64_t>(INT32_MAX, unix_seconds));
  const time_t ts = (time_t)c;
  struct tm tm_out;
  if (!gmtime_r(&ts, &tm_out)) throw std::runtime_error("gmtime_r failed while formatting epoch");
  char buf[32];
  std::snprintf(buf, sizeof buf, "%04d%03d%02d%02d%02d", tm_out.tm_year + 1900, tm_out.tm_yday + 1,
                tm_out.tm_hour, tm_out.tm_min, tm_out.tm_sec);
  return buf;
}

}  // namespace yi
