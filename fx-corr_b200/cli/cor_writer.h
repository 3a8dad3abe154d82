// cor_writer.h — GICO3-compatible .cor output (format of fx-corr src/cor.rs).
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>

namespace yi {

struct CorStation {
  std::string name;
  uint8_t code = 0;
  double ecef_m[3] = {0, 0, 0};
};

struct CorHeaderConfig {
  int32_t sampling_speed_hz = 0;
  double observing_frequency_hz = 0.0;
  int32_t fft_point = 0;
  int32_t number_of_sector_hint = 0;
  int64_t clock_reference_unix_sec = 0;
  std::string source_name;
  double source_ra_rad = 0.0, source_dec_rad = 0.0;
};

// 256-byte file header (cor.rs:152-203); throws std::runtime_error on invalid values.
void build_cor_file_header(const CorHeaderConfig& cfg, const CorStation& st1,
                           const CorStation& st2, uint8_t out[256]);
// 128-byte sector header (cor.rs:234-285, no clock model).
void build_cor_sector_header(int64_t timestamp_unix_sec, float effective_integ_time_s,
                             uint8_t out[128]);

// Sequential writer: header, then per sector a 128-byte header and fft/2
// (f32 re, f32 im) pairs; finalize() patches the sector count at byte 28.
class CorWriter {
 public:
  CorWriter(const std::string& path, const CorHeaderConfig& cfg, const CorStation& st1,
            const CorStation& st2);
  ~CorWriter();
  CorWriter(const CorWriter&) = delete;
  CorWriter& operator=(const CorWriter&) = delete;
  void write_sector(int64_t timestamp_unix_sec, float effective_integ_time_s,
                    const float* spectrum_re_im);
  void finalize();
  const std::string& path() const { return path_; }

 private:
  std::string path_;
  FILE* f_ = nullptr;
  int32_t fft_half_ = 0;
  int32_t sectors_ = 0;
};

// YYYYDDDhhmmss of a unix time (cor.rs:308-320, UTC, clamped to i32 range).
std::string unix_seconds_to_yyyydddhhmmss(int64_t unix_seconds);

}  // namespace yi
