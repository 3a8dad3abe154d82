// args.h — command line of the yi-* tools (flags, aliases and value rules of
// fx-corr src/args.rs:23-170) and the per-antenna value helpers
// (src/args.rs:172-226, src/main.rs:389-434).
#pragma once

#include <cstddef>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace yi {

constexpr size_t kDefaultFft = 16384;  // args.rs:9

struct Args {
  std::optional<std::string> schedule;
  bool mkxml = false;
  std::optional<std::string> raw_directory, ant1, ant2, cor_directory;
  std::optional<std::string> ra, dec, epoch;
  double obsfreq = 0.0;
  double sampling = 1024.0;
  size_t fft = kDefaultFft;
  std::vector<std::string> bin, level, shuffle_in, sideband, rotation;
  std::optional<double> coarse;
  double delay = 0.0, rate = 0.0, resdelay = 0.0, resrate = 0.0;
  double skip = 0.0;
  std::optional<double> length;
  std::vector<std::string> tsys, diameter, eta, gain, sefd;
  bool fringe = false;
  std::optional<size_t> cpu, chunk_frames, pipeline_depth, process_index;
  std::optional<size_t> jobs;  // extension: <process> entries run at once
  bool razoku5bay = false, debug = false, stdout_log = false, compact_logs = false;
  std::string delay_reference = "ant2";
};

// Usage error: message for stderr, exit status 2; `help` is a --help/--version
// request (print message, exit 0).
struct ArgsExit : std::runtime_error {
  int code;
  explicit ArgsExit(const std::string& m, int c) : std::runtime_error(m), code(c) {}
};

// Parses argv[1..] (clap rules: --name value / --name=value, unique prefixes
// of long names, visible aliases, multi-value flags, hyphen-value rules).
// Throws ArgsExit.
Args parse_args(int argc, char** argv, const std::string& prog);
std::string help_text(const std::string& prog);

// resolve_per_antenna_config (args.rs:172-192) for the three value types used.
std::pair<std::string, std::string> per_antenna_str(const std::vector<std::string>& list,
                                                    const std::string& dflt,
                                                    bool uppercase = false);
std::pair<double, double> per_antenna_f64(const std::vector<std::string>& list, double dflt);
std::pair<size_t, size_t> per_antenna_usize(const std::vector<std::string>& list, size_t dflt);

// parse_levels (args.rs:194-200) / parse_shuffle (args.rs:202-210): throw
// std::runtime_error with the reference's messages.
std::vector<double> parse_levels(size_t bit, const std::string& list);
std::vector<int> parse_shuffle_internal(const std::string& list);  // internal[31-i] = ext[i]
// normalize_level_args / normalize_shuffle_args (main.rs:389-434)
std::vector<std::string> normalize_level_args(const std::vector<std::string>& a, size_t b1,
                                              size_t b2);
std::vector<std::string> normalize_shuffle_args(const std::vector<std::string>& a);

// resolve_weight (args.rs:212-226): (weight, ...) of a station.
double resolve_weight(double tsys, double gain, std::optional<double> sefd,
                      std::optional<double> diameter, double eta, const std::string& label);

// Rust-compatible number parsing (f64::from_str / usize::from_str).
double parse_f64(const std::string& s);
size_t parse_usize(const std::string& s);

}  // namespace yi
