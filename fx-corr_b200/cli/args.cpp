// args.cpp — see args.h.
#include "args.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <sstream>

namespace yi {

namespace {

constexpr double kBoltzmann = 1.380649e-23;  // J/K (args.rs:6)
constexpr double kSiToJy = 1.0e26;           // args.rs:7
constexpr double kPi = 3.14159265358979323846;

enum class Kind { Flag, One, Many };

struct Spec {
  std::string name;                  // long name
  std::vector<std::string> aliases;  // visible aliases
  Kind kind;
  bool hyphen_values = false;        // allow_hyphen_values
  bool negative_numbers = false;     // allow_negative_numbers
  size_t max_values = 1000000;       // num_args upper bound (Many)
  std::string value_name;
  std::string help;
  bool hidden = false;
  std::function<void(Args&, const std::vector<std::string>&)> set;
};

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

bool is_number(const std::string& s) {
  if (s.empty()) return false;
  try {
    parse_f64(s);
    return true;
  } catch (...) {
    return false;
  }
}

std::vector<Spec> specs() {
  std::vector<Spec> v;
  auto one_s = [](std::optional<std::string> Args::*m) {
    return [m](Args& a, const std::vector<std::string>& x) { a.*m = x[0]; };
  };
  auto one_f = [](double Args::*m) {
    return [m](Args& a, const std::vector<std::string>& x) { a.*m = parse_f64(x[0]); };
  };
  auto opt_f = [](std::optional<double> Args::*m) {
    return [m](Args& a, const std::vector<std::string>& x) { a.*m = parse_f64(x[0]); };
  };
  auto opt_u = [](std::optional<size_t> Args::*m) {
    return [m](Args& a, const std::vector<std::string>& x) { a.*m = parse_usize(x[0]); };
  };
  auto many = [](std::vector<std::string> Args::*m) {
    return [m](Args& a, const std::vector<std::string>& x) {
      (a.*m).insert((a.*m).end(), x.begin(), x.end());
    };
  };
  auto flag = [](bool Args::*m) {
    return [m](Args& a, const std::vector<std::string>&) { a.*m = true; };
  };
  v.push_back({"schedule", {"sc"}, Kind::One, false, false, 1, "XML",
               "Observation schedule XML file (.xml)", false, one_s(&Args::schedule)});
  v.push_back({"mkxml", {}, Kind::Flag, false, false, 0, "",
               "Write example schedule XML to example.xml and exit", false, flag(&Args::mkxml)});
  v.push_back({"raw-directory", {"data", "raw"}, Kind::One, false, false, 1, "DIR",
               "Directory containing input raw files", false, one_s(&Args::raw_directory)});
  v.push_back({"ant1", {}, Kind::One, false, false, 1, "FILE", "Input raw file for antenna 1",
               false, one_s(&Args::ant1)});
  v.push_back({"ant2", {}, Kind::One, false, false, 1, "FILE", "Input raw file for antenna 2",
               false, one_s(&Args::ant2)});
  v.push_back({"cor-directory", {"output", "cor"}, Kind::One, false, false, 1, "DIR",
               "Directory for output .cor/.raw products", false, one_s(&Args::cor_directory)});
  v.push_back({"ra", {}, Kind::One, false, false, 1, "HMS",
               "Source right ascension (HHhMMmSS.s or degrees)", false, one_s(&Args::ra)});
  v.push_back({"dec", {}, Kind::One, true, false, 1, "DMS",
               "Source declination (DDdMMmSS.s or degrees)", false, one_s(&Args::dec)});
  v.push_back({"epoch", {}, Kind::One, false, false, 1, "YYYY/DDD HH:MM:SS",
               "Observation epoch (UTC)", false, one_s(&Args::epoch)});
  v.push_back({"obsfreq", {}, Kind::One, false, false, 1, "MHZ",
               "Reference observing frequency [MHz] [default: 0]", false, one_f(&Args::obsfreq)});
  v.push_back({"sampling", {}, Kind::One, false, false, 1, "MSPS",
               "Sampling rate [Msps] [default: 1024]", false, one_f(&Args::sampling)});
  v.push_back({"fft", {}, Kind::One, false, false, 1, "POINTS",
               "FFT size [samples/frame] [default: 16384]", false,
               [](Args& a, const std::vector<std::string>& x) { a.fft = parse_usize(x[0]); }});
  v.push_back({"bin", {"bit"}, Kind::Many, false, false, 1000000, "BITS",
               "Quantization bits per sample [bits] (e.g. \"2\" or \"ant1:2 ant2:4\")", false,
               many(&Args::bin)});
  v.push_back({"level", {}, Kind::Many, false, true, 1000000, "LEVEL",
               "Quantization levels [a.u.] (e.g. \"ant1:-1.5,0.5,-0.5,1.5\" or space-separated "
               "values)", false, many(&Args::level)});
  v.push_back({"shuffle", {}, Kind::Many, false, false, 32, "BIT",
               "Bit shuffle map [bit index] (e.g. \"ant1:31,30...0\" or 32 space-separated "
               "indices)", false, many(&Args::shuffle_in)});
  v.push_back({"sideband", {}, Kind::Many, false, false, 1000000, "LSB|USB",
               "Input sampler sideband [default: LSB]", false, many(&Args::sideband)});
  v.push_back({"coarse", {}, Kind::One, true, false, 1, "S", "Fixed coarse delay [s]", false,
               opt_f(&Args::coarse)});
  v.push_back({"delay", {}, Kind::One, true, false, 1, "SAMPLES",
               "Residual delay applied to ant2 [samples] [default: 0]", false,
               one_f(&Args::delay)});
  v.push_back({"rate", {}, Kind::One, true, false, 1, "HZ",
               "Residual fringe rate correction [Hz] [default: 0]", false, one_f(&Args::rate)});
  v.push_back({"resdelay", {}, Kind::One, true, false, 1, "SAMPLES",
               "Additional residual delay [samples] [default: 0]", false,
               one_f(&Args::resdelay)});
  v.push_back({"resrate", {}, Kind::One, true, false, 1, "HZ",
               "Additional residual rate [Hz] [default: 0]", false, one_f(&Args::resrate)});
  v.push_back({"rotation", {}, Kind::Many, true, false, 1000000, "HZ",
               "Per-antenna rotation frequency [Hz] (e.g. \"ant1:343000000 ant2:0\")", false,
               many(&Args::rotation)});
  v.push_back({"skip", {}, Kind::One, false, false, 1, "S",
               "Start offset from input head [s] [default: 0]", false, one_f(&Args::skip)});
  v.push_back({"length", {}, Kind::One, false, false, 1, "S", "Processing duration [s]", false,
               opt_f(&Args::length)});
  v.push_back({"tsys", {}, Kind::Many, false, false, 1000000, "K", "System temperature [K]",
               false, many(&Args::tsys)});
  v.push_back({"diameter", {}, Kind::Many, false, false, 1000000, "M", "Antenna diameter [m]",
               false, many(&Args::diameter)});
  v.push_back({"eta", {}, Kind::Many, false, false, 1000000, "RATIO",
               "Antenna aperture efficiency [0..1]", false, many(&Args::eta)});
  v.push_back({"gain", {}, Kind::Many, false, false, 1000000, "SCALE",
               "Per-antenna amplitude scale [a.u.]", false, many(&Args::gain)});
  v.push_back({"sefd", {}, Kind::Many, false, false, 1000000, "JY", "SEFD [Jy]", false,
               many(&Args::sefd)});
  v.push_back({"fringe", {}, Kind::Flag, false, false, 0, "",
               "Enable fringe search in yi-phasedarray mode only", false, flag(&Args::fringe)});
  v.push_back({"cpu", {}, Kind::One, false, false, 1, "N",
               "Number of host threads for reading and packing [default: logical CPU count - 2, "
               "min 1]", false, opt_u(&Args::cpu)});
  v.push_back({"chunk-frames", {}, Kind::One, false, false, 1, "N",
               "Reader chunk size [frames] (auto when omitted)", false,
               opt_u(&Args::chunk_frames)});
  v.push_back({"razoku5bay", {}, Kind::Flag, false, false, 0, "",
               "Force small I/O chunking at 0.5-second intervals (overrides --chunk-frames)",
               false, flag(&Args::razoku5bay)});
  v.push_back({"pipeline-depth", {}, Kind::One, false, false, 1, "N",
               "Reader-worker queue depth [chunks] (auto when omitted)", false,
               opt_u(&Args::pipeline_depth)});
  v.push_back({"jobs", {}, Kind::One, false, false, 1, "N",
               "Run up to N <process> entries of the schedule at once, their sectors computed "
               "together in batches on the GPU (this build's extension) [default: 1, one after "
               "another]", false, opt_u(&Args::jobs)});
  v.push_back({"debug", {}, Kind::Flag, false, false, 0, "",
               "Enable diagnostic debug logging to file (all frames)", false,
               flag(&Args::debug)});
  v.push_back({"stdout", {}, Kind::Flag, false, false, 0, "",
               "Write yi-corr runtime stdout log to ./stdout/stdout_<yyyydddhhmmss>.log", false,
               flag(&Args::stdout_log)});
  v.push_back({"process-index", {}, Kind::One, false, false, 1, "N", "", true,
               opt_u(&Args::process_index)});
  v.push_back({"delay-reference", {}, Kind::One, false, false, 1, "REF", "", true,
               [](Args& a, const std::vector<std::string>& x) {
                 if (x[0] != "ant1" && x[0] != "ant2")
                   throw ArgsExit("error: invalid value '" + x[0] +
                                      "' for '--delay-reference <REF>'\n  [possible values: "
                                      "ant1, ant2]",
                                  2);
                 a.delay_reference = x[0];
               }});
  v.push_back({"compact-logs", {}, Kind::Flag, false, false, 0, "", "", true,
               flag(&Args::compact_logs)});
  return v;
}

}  // namespace

double parse_f64(const std::string& s) {
  // Rust f64::from_str: [+-]? (digits [. digits?] | . digits) ([eE][+-]?digits)?, or
  // inf / infinity / nan in any case; nothing else (no spaces, no hex).
  const std::string l = lower(s);
  size_t i = 0;
  if (i < l.size() && (l[i] == '+' || l[i] == '-')) ++i;
  const std::string body = l.substr(i);
  if (body == "inf" || body == "infinity" || body == "nan") {
    const double v = body == "nan" ? NAN : INFINITY;
    return (i && l[0] == '-') ? -v : v;
  }
  size_t d0 = i;
  while (i < l.size() && std::isdigit((unsigned char)l[i])) ++i;
  size_t nd = i - d0;
  if (i < l.size() && l[i] == '.') {
    ++i;
    size_t f0 = i;
    while (i < l.size() && std::isdigit((unsigned char)l[i])) ++i;
    nd += i - f0;
  }
  if (nd == 0) throw std::runtime_error("invalid float literal");
  if (i < l.size() && l[i] == 'e') {
    ++i;
    if (i < l.size() && (l[i] == '+' || l[i] == '-')) ++i;
    size_t e0 = i;
    while (i < l.size() && std::isdigit((unsigned char)l[i])) ++i;
    if (i == e0) throw std::runtime_error("invalid float literal");
  }
  if (i != l.size()) throw std::runtime_error("invalid float literal");
  return std::strtod(s.c_str(), nullptr);
}

size_t parse_usize(const std::string& s) {
  size_t i = (!s.empty() && s[0] == '+') ? 1 : 0;
  if (i == s.size()) throw std::runtime_error("cannot parse integer from empty string");
  unsigned long long v = 0;
  for (; i < s.size(); ++i) {
    if (!std::isdigit((unsigned char)s[i])) throw std::runtime_error("invalid digit found in string");
    const unsigned long long d = (unsigned long long)(s[i] - '0');
    if (v > (~0ULL - d) / 10) throw std::runtime_error("number too large to fit in target type");
    v = v * 10 + d;
  }
  return (size_t)v;
}

std::string help_text(const std::string& prog) {
  std::ostringstream o;
  o << "yi toolkit for FX correlation and phased-array processing\n\n"
    << "yi-acf: auto-correlation only\nyi-xcf: cross-correlation only\n"
    << "yi-corr: auto + cross correlation\nyi-phasedarray: phased-array synthesis and spectrum "
       "plots\n\n"
    << "Usage: " << prog << " [OPTIONS]\n\nOptions:\n";
  for (const auto& s : specs()) {
    if (s.hidden) continue;
    std::string left = "      --" + s.name;
    if (s.kind != Kind::Flag) left += " <" + s.value_name + ">" + (s.kind == Kind::Many ? "..." : "");
    o << left;
    if (left.size() < 40) o << std::string(40 - left.size(), ' ');
    else o << "\n" << std::string(40, ' ');
    o << s.help;
    if (!s.aliases.empty()) {
      o << " [aliases: ";
      for (size_t k = 0; k < s.aliases.size(); ++k) o << (k ? ", --" : "--") << s.aliases[k];
      o << "]";
    }
    o << "\n";
  }
  o << "  -h, --help                            Print help\n"
    << "  -V, --version                         Print version\n";
  return o.str();
}

Args parse_args(int argc, char** argv, const std::string& prog) {
  const std::vector<Spec> sp = specs();
  std::vector<std::string> tok(argv + 1, argv + argc);
  if (tok.empty()) throw ArgsExit(help_text(prog), 2);  // arg_required_else_help
  Args a;
  std::vector<bool> seen(sp.size(), false);
  auto find = [&](const std::string& name) -> int {
    // exact long name or alias, else a unique prefix of them (infer_long_args)
    for (size_t k = 0; k < sp.size(); ++k) {
      if (sp[k].name == name) return (int)k;
      for (const auto& al : sp[k].aliases)
        if (al == name) return (int)k;
    }
    int hit = -1;
    std::vector<std::string> cands;
    for (size_t k = 0; k < sp.size(); ++k) {
      if (sp[k].hidden) continue;
      bool m = sp[k].name.compare(0, name.size(), name) == 0;
      for (const auto& al : sp[k].aliases) m = m || al.compare(0, name.size(), name) == 0;
      if (m) {
        cands.push_back(sp[k].name);
        hit = (int)k;
      }
    }
    if (cands.size() > 1) {
      std::string msg = "error: unexpected argument '--" + name + "' found\n\n  tip: '--" + name +
                        "' matches more than one argument:";
      for (const auto& c : cands) msg += " --" + c;
      throw ArgsExit(msg, 2);
    }
    return cands.empty() ? -1 : hit;
  };
  auto is_flag_token = [&](const std::string& t) {
    if (t.size() < 2 || t[0] != '-') return false;
    if (t == "--") return true;
    if (t[1] != '-') return true;  // short options (-h, -V)
    return true;
  };
  for (size_t i = 0; i < tok.size(); ++i) {
    const std::string& t = tok[i];
    if (t == "-h" || t == "--help") throw ArgsExit(help_text(prog), 0);
    if (t == "-V" || t == "--version") throw ArgsExit(prog + " 0.1.0", 0);
    if (t.size() < 3 || t[0] != '-' || t[1] != '-')
      throw ArgsExit("error: unexpected argument '" + t + "' found\n\nUsage: " + prog +
                         " [OPTIONS]\n\nFor more information, try '--help'.",
                     2);
    std::string name = t.substr(2);
    std::optional<std::string> inline_val;
    const size_t eq = name.find('=');
    if (eq != std::string::npos) {
      inline_val = name.substr(eq + 1);
      name = name.substr(0, eq);
    }
    const int k = find(name);
    if (k < 0)
      throw ArgsExit("error: unexpected argument '--" + name + "' found\n\nUsage: " + prog +
                         " [OPTIONS]\n\nFor more information, try '--help'.",
                     2);
    const Spec& s = sp[(size_t)k];
    const std::string disp =
        "--" + s.name + (s.kind == Kind::Flag ? "" : " <" + s.value_name + ">" +
                                                        (s.kind == Kind::Many ? "..." : ""));
    if (s.kind != Kind::Many && seen[(size_t)k])
      throw ArgsExit("error: the argument '" + disp + "' cannot be used multiple times", 2);
    seen[(size_t)k] = true;
    std::vector<std::string> vals;
    if (s.kind == Kind::Flag) {
      if (inline_val)
        throw ArgsExit("error: unexpected value '" + *inline_val + "' for '--" + s.name +
                           "' found; no more were expected",
                       2);
    } else {
      auto value_ok = [&](const std::string& v) {
        if (v.empty() || v[0] != '-' || v == "-") return true;
        if (v == "--") return false;
        if (s.hyphen_values) {
          // a known long flag still ends the values
          if (v.size() > 2 && v[1] == '-') {
            std::string nm = v.substr(2);
            const size_t e2 = nm.find('=');
            if (e2 != std::string::npos) nm = nm.substr(0, e2);
            try {
              if (find(nm) >= 0) return false;
            } catch (const ArgsExit&) {
              return false;
            }
          }
          return true;
        }
        return s.negative_numbers && is_number(v);
      };
      if (inline_val) {
        vals.push_back(*inline_val);
      } else {
        while (i + 1 < tok.size() && vals.size() < (s.kind == Kind::Many ? s.max_values : 1) &&
               value_ok(tok[i + 1])) {
          vals.push_back(tok[++i]);
          if (s.kind == Kind::One) break;
        }
      }
      if (vals.empty())
        throw ArgsExit("error: a value is required for '" + disp + "' but none was supplied", 2);
    }
    (void)is_flag_token;
    try {
      s.set(a, vals);
    } catch (const ArgsExit&) {
      throw;
    } catch (const std::exception& e) {
      throw ArgsExit("error: invalid value '" + (vals.empty() ? std::string() : vals[0]) +
                         "' for '" + disp + "': " + e.what(),
                     2);
    }
  }
  if (a.sideband.empty()) a.sideband = {"LSB"};  // default_value = "LSB"
  return a;
}

namespace {

template <class T>
std::pair<T, T> per_antenna(const std::vector<std::string>& list, T dflt,
                            const std::function<T(const std::string&)>& parse) {
  T v1 = dflt, v2 = dflt;
  auto trim = [](const std::string& s) {
    size_t x = 0, y = s.size();
    while (x < y && std::isspace((unsigned char)s[x])) ++x;
    while (y > x && std::isspace((unsigned char)s[y - 1])) --y;
    return s.substr(x, y - x);
  };
  for (const auto& entry : list) {
    if (entry.find("ant1:") != std::string::npos || entry.find("ant2:") != std::string::npos) {
      std::vector<std::string> parts;
      std::string cur;
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
        if (part.rfind("ant1:", 0) == 0) v1 = parse(trim(part.substr(5)));
        else if (part.rfind("ant2:", 0) == 0) v2 = parse(trim(part.substr(5)));
        else {
          const T v = parse(trim(part));
          v1 = v;
          v2 = v;
        }
      }
    } else {
      const T v = parse(trim(entry));
      v1 = v;
      v2 = v;
    }
  }
  return {v1, v2};
}

}  // namespace

std::pair<std::string, std::string> per_antenna_str(const std::vector<std::string>& list,
                                                    const std::string& dflt, bool uppercase) {
  return per_antenna<std::string>(list, dflt, [uppercase](const std::string& s) {
    std::string r = s;
    if (uppercase)
      for (auto& c : r) c = (char)std::toupper((unsigned char)c);
    return r;
  });
}

std::pair<double, double> per_antenna_f64(const std::vector<std::string>& list, double dflt) {
  return per_antenna<double>(list, dflt, [](const std::string& s) { return parse_f64(s); });
}

std::pair<size_t, size_t> per_antenna_usize(const std::vector<std::string>& list, size_t dflt) {
  return per_antenna<size_t>(list, dflt, [](const std::string& s) { return parse_usize(s); });
}

std::vector<double> parse_levels(size_t bit, const std::string& list) {
  if (bit == 0) throw std::runtime_error("Bit depth must be at least 1");
  if (bit >= 63) throw std::runtime_error("Bit depth too large");
  const size_t expected = (size_t)1 << bit;
  std::vector<double> lv;
  std::string cur;
  std::istringstream is(list);
  while (std::getline(is, cur, ',')) {
    size_t x = 0, y = cur.size();
    while (x < y && std::isspace((unsigned char)cur[x])) ++x;
    while (y > x && std::isspace((unsigned char)cur[y - 1])) --y;
    lv.push_back(parse_f64(cur.substr(x, y - x)));
  }
  if (!list.empty() && list.back() == ',') lv.push_back(parse_f64(""));  // trailing empty item
  if (list.empty()) lv.push_back(parse_f64(""));
  if (lv.size() != expected)
    throw std::runtime_error("Expected " + std::to_string(expected) + " levels, received " +
                             std::to_string(lv.size()));
  return lv;
}

std::vector<int> parse_shuffle_internal(const std::string& list) {
  std::vector<size_t> ext;
  std::string cur;
  std::istringstream is(list);
  while (std::getline(is, cur, ',')) {
    size_t x = 0, y = cur.size();
    while (x < y && std::isspace((unsigned char)cur[x])) ++x;
    while (y > x && std::isspace((unsigned char)cur[y - 1])) --y;
    ext.push_back(parse_usize(cur.substr(x, y - x)));
  }
  if (!list.empty() && list.back() == ',') ext.push_back(parse_usize(""));
  if (ext.size() != 32) throw std::runtime_error("Shuffle map must contain exactly 32 entries");
  std::vector<size_t> sorted = ext;
  std::sort(sorted.begin(), sorted.end());
  for (size_t k = 0; k < 32; ++k)
    if (sorted[k] != k) throw std::runtime_error("Shuffle map must be a permutation of 0..31");
  std::vector<int> internal(32, 0);
  for (size_t idx = 0; idx < 32; ++idx) internal[31 - idx] = (int)ext[idx];
  return internal;
}

std::vector<std::string> normalize_level_args(const std::vector<std::string>& a, size_t b1,
                                              size_t b2) {
  if (a.empty()) return a;
  for (const auto& v : a)
    if (v.find("ant1:") != std::string::npos || v.find("ant2:") != std::string::npos) return a;
  if (b1 != b2) return a;
  const size_t expected = (size_t)1 << b1;
  const bool all_numeric = std::all_of(a.begin(), a.end(), [](const std::string& v) {
    try {
      parse_f64(v);
      return true;
    } catch (...) {
      return false;
    }
  });
  if (all_numeric) {
    if (a.size() != expected)
      throw std::runtime_error("--level without ant1:/ant2: must provide exactly " +
                               std::to_string(expected) + " values for --bin " +
                               std::to_string(b1));
    std::string j;
    for (size_t k = 0; k < a.size(); ++k) j += (k ? "," : "") + a[k];
    return {j};
  }
  return a;
}

std::vector<std::string> normalize_shuffle_args(const std::vector<std::string>& a) {
  if (a.empty()) return a;
  for (const auto& v : a)
    if (v.find("ant1:") != std::string::npos || v.find("ant2:") != std::string::npos) return a;
  const bool all_numeric = std::all_of(a.begin(), a.end(), [](const std::string& v) {
    try {
      parse_usize(v);
      return true;
    } catch (...) {
      return false;
    }
  });
  if (all_numeric) {
    if (a.size() != 32)
      throw std::runtime_error("--shuffle without ant1:/ant2: must provide exactly 32 values");
    std::string j;
    for (size_t k = 0; k < a.size(); ++k) j += (k ? "," : "") + a[k];
    return {j};
  }
  return a;
}

double resolve_weight(double tsys, double gain, std::optional<double> sefd,
                      std::optional<double> diameter, double eta, const std::string& label) {
  if (tsys == 0.0) throw std::runtime_error(label + " Tsys must be non-zero");
  if (sefd) {
    if (*sefd <= 0.0) throw std::runtime_error(label + " SEFD must be positive");
    return 1.0 / *sefd;
  }
  if (diameter) {
    if (*diameter <= 0.0 || eta <= 0.0)
      throw std::runtime_error(label + " diameter/eta must be positive");
    const double geom_area = kPi * std::pow(*diameter / 2.0, 2);
    const double eff_area = eta * geom_area;
    const double sefd_jy = (2.0 * kBoltzmann * tsys) / eff_area * kSiToJy;
    return 1.0 / sefd_jy;
  }
  if (gain <= 0.0) throw std::runtime_error(label + " gain must be positive");
  return gain / tsys;
}

}  // namespace yi
