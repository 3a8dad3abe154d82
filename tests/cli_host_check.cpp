// cli_host_check.cpp — test driver for the yi-* tools' host logic (argument
// parsing, epochs and geometry, .cor headers, XML schedules), built by
// tests/test_cli_host.py from the cli sources without the GPU library.
// Usage: cli_host_check <command> [args...]; prints one result per line.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "args.h"
#include "cor_writer.h"
#include "geom.h"
#include "schedule.h"

using namespace yi;

static void hex(const uint8_t* b, size_t n) {
  for (size_t i = 0; i < n; ++i) std::printf("%02x", b[i]);
  std::printf("\n");
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string cmd = argv[1];
  try {
    if (cmd == "ra") {
      std::printf("%.17g\n", parse_ra(argv[2]));
    } else if (cmd == "dec") {
      std::printf("%.17g\n", parse_dec(argv[2]));
    } else if (cmd == "mjd") {
      std::printf("%.17g\n", parse_epoch_to_mjd(argv[2]));
    } else if (cmd == "unix") {
      std::printf("%" PRId64 "\n", epoch_to_unix_seconds(argv[2]));
    } else if (cmd == "tag") {
      std::printf("%s\n", unix_seconds_to_yyyydddhhmmss(std::stoll(argv[2])).c_str());
    } else if (cmd == "gmst") {
      std::printf("%.17g\n", gmst_rad(std::stod(argv[2])));
    } else if (cmd == "gast") {
      std::printf("%.17g\n", gast_rad(std::stod(argv[2])));
    } else if (cmd == "geodelay") {
      // x1 y1 z1 x2 y2 z2 ra_rad dec_rad mjd
      double a[3], b[3];
      for (int k = 0; k < 3; ++k) {
        a[k] = std::stod(argv[2 + k]);
        b[k] = std::stod(argv[5 + k]);
      }
      const GeomDelay g = geometric_delay_and_derivatives(a, b, std::stod(argv[8]),
                                                          std::stod(argv[9]), std::stod(argv[10]));
      std::printf("%.17g %.17g %.17g %.17g %.17g\n", g.delay1, g.delay2, g.delay, g.rate, g.accel);
    } else if (cmd == "precess") {
      double ra, dec;
      precess_j2000_to_mean_of_date(std::stod(argv[2]), std::stod(argv[3]), std::stod(argv[4]),
                                    &ra, &dec);
      std::printf("%.17g %.17g\n", ra, dec);
    } else if (cmd == "header") {
      CorHeaderConfig c;
      c.sampling_speed_hz = 1024000000;
      c.observing_frequency_hz = 8.4e9;
      c.fft_point = 8192;
      c.number_of_sector_hint = 10;
      c.clock_reference_unix_sec = 1707753120;
      c.source_name = "3C273";
      c.source_ra_rad = 3.25;
      c.source_dec_rad = 0.035;
      CorStation s1{"YAMAGU32", 'A', {-3502544.587, 3950966.235, 3566381.192}};
      CorStation s2{"YAMAGU34", 'B', {-3502567.576, 3950885.734, 3566449.115}};
      uint8_t h[256];
      build_cor_file_header(c, s1, s2, h);
      hex(h, 256);
    } else if (cmd == "sector") {
      uint8_t h[128];
      build_cor_sector_header(std::stoll(argv[2]), std::stof(argv[3]), h);
      hex(h, 128);
    } else if (cmd == "levels") {
      for (double v : parse_levels(std::stoul(argv[2]), argv[3])) std::printf("%.17g ", v);
      std::printf("\n");
    } else if (cmd == "shuffle") {
      for (int v : parse_shuffle_internal(argv[2])) std::printf("%d ", v);
      std::printf("\n");
    } else if (cmd == "perant") {  // default then entries
      std::vector<std::string> l(argv + 3, argv + argc);
      const auto p = per_antenna_str(l, argv[2]);
      std::printf("%s|%s\n", p.first.c_str(), p.second.c_str());
    } else if (cmd == "weight") {
      const double sefd = std::stod(argv[4]), dia = std::stod(argv[5]);
      std::printf("%.17g\n", resolve_weight(std::stod(argv[2]), std::stod(argv[3]),
                                            sefd > 0 ? std::optional<double>(sefd) : std::nullopt,
                                            dia > 0 ? std::optional<double>(dia) : std::nullopt,
                                            std::stod(argv[6]), "A1"));
    } else if (cmd == "args") {
      const Args a = parse_args(argc - 1, argv + 1, "yi-corr");
      auto join = [](const std::vector<std::string>& v) {
        std::string s;
        for (size_t i = 0; i < v.size(); ++i) s += (i ? ";" : "") + v[i];
        return s;
      };
      std::printf("schedule=%s\n", a.schedule ? a.schedule->c_str() : "-");
      std::printf("raw=%s\n", a.raw_directory ? a.raw_directory->c_str() : "-");
      std::printf("cor=%s\n", a.cor_directory ? a.cor_directory->c_str() : "-");
      std::printf("dec=%s\n", a.dec ? a.dec->c_str() : "-");
      std::printf("fft=%zu\n", a.fft);
      std::printf("sampling=%.17g\n", a.sampling);
      std::printf("bin=%s\n", join(a.bin).c_str());
      std::printf("level=%s\n", join(a.level).c_str());
      std::printf("sideband=%s\n", join(a.sideband).c_str());
      std::printf("rotation=%s\n", join(a.rotation).c_str());
      std::printf("delay=%.17g\n", a.delay);
      std::printf("coarse=%s\n", a.coarse ? std::to_string(*a.coarse).c_str() : "-");
      std::printf("mkxml=%d fringe=%d\n", (int)a.mkxml, (int)a.fringe);
    } else if (cmd == "mkxml") {
      write_example_xml(argv[2]);
    } else if (cmd == "xml") {
      const Schedule s = parse_xml_schedule(argv[2]);
      std::printf("ra=%s dec=%s\n", s.ra.c_str(), s.dec.c_str());
      std::printf("epoch=%s source=%s\n", s.epoch ? s.epoch->c_str() : "-",
                  s.source ? s.source->c_str() : "-");
      std::printf("fs=%.17g obs_mhz=%.17g fft=%zu\n", s.sampling_hz.value_or(-1),
                  s.obsfreq_mhz.value_or(-1), s.fft.value_or(0));
      std::printf("names=%s,%s keys=%s,%s\n", s.ant1_station_name.value_or("-").c_str(),
                  s.ant2_station_name.value_or("-").c_str(), s.ant1_station_key.value_or("-").c_str(),
                  s.ant2_station_key.value_or("-").c_str());
      std::printf("bits=%zu,%zu level=%s\n", s.ant1_bit.value_or(0), s.ant2_bit.value_or(0),
                  s.ant1_level.value_or("-").c_str());
      std::printf("sideband=%s,%s rot=%.17g,%.17g\n", s.ant1_sideband.value_or("-").c_str(),
                  s.ant2_sideband.value_or("-").c_str(), s.ant1_rotation_hz.value_or(-1),
                  s.ant2_rotation_hz.value_or(-1));
      std::printf("clock=%.17g,%.17g processes=%zu\n", s.ant1_clock_delay_s.value_or(-1),
                  s.ant2_clock_delay_s.value_or(-1), s.processes.size());
      for (const auto& p : s.processes)
        std::printf("process epoch=%s skip=%.17g length=%s fft=%s bit=%s level=%s\n",
                    p.epoch.c_str(), p.skip_sec,
                    p.length_sec ? std::to_string(*p.length_sec).c_str() : "-",
                    p.fft ? std::to_string(*p.fft).c_str() : "-",
                    p.bit ? std::to_string(*p.bit).c_str() : "-",
                    p.level ? p.level->c_str() : "-");
    } else {
      return 2;
    }
  } catch (const ArgsExit& e) {
    std::printf("ARGSEXIT %d %s\n", e.code, e.what());
  } catch (const std::exception& e) {
    std::printf("ERROR %s\n", e.what());
  }
  return 0;
}
