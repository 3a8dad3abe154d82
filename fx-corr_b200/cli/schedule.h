// schedule.h — XML observation schedule (fx-corr src/xml.rs, src/ifile.rs).
#pragma once

#include <map>
#include <memory>
#include <optional>
#include <string>
#include <vector>

namespace yi {

// Minimal XML element tree: elements, attributes, text, comments, processing
// instructions, CDATA and the five predefined entities.
struct XmlNode {
  std::string tag;
  std::map<std::string, std::string> attrs;
  std::string text;  // text before the first child element (roxmltree Node::text)
  std::vector<std::unique_ptr<XmlNode>> children;
  const XmlNode* child(const std::string& tag_ci) const;  // first child, case-insensitive
  std::optional<std::string> child_text(const std::string& tag_ci) const;  // trimmed
  std::optional<std::string> attr(const std::string& name) const;
  void descendants(std::vector<const XmlNode*>& out) const;  // pre-order, self first
};

std::unique_ptr<XmlNode> parse_xml(const std::string& text);  // throws std::runtime_error

// ProcessEntry / IFileData (src/ifile.rs:22-63)
struct ProcessEntry {
  std::string epoch;
  double skip_sec = 0.0;
  std::optional<double> length_sec;
  std::optional<std::string> object, stations, ra, dec;
  // this build's extension (the reference has one <stream> fft and takes the
  // bit depth from the command line): per-process FFT length, bit depth of
  // both stations and level table
  std::optional<size_t> fft, bit;
  std::optional<std::string> level;
};

struct Schedule {
  std::string ra, dec;
  std::optional<std::string> epoch, source, stream_label;
  std::optional<size_t> fft;
  std::optional<double> sampling_hz;
  std::optional<size_t> ant1_bit, ant2_bit;
  std::optional<std::string> ant1_level, ant2_level, ant1_shuffle, ant2_shuffle;
  std::optional<double> obsfreq_mhz, clock_delay_s, clock_rate_sps;
  std::optional<double> ant1_clock_delay_s, ant2_clock_delay_s, ant1_clock_rate_sps,
      ant2_clock_rate_sps;
  std::optional<std::string> ant1_clock_epoch, ant2_clock_epoch;
  std::optional<std::string> ant1_sideband, ant2_sideband;
  std::optional<double> ant1_rotation_hz, ant2_rotation_hz;
  std::optional<double> ant1_center_mhz, ant2_center_mhz, ant1_bw_mhz, ant2_bw_mhz;
  std::optional<std::string> ant1_station_name, ant2_station_name, ant1_station_key,
      ant2_station_key;
  std::optional<std::vector<double>> ant1_ecef_m, ant2_ecef_m;
  std::vector<std::string> process_epochs;
  std::optional<double> process_skip_sec, process_length_sec;
  std::vector<ProcessEntry> processes;
};

// parse_xml_schedule (src/xml.rs:66-348)
Schedule parse_xml_schedule(const std::string& path);
// write_example_xml (src/xml.rs:350-424): the editable template
void write_example_xml(const std::string& path);

}  // namespace yi
