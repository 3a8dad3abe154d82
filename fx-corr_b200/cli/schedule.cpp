// schedule.cpp — XML schedule reader (fx-corr src/xml.rs:66-348).
#include "schedule.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <set>
#include <sstream>
#include <stdexcept>

namespace yi {

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

bool ieq(const std::string& a, const std::string& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
  return true;
}

std::string decode_entities(const std::string& s) {
  std::string out;
  for (size_t i = 0; i < s.size(); ++i) {
    if (s[i] != '&') {
      out += s[i];
      continue;
    }
    const size_t semi = s.find(';', i);
    if (semi == std::string::npos) throw std::runtime_error("XML: unterminated entity");
    const std::string ent = s.substr(i + 1, semi - i - 1);
    if (ent == "lt") out += '<';
    else if (ent == "gt") out += '>';
    else if (ent == "amp") out += '&';
    else if (ent == "quot") out += '"';
    else if (ent == "apos") out += '\'';
    else if (!ent.empty() && ent[0] == '#') {
      const unsigned long cp = (ent.size() > 1 && (ent[1] == 'x' || ent[1] == 'X'))
                                   ? std::stoul(ent.substr(2), nullptr, 16)
                                   : std::stoul(ent.substr(1));
      if (cp < 0x80) {
        out += (char)cp;
      } else if (cp < 0x800) {
        out += (char)(0xC0 | (cp >> 6));
        out += (char)(0x80 | (cp & 0x3F));
      } else {
        out += (char)(0xE0 | (cp >> 12));
        out += (char)(0x80 | ((cp >> 6) & 0x3F));
        out += (char)(0x80 | (cp & 0x3F));
      }
    } else {
      throw std::runtime_error("XML: unknown entity &" + ent + ";");
    }
    i = semi;
  }
  return out;
}

double parse_f64(const std::string& s, const char* what) {
  size_t pos = 0;
  double v;
  try {
    v = std::stod(s, &pos);
  } catch (const std::exception&) {
    throw std::runtime_error(std::string("invalid float in ") + what + ": '" + s + "'");
  }
  if (pos != s.size()) throw std::runtime_error(std::string("invalid float in ") + what + ": '" + s + "'");
  return v;
}

bool try_f64(const std::string& s, double* v) {
  try {
    *v = parse_f64(s, "");
    return true;
  } catch (const std::exception&) {
    return false;
  }
}

size_t parse_usize(const std::string& s, const char* what) {
  if (s.empty() || !std::all_of(s.begin(), s.end(), [](char c) { return std::isdigit((unsigned char)c) || c == '+'; }))
    throw std::runtime_error(std::string("invalid integer in ") + what + ": '" + s + "'");
  return (size_t)std::stoull(s);
}

}  // namespace

const XmlNode* XmlNode::child(const std::string& t) const {
  for (const auto& c : children)
    if (ieq(c->tag, t)) return c.get();
  return nullptr;
}

std::optional<std::string> XmlNode::child_text(const std::string& t) const {
  const XmlNode* c = child(t);
  if (!c) return std::nullopt;
  return trim(c->text);
}

std::optional<std::string> XmlNode::attr(const std::string& name) const {
  auto it = attrs.find(name);
  if (it == attrs.end()) return std::nullopt;
  return it->second;
}

void XmlNode::descendants(std::vector<const XmlNode*>& out) const {
  out.push_back(this);
  for (const auto& c : children) c->descendants(out);
}

std::unique_ptr<XmlNode> parse_xml(const std::string& src) {
  auto root = std::make_unique<XmlNode>();
  root->tag = "#document";
  std::vector<XmlNode*> stack{root.get()};
  size_t i = 0;
  if (src.compare(0, 3, "\xEF\xBB\xBF") == 0) i = 3;
  auto add_text = [&](const std::string& t) {
    XmlNode* cur = stack.back();
    if (cur->children.empty()) cur->text += t;
  };
  while (i < src.size()) {
    if (src[i] != '<') {
      const size_t lt = src.find('<', i);
      const size_t end = lt == std::string::npos ? src.size() : lt;
      add_text(decode_entities(src.substr(i, end - i)));
      i = end;
      continue;
    }
    if (src.compare(i, 4, "<!--") == 0) {
      const size_t e = src.find("-->", i + 4);
      if (e == std::string::npos) throw std::runtime_error("XML: unterminated comment");
      i = e + 3;
    } else if (src.compare(i, 9, "<![CDATA[") == 0) {
      const size_t e = src.find("]]>", i + 9);
      if (e == std::string::npos) throw std::runtime_error("XML: unterminated CDATA");
      add_text(src.substr(i + 9, e - i - 9));
      i = e + 3;
    } else if (src.compare(i, 2, "<?") == 0) {
      const size_t e = src.find("?>", i + 2);
      if (e == std::string::npos) throw std::runtime_error("XML: unterminated declaration");
      i = e + 2;
    } else if (src.compare(i, 2, "<!") == 0) {
      const size_t e = src.find('>', i + 2);
      if (e == std::string::npos) throw std::runtime_error("XML: unterminated markup");
      i = e + 1;
    } else if (src.compare(i, 2, "</") == 0) {
      const size_t e = src.find('>', i + 2);
      if (e == std::string::npos) throw std::runtime_error("XML: unterminated end tag");
      const std::string name = trim(src.substr(i + 2, e - i - 2));
      if (stack.size() < 2 || stack.back()->tag != name)
        throw std::runtime_error("XML: mismatched end tag </" + name + ">");
      stack.pop_back();
      i = e + 1;
    } else {
      size_t j = i + 1;
      while (j < src.size() && !std::isspace((unsigned char)src[j]) && src[j] != '>' &&
             src[j] != '/')
        ++j;
      auto node = std::make_unique<XmlNode>();
      node->tag = src.substr(i + 1, j - i - 1);
      if (node->tag.empty()) throw std::runtime_error("XML: empty tag name");
      bool self_close = false;
      for (;;) {
        while (j < src.size() && std::isspace((unsigned char)src[j])) ++j;
        if (j >= src.size()) throw std::runtime_error("XML: unterminated start tag");
        if (src[j] == '>') {
          ++j;
          break;
        }
        if (src.compare(j, 2, "/>") == 0) {
          self_close = true;
          j += 2;
          break;
        }
        size_t k = j;
        while (k < src.size() && src[k] != '=' && !std::isspace((unsigned char)src[k])) ++k;
        const std::string an = src.substr(j, k - j);
        while (k < src.size() && std::isspace((unsigned char)src[k])) ++k;
        if (k >= src.size() || src[k] != '=') throw std::runtime_error("XML: attribute without value");
        ++k;
        while (k < src.size() && std::isspace((unsigned char)src[k])) ++k;
        if (k >= src.size() || (src[k] != '"' && src[k] != '\''))
          throw std::runtime_error("XML: unquoted attribute value");
        const char q = src[k];
        const size_t e = src.find(q, k + 1);
        if (e == std::string::npos) throw std::runtime_error("XML: unterminated attribute value");
        node->attrs[an] = decode_entities(src.substr(k + 1, e - k - 1));
        j = e + 1;
      }
      XmlNode* raw = node.get();
      stack.back()->children.push_back(std::move(node));
      if (!self_close) stack.push_back(raw);
      i = j;
    }
  }
  if (stack.size() != 1) throw std::runtime_error("XML: unclosed element <" + stack.back()->tag + ">");
  return root;
}

Schedule parse_xml_schedule(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot read " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  const auto doc = parse_xml(ss.str());
  std::vector<const XmlNode*> all;
  doc->descendants(all);
  auto tagged = [&](const char* t) {
    std::vector<const XmlNode*> v;
    for (auto* n : all)
      if (ieq(n->tag, t)) v.push_back(n);
    return v;
  };
  Schedule d;
  const auto procs = tagged("process");
  if (procs.empty()) throw std::runtime_error("process node not found in XML schedule");
  const XmlNode* process = procs[0];
  for (auto* p : procs)
    if (auto e = p->child_text("epoch")) d.process_epochs.push_back(*e);
  d.source = process->child_text("object");
  d.epoch = process->child_text("epoch");
  if (auto s = process->child_text("skip"); s && !s->empty()) d.process_skip_sec = parse_f64(*s, "process/skip");
  if (auto s = process->child_text("length"); s && !s->empty())
    d.process_length_sec = parse_f64(*s, "process/length");

  std::map<std::string, const XmlNode*> station_by_key;
  for (auto* n : tagged("station"))
    if (auto k = n->attr("key")) station_by_key[trim(*k)] = n;
  // pick_ant_keys (xml.rs:44-64)
  std::string k1, k2;
  bool picked = false;
  if (auto st = process->child_text("stations")) {
    std::vector<std::string> keys;
    for (char c : *st)
      if (!std::isspace((unsigned char)c)) keys.emplace_back(1, c);
    if (keys.size() >= 2) {
      k1 = keys[0];
      k2 = keys[1];
      picked = true;
    }
  }
  if (!picked) {
    if (station_by_key.size() < 2)
      throw std::runtime_error("failed to determine ant1/ant2 station keys from XML");
    auto it = station_by_key.begin();
    k1 = it->first;
    k2 = (++it)->first;
  }
  auto find_station = [&](const std::string& k) {
    auto it = station_by_key.find(k);
    if (it == station_by_key.end()) throw std::runtime_error("station key '" + k + "' not found");
    return it->second;
  };
  const XmlNode* st1 = find_station(k1);
  const XmlNode* st2 = find_station(k2);
  d.ant1_station_name = st1->child_text("name");
  d.ant2_station_name = st2->child_text("name");
  auto ecef = [](const XmlNode* n) -> std::optional<std::vector<double>> {
    auto x = n->child_text("pos-x"), y = n->child_text("pos-y"), z = n->child_text("pos-z");
    std::optional<double> xv, yv, zv;
    if (x && !x->empty()) xv = parse_f64(*x, "pos-x");
    if (y && !y->empty()) yv = parse_f64(*y, "pos-y");
    if (z && !z->empty()) zv = parse_f64(*z, "pos-z");
    if (xv && yv && zv) return std::vector<double>{*xv, *yv, *zv};
    return std::nullopt;
  };
  d.ant1_ecef_m = ecef(st1);
  d.ant2_ecef_m = ecef(st2);

  std::map<std::string, const XmlNode*> terminal_by_name;
  for (auto* n : tagged("terminal"))
    if (auto nm = n->attr("name")) terminal_by_name[trim(*nm)] = n;
  auto term_of = [&](const XmlNode* st) -> const XmlNode* {
    auto t = st->child_text("terminal");
    if (!t) return nullptr;
    auto it = terminal_by_name.find(*t);
    return it == terminal_by_name.end() ? nullptr : it->second;
  };
  const XmlNode* t1 = term_of(st1);
  const XmlNode* t2 = term_of(st2);
  std::optional<std::string> speed;
  if (t1) speed = t1->child_text("speed");
  if (!speed && t2) speed = t2->child_text("speed");
  if (speed) d.sampling_hz = parse_f64(*speed, "terminal/speed");
  if (t1)
    if (auto b = t1->child_text("bit")) d.ant1_bit = parse_usize(*b, "terminal/bit");
  if (t2)
    if (auto b = t2->child_text("bit")) d.ant2_bit = parse_usize(*b, "terminal/bit");
  if (t1) d.ant1_level = t1->child_text("level");
  if (t2) d.ant2_level = t2->child_text("level");

  std::map<std::string, std::string> shuffle_by_key;
  for (auto* n : tagged("shuffle"))
    if (auto k = n->attr("key")) shuffle_by_key[trim(*k)] = trim(n->text);
  if (shuffle_by_key.count(k1)) d.ant1_shuffle = shuffle_by_key[k1];
  if (shuffle_by_key.count(k2)) d.ant2_shuffle = shuffle_by_key[k2];

  const auto streams = tagged("stream");
  if (streams.empty()) throw std::runtime_error("stream node not found in XML schedule");
  const XmlNode* stream = streams[0];
  d.stream_label = stream->child_text("label");
  auto fq = stream->child_text("frequency");
  if (!fq) throw std::runtime_error("stream/frequency missing");
  const double frequency_hz = parse_f64(*fq, "stream/frequency");
  d.obsfreq_mhz = std::fabs(frequency_hz) / 1e6;
  if (auto f = stream->child_text("fft")) d.fft = parse_usize(*f, "stream/fft");
  const std::string default_sb = frequency_hz < 0.0 ? "LSB" : "USB";
  std::map<std::string, const XmlNode*> special_by_key;
  for (const auto& c : stream->children)
    if (ieq(c->tag, "special"))
      if (auto k = c->attr("key")) special_by_key[trim(*k)] = c.get();
  auto special = [&](const std::string& k) -> const XmlNode* {
    auto it = special_by_key.find(k);
    return it == special_by_key.end() ? nullptr : it->second;
  };
  auto upper = [](std::string s) {
    for (auto& c : s) c = (char)std::toupper((unsigned char)c);
    return s;
  };
  const XmlNode* sp1 = special(k1);
  const XmlNode* sp2 = special(k2);
  d.ant1_sideband = upper((sp1 && sp1->child_text("sideband")) ? *sp1->child_text("sideband") : default_sb);
  d.ant2_sideband = upper((sp2 && sp2->child_text("sideband")) ? *sp2->child_text("sideband") : default_sb);
  if (sp1)
    if (auto r = sp1->child_text("rotation"); r && !r->empty()) d.ant1_rotation_hz = parse_f64(*r, "rotation");
  if (sp2)
    if (auto r = sp2->child_text("rotation"); r && !r->empty()) d.ant2_rotation_hz = parse_f64(*r, "rotation");

  struct Clock {
    double delay = 0.0, rate = 0.0;
    std::optional<std::string> epoch;
  };
  std::map<std::string, Clock> clock_by_key;
  for (auto* n : tagged("clock")) {
    auto k = n->attr("key");
    if (!k) continue;
    Clock c;
    if (auto v = n->child_text("delay")) try_f64(*v, &c.delay);
    if (auto v = n->child_text("rate")) try_f64(*v, &c.rate);
    c.epoch = n->child_text("epoch");
    clock_by_key[trim(*k)] = c;
  }
  const Clock c1 = clock_by_key.count(k1) ? clock_by_key[k1] : Clock{};
  const Clock c2 = clock_by_key.count(k2) ? clock_by_key[k2] : Clock{};
  d.clock_delay_s = c2.delay - c1.delay;
  d.clock_rate_sps = c2.rate - c1.rate;
  d.ant1_clock_delay_s = c1.delay;
  d.ant2_clock_delay_s = c2.delay;
  d.ant1_clock_rate_sps = c1.rate;
  d.ant2_clock_rate_sps = c2.rate;
  d.ant1_clock_epoch = c1.epoch;
  d.ant2_clock_epoch = c2.epoch;

  const auto sources = tagged("source");
  const XmlNode* src = nullptr;
  if (d.source)
    for (auto* n : sources)
      if (auto nm = n->attr("name"); nm && trim(*nm) == *d.source) {
        src = n;
        break;
      }
  if (!src && !sources.empty()) src = sources[0];
  if (!src) throw std::runtime_error("source node not found in XML schedule");
  auto ra = src->child_text("ra");
  if (!ra) throw std::runtime_error("source/ra missing");
  auto dec = src->child_text("dec");
  if (!dec) throw std::runtime_error("source/dec missing");
  d.ra = *ra;
  d.dec = *dec;
  std::map<std::string, std::pair<std::string, std::string>> radec_by_name;
  for (auto* n : sources) {
    auto nm = n->attr("name");
    auto r = n->child_text("ra"), dc = n->child_text("dec");
    if (nm && r && dc) radec_by_name[trim(*nm)] = {*r, *dc};
  }
  for (auto* p : procs) {
    ProcessEntry e;
    e.epoch = p->child_text("epoch") ? *p->child_text("epoch") : std::string("2000");
    if (auto s = p->child_text("skip")) try_f64(*s, &e.skip_sec);
    if (auto s = p->child_text("length")) {
      double v;
      if (try_f64(*s, &v)) e.length_sec = v;
    }
    e.object = p->child_text("object");
    if (auto s = p->child_text("fft"); s && !s->empty()) e.fft = parse_usize(trim(*s), "process/fft");
    if (auto s = p->child_text("bit"); s && !s->empty()) e.bit = parse_usize(trim(*s), "process/bit");
    if (auto s = p->child_text("level"); s && !s->empty()) e.level = trim(*s);
    e.stations = p->child_text("stations");
    if (e.stations) {
      std::string stn;
      for (char c : *e.stations)
        if (!std::isspace((unsigned char)c)) stn += c;
      if (stn.find(k1) == std::string::npos || stn.find(k2) == std::string::npos) continue;
    }
    if (e.object) {
      auto it = radec_by_name.find(*e.object);
      if (it != radec_by_name.end()) {
        e.ra = it->second.first;
        e.dec = it->second.second;
      }
    }
    d.processes.push_back(e);
  }
  if (d.sampling_hz) {
    const double bw = *d.sampling_hz / 2e6;
    d.ant1_bw_mhz = bw;
    d.ant2_bw_mhz = bw;
    d.ant1_center_mhz = *d.obsfreq_mhz + d.ant1_rotation_hz.value_or(0.0) / 1e6 + 0.5 * bw;
    d.ant2_center_mhz = *d.obsfreq_mhz + d.ant2_rotation_hz.value_or(0.0) / 1e6 + 0.5 * bw;
  }
  d.ant1_station_key = k1;
  d.ant2_station_key = k2;
  return d;
}

void write_example_xml(const std::string& path) {
  std::ofstream f(path);
  if (!f) throw std::runtime_error("cannot create " + path);
  f << "<?xml version=\"1.0\" encoding=\"UTF-8\"?>\n"
       "<!-- Observation schedule for yi-corr / yi-acf / yi-xcf / yi-phasedarray. -->\n"
       "<schedule>\n"
       "  <!-- one <station> per antenna; key is a single character -->\n"
       "  <station key=\"A\"><name>ANT1</name><pos-x>-3502544.587</pos-x>"
       "<pos-y>+3950966.235</pos-y><pos-z>+3566381.192</pos-z><terminal>term1</terminal></station>\n"
       "  <station key=\"B\"><name>ANT2</name><pos-x>-3502567.576</pos-x>"
       "<pos-y>+3950885.734</pos-y><pos-z>+3566449.115</pos-z><terminal>term2</terminal></station>\n"
       "  <!-- clock delay [s] and rate [s/s], optionally referenced to an <epoch> -->\n"
       "  <clock key=\"A\"><delay>0</delay><rate>0</rate></clock>\n"
       "  <clock key=\"B\"><delay>0</delay><rate>0</rate></clock>\n"
       "  <!-- sampler: rate [Hz], bits per sample, level of each code -->\n"
       "  <terminal name=\"term1\"><speed>1024000000</speed><channel>1</channel><bit>2</bit>"
       "<level>-1.5,-0.5,+0.5,+1.5</level></terminal>\n"
       "  <terminal name=\"term2\"><speed>1024000000</speed><channel>1</channel><bit>2</bit>"
       "<level>-1.5,-0.5,+0.5,+1.5</level></terminal>\n"
       "  <!-- 32-entry bit order of each recorded word, most significant first -->\n"
       "  <shuffle key=\"A\">31,30,29,28,27,26,25,24,23,22,21,20,19,18,17,16,15,14,13,12,11,10,"
       "9,8,7,6,5,4,3,2,1,0</shuffle>\n"
       "  <shuffle key=\"B\">31,30,29,28,27,26,25,24,23,22,21,20,19,18,17,16,15,14,13,12,11,10,"
       "9,8,7,6,5,4,3,2,1,0</shuffle>\n"
       "  <source name=\"TARGET\"><ra>00h00m00.00000</ra><dec>+00d00'00.0000</dec></source>\n"
       "  <!-- observing frequency [Hz] (set it: rates are divided by it), FFT length, per-antenna"
       " rotation [Hz] and sideband -->\n"
       "  <stream>\n"
       "    <frequency>8400000000</frequency>\n"
       "    <fft>16384</fft>\n"
       "    <special key=\"A\"><rotation>0</rotation><sideband>LSB</sideband></special>\n"
       "    <special key=\"B\"><rotation>0</rotation><sideband>LSB</sideband></special>\n"
       "  </stream>\n"
       "  <process><epoch>2000/001 00:00:00</epoch><length>1</length><object>TARGET</object>"
       "<stations>AB</stations></process>\n"
       "</schedule>\n";
}

}  // namespace yi
