// Oracle (test infrastructure only): shared parameter parsing for the CPU
// restatement of AMRClaw's level-advance path. Only tests/, the smoke check and
// the CPU-baseline leg of bench.py may load this code; the GPU product never does.
//
// The input files follow the read order of src/2d/amr2.f90:148-394 (claw.data,
// amr.data), src/2d/regions_module.f90:50-60 (regions.data) and
// src/2d/gauges_module.f90:92 (gauges.data). Each line is "values =: name",
// the layout clawpack's data writers produce; this parser keys on the name.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <map>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace orc {

struct DataFile {
  std::map<std::string, std::vector<std::string>> kv;
  std::vector<std::vector<std::string>> rows;  // lines without "=:" (region/gauge rows)
  bool load(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
      if (line.empty() || line[0] == '#') continue;
      size_t p = line.find("=:");
      std::string vals = (p == std::string::npos) ? line : line.substr(0, p);
      std::vector<std::string> toks;
      std::istringstream ss(vals);
      std::string t;
      while (ss >> t) toks.push_back(t);
      if (p == std::string::npos) {
        if (!toks.empty()) rows.push_back(toks);
        continue;
      }
      std::istringstream ns(line.substr(p + 2));
      std::string name;
      ns >> name;
      kv[name] = toks;
    }
    return true;
  }
  bool has(const std::string& k) const { return kv.count(k) > 0; }
  const std::vector<std::string>& get(const std::string& k) const {
    auto it = kv.find(k);
    if (it == kv.end()) throw std::runtime_error("missing key in data file: " + k);
    return it->second;
  }
  static double tod(const std::string& s) {
    std::string t = s;
    for (auto& c : t) if (c == 'd' || c == 'D') c = 'e';
    return std::strtod(t.c_str(), nullptr);
  }
  static bool tob(const std::string& s) {
    return s == "T" || s == "True" || s == "true" || s == ".true." || s == "1";
  }
  double d(const std::string& k, int i = 0) const { return tod(get(k).at(i)); }
  int i(const std::string& k, int j = 0) const { return (int)std::lround(tod(get(k).at(j))); }
  bool b(const std::string& k, int j = 0) const { return tob(get(k).at(j)); }
  std::string s(const std::string& k, int j = 0) const {
    std::string v = get(k).at(j);
    if (v.size() >= 2 && (v[0] == '\'' || v[0] == '"')) v = v.substr(1, v.size() - 2);
    return v;
  }
  double dget(const std::string& k, double def) const { return has(k) ? d(k) : def; }
  int iget(const std::string& k, int def) const { return has(k) ? i(k) : def; }
  std::string sget(const std::string& k, const std::string& def) const { return has(k) ? s(k) : def; }
};

// Fortran E-format output (Ew.d), e.g. e26.16 -> "   0.1000000000000000E+01".
inline std::string fmtE(double v, int w, int d) {
  char buf[64];
  if (v == 0.0) {
    std::string m = "0." + std::string(d, '0') + "E+00";
    if (std::signbit(v)) m = "-" + m;
    if ((int)m.size() < w) m = std::string(w - m.size(), ' ') + m;
    return m;
  }
  // value = 0.ddddd * 10^e
  std::snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(v));
  // buf = "D.DDDDe+XX": mantissa digits and exponent
  std::string s(buf);
  size_t epos = s.find('e');
  std::string mant = s.substr(0, epos);
  int ex = std::atoi(s.c_str() + epos + 1);
  std::string digits;
  for (char c : mant) if (c != '.') digits.push_back(c);
  ex += 1;
  char eb[16];
  std::string out = std::string(std::signbit(v) ? "-" : "") + "0." + digits;
  if (std::abs(ex) <= 99) {
    std::snprintf(eb, sizeof(eb), "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
  } else {
    std::snprintf(eb, sizeof(eb), "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
  }
  out += eb;
  if ((int)out.size() < w) out = std::string(w - out.size(), ' ') + out;
  return out;
}

}  // namespace orc
