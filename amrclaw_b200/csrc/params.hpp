// Run parameters read from the setrun.py data files (claw.data, amr.data,
// regions.data, gauges.data, setprob.data). Field order and meaning follow the
// reference reader src/2d/amr2.f90:148-394 and src/3d/amr3.f90; each file line is
// "values =: name" so lines are matched by name.
#pragma once
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace amrb {

struct KeyFile {
  std::map<std::string, std::vector<std::string>> kv;
  std::vector<std::vector<std::string>> rows;
  bool read(const std::string& path) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
      if (line.empty() || line[0] == '#') continue;
      const size_t p = line.find("=:");
      std::istringstream vs(p == std::string::npos ? line : line.substr(0, p));
      std::vector<std::string> toks;
      for (std::string t; vs >> t;) toks.push_back(t);
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
  const std::vector<std::string>& at(const std::string& k) const {
    auto it = kv.find(k);
    if (it == kv.end()) throw std::runtime_error("data file lacks '" + k + "'");
    return it->second;
  }
  bool has(const std::string& k) const { return kv.count(k) != 0; }
  static double num(std::string s) {
    for (char& c : s) if (c == 'd' || c == 'D') c = 'e';
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) throw std::runtime_error("not a number: " + s);
    return v;
  }
  double f(const std::string& k, int i = 0) const { return num(at(k).at(i)); }
  int n(const std::string& k, int i = 0) const { return (int)std::lround(num(at(k).at(i))); }
  bool b(const std::string& k, int i = 0) const {
    const std::string& s = at(k).at(i);
    return s == "T" || s == "True" || s == "true" || s == ".true." || s == "1";
  }
  std::string str(const std::string& k, int i = 0) const {
    std::string s = at(k).at(i);
    if (s.size() >= 2 && (s[0] == '\'' || s[0] == '"')) s = s.substr(1, s.size() - 2);
    return s;
  }
  double f_or(const std::string& k, double d) const { return has(k) ? f(k) : d; }
  int n_or(const std::string& k, int d) const { return has(k) ? n(k) : d; }
};

struct RegionSpec { int minlevel, maxlevel; double t1, t2, x1, x2, y1, y2, z1, z2; };
struct GaugeSpec { int num; double x, y, z, t1, t2, min_inc; };

struct RunParams {
  int ndim = 2;
  double lower[3] = {0, 0, 0}, upper[3] = {1, 1, 1};
  int ncells[3] = {1, 1, 1};
  int nvar = 1, mwaves = 1, naux = 0;
  double t0 = 0;
  int output_style = 1, nout = 0, iout = 0, nstop = 999999999;
  int output_format = 1;  // 1 ascii, 2 netcdf, 3 binary (valout.f90:108-113)
  std::vector<int> output_aux_components;  // per aux component, 1: written to fort.aNNNN (amr2.f90:212-218)
  bool output_aux_onlyonce = true;
  double tfinal = 0;
  bool output_t0 = true;
  std::vector<double> tout;
  double dt_initial = 1e-3, dt_max = 1e99, cfl_max = 1, cfl_desired = 0.9;
  int steps_max = 100000;
  bool vtime = true;
  int order = 2, trans = 2, dimsplit = 0, verbosity = 0, src_split = 0, mcapa = 0;
  bool use_fwaves = false;
  std::vector<int> mthlim;
  int nghost = 2;
  int mthbc[7] = {0};  // 1..2n: lower/upper per dimension in the reference's numbering
  int mxnest = 1;
  int ratx[12] = {0}, raty[12] = {0}, ratz[12] = {0}, ratt[12] = {0};
  std::vector<std::string> auxtype;
  bool flag_richardson = false, flag_gradient = true;
  double tol = -1, tolsp = 0.05, cut = 0.7;
  int kcheck = 2, ibuff = 3, max1d = 60;
  std::vector<RegionSpec> regions;
  std::vector<GaugeSpec> gauges;
  // problem plugin (setprob.data)
  std::string problem;
  std::map<std::string, double> probnum;
  std::map<std::string, std::string> probstr;
  int flag_component = 0;
  std::string flag_mode;
  // restart and checkpointing (amr3.f90:308-325)
  bool restart = false;
  std::string restart_file;
  int checkpt_style = 0, checkpt_interval = 0;
  std::vector<double> tchk;

  void load(const std::string& dir) {
    KeyFile c, a, r, g, s;
    if (!c.read(dir + "/claw.data")) throw std::runtime_error("cannot read " + dir + "/claw.data");
    if (!a.read(dir + "/amr.data")) throw std::runtime_error("cannot read " + dir + "/amr.data");
    ndim = c.n("num_dim");
    for (int d = 0; d < ndim; ++d) { lower[d] = c.f("lower", d); upper[d] = c.f("upper", d); ncells[d] = c.n("num_cells", d); }
    nvar = c.n("num_eqn"); mwaves = c.n("num_waves"); naux = c.n("num_aux");
    t0 = c.f("t0");
    output_style = c.n("output_style");
    if (c.has("output_format")) output_format = c.n("output_format");
    if (naux > 0 && c.has("output_aux_components")) {
      for (int k = 0; k < naux; ++k) output_aux_components.push_back(c.n("output_aux_components", k));
      if (c.has("output_aux_onlyonce")) output_aux_onlyonce = c.b("output_aux_onlyonce");
    }
    if (output_style == 1) {
      nout = c.n("num_output_times"); tfinal = c.f("tfinal"); output_t0 = c.b("output_t0");
      for (int k = 1; k <= nout; ++k) tout.push_back(t0 + k * (tfinal - t0) / (double)nout);
    } else if (output_style == 2) {
      for (auto& v : c.at("output_times")) tout.push_back(KeyFile::num(v));
      output_t0 = !tout.empty() && tout[0] == t0;
      if (output_t0) tout.erase(tout.begin());
      nout = (int)tout.size();
      tfinal = tout.empty() ? t0 : tout.back();
    } else if (output_style == 3) {
      iout = c.n("output_step_interval"); nstop = c.n("total_steps"); output_t0 = c.b("output_t0");
      nout = 0; tfinal = (double)10.e32f;
    } else throw std::runtime_error("output_style must be 1, 2 or 3");
    dt_initial = c.f("dt_initial"); dt_max = c.f("dt_max"); cfl_max = c.f("cfl_max"); cfl_desired = c.f("cfl_desired");
    steps_max = c.n("steps_max");
    if (output_style != 3) nstop = 999999999;
    vtime = c.b("dt_variable");
    order = c.n("order"); trans = c.n("transverse_waves"); dimsplit = c.n("dimensional_split");
    verbosity = c.n("verbosity"); src_split = c.n("source_split"); mcapa = c.n("capa_index");
    use_fwaves = c.b("use_fwaves");
    for (int k = 0; k < mwaves; ++k) mthlim.push_back(c.n("limiter", k));
    nghost = c.n("num_ghost");
    restart = c.has("restart") && c.b("restart");
    restart_file = c.has("restart_file") ? c.str("restart_file") : std::string();
    checkpt_style = c.n_or("checkpt_style", 0);
    if (checkpt_style == 2 || checkpt_style == -2) {
      if (c.has("checkpt_times")) for (auto& v : c.at("checkpt_times")) tchk.push_back(KeyFile::num(v));
    } else if (checkpt_style == 3 || checkpt_style == -3) {
      checkpt_interval = c.n("checkpt_interval");
      if (checkpt_interval < 1) throw std::runtime_error("checkpt_interval must be positive");
    }
    for (int d = 0; d < ndim; ++d) { mthbc[2 * d + 1] = c.n("bc_lower", d); mthbc[2 * d + 2] = c.n("bc_upper", d); }
    for (int d = 0; d < ndim; ++d)
      if ((mthbc[2 * d + 1] == 2) != (mthbc[2 * d + 2] == 2))
        throw std::runtime_error("periodic boundary conditions must be set on both sides");
    mxnest = a.n("amr_levels_max");
    if (mxnest < 1 || mxnest > 10) throw std::runtime_error("amr_levels_max must be in 1..10");
    const int nr = std::max(1, mxnest - 1);
    for (int k = 0; k < nr; ++k) {
      ratx[k + 1] = a.n("refinement_ratios_x", k);
      raty[k + 1] = a.n("refinement_ratios_y", k);
      if (ndim == 3) ratz[k + 1] = a.n("refinement_ratios_z", k);
      ratt[k + 1] = a.n("refinement_ratios_t", k);
    }
    if (naux > 0) for (int k = 0; k < naux; ++k) auxtype.push_back(a.str("aux_type", k));
    flag_richardson = a.b("flag_richardson"); tol = a.f("flag_richardson_tol");
    flag_gradient = a.b("flag2refine"); tolsp = a.f("flag2refine_tol");
    kcheck = a.n("regrid_interval"); ibuff = a.n("regrid_buffer_width"); cut = a.f("clustering_cutoff");
    max1d = a.n_or("max1d", ndim == 2 ? 60 : 32);
    if (r.read(dir + "/regions.data"))
      for (auto& row : r.rows) {
        if ((int)row.size() < 2 + 2 + 2 * ndim) continue;
        RegionSpec rg{};
        rg.minlevel = (int)KeyFile::num(row[0]); rg.maxlevel = (int)KeyFile::num(row[1]);
        rg.t1 = KeyFile::num(row[2]); rg.t2 = KeyFile::num(row[3]);
        rg.x1 = KeyFile::num(row[4]); rg.x2 = KeyFile::num(row[5]);
        rg.y1 = KeyFile::num(row[6]); rg.y2 = KeyFile::num(row[7]);
        if (ndim == 3) { rg.z1 = KeyFile::num(row[8]); rg.z2 = KeyFile::num(row[9]); }
        regions.push_back(rg);
      }
    if (g.read(dir + "/gauges.data"))
      for (auto& row : g.rows) {
        if ((int)row.size() < 3 + ndim) continue;
        GaugeSpec gs{};
        int k = 0;
        gs.num = (int)KeyFile::num(row[k++]);
        gs.x = KeyFile::num(row[k++]); gs.y = KeyFile::num(row[k++]);
        if (ndim == 3) gs.z = KeyFile::num(row[k++]);
        gs.t1 = KeyFile::num(row[k++]); gs.t2 = KeyFile::num(row[k++]);
        gs.min_inc = (k < (int)row.size()) ? KeyFile::num(row[k]) : 0.0;
        gauges.push_back(gs);
      }
    if (!s.read(dir + "/setprob.data")) throw std::runtime_error("cannot read " + dir + "/setprob.data");
    problem = s.str("problem");
    for (auto& kvp : s.kv) {
      if (kvp.first == "problem" || kvp.second.empty()) continue;
      probstr[kvp.first] = s.str(kvp.first);
      try { probnum[kvp.first] = KeyFile::num(kvp.second[0]); } catch (...) {}
    }
    flag_component = s.n_or("flag_component", 0);
    flag_mode = s.has("flag_mode") ? s.str("flag_mode") : std::string("component");
  }
  // valout.f90: aux arrays go to fort.aNNNN when any component is requested, every frame or
  // (output_aux_onlyonce) only at the initial time
  bool out_aux(double time) const {
    int n = 0;
    for (int x : output_aux_components) n += x;
    return n > 0 && (!output_aux_onlyonce || std::fabs(time - t0) < 1e-90);
  }
  double pn(const std::string& k, double d) const { auto it = probnum.find(k); return it == probnum.end() ? d : it->second; }
  std::string ps(const std::string& k, const std::string& d) const { auto it = probstr.find(k); return it == probstr.end() ? d : it->second; }
};

}  // namespace amrb
