// Text of the fort.qNNNN / fort.tNNNN output files (src/2d/valout.f90:51-65,149-165 and
// src/3d/valout.f90:45-62,140-160): the files are the drop-in contract with the plotting
// tools, so their layout follows the reference's Fortran edit descriptors exactly.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

namespace amrb {

// Fortran Ew.d text of a double: "0.ddd...E+xx" right-justified in w columns (the e26.16 /
// e18.8 fields); exponents beyond two digits drop the 'E' as Fortran does.
inline std::string fort_e(double v, int w, int d) {
  std::string out;
  if (v == 0.0) {
    out = std::string(std::signbit(v) ? "-" : "") + "0." + std::string(d, '0') + "E+00";
  } else {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(v));
    const std::string s(buf);
    const size_t e = s.find('e');
    std::string digits;
    for (size_t k = 0; k < e; ++k) if (s[k] != '.') digits.push_back(s[k]);
    const int ex = std::atoi(s.c_str() + e + 1) + 1;
    char eb[16];
    if (std::abs(ex) <= 99) std::snprintf(eb, sizeof(eb), "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else std::snprintf(eb, sizeof(eb), "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    out = std::string(std::signbit(v) ? "-" : "") + "0." + digits + eb;
  }
  if ((int)out.size() < w) out = std::string(w - out.size(), ' ') + out;
  return out;
}

inline FILE* open_output(const std::string& dir, const char* stem, int frame, const char* mode = "w") {
  char fn[64];
  std::snprintf(fn, sizeof(fn), "/%s%04d", stem, frame);
  FILE* f = std::fopen((dir + fn).c_str(), mode);
  if (!f) throw std::runtime_error("cannot write " + dir + fn);
  return f;
}

// Grid header of a fort.q (or fort.a) file: header_format_2d / header_format of valout.f90.
inline void write_grid_header(FILE* f, int ndim, int grid, int level, const int* n, const double* lower,
                              const double* delta) {
  static const char* nn[3] = {"mx", "my", "mz"};
  static const char* ll[3] = {"xlow", "ylow", "zlow"};
  static const char* dd[3] = {"dx", "dy", "dz"};
  std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n", grid, level);
  for (int d = 0; d < ndim; ++d) std::fprintf(f, "%6d                 %s\n", n[d], nn[d]);
  for (int d = 0; d < ndim; ++d) std::fprintf(f, "%s    %s\n", fort_e(lower[d], 26, 16).c_str(), ll[d]);
  for (int d = 0; d < ndim; ++d) std::fprintf(f, "%s    %s\n", fort_e(delta[d], 26, 16).c_str(), dd[d]);
  std::fputc('\n', f);
}

// raw doubles of a binary output file (stream access, no record markers); closes f
inline void write_raw(FILE* f, const std::vector<double>& v, const std::string& dir) {
  const size_t n = v.empty() ? 0 : std::fwrite(v.data(), sizeof(double), v.size(), f);
  const bool ok = n == v.size();
  if (std::fclose(f) != 0 || !ok) throw std::runtime_error("cannot write binary output in " + dir);
}

// fort.tNNNN (t_file_format of valout.f90)
inline void write_fort_t(const std::string& dir, int frame, double t, int meqn, int ngrids, int naux, int ndim,
                         int nghost) {
  FILE* f = open_output(dir, "fort.t", frame);
  std::fprintf(f, "%s    time\n%6d                 meqn\n%6d                 ngrids\n%6d                 naux\n%6d                 ndim\n%6d                 nghost\n\n",
               fort_e(t, 18, 8).c_str(), meqn, ngrids, naux, ndim, nghost);
  if (std::fclose(f) != 0) throw std::runtime_error("cannot close fort.t in " + dir);
}

}  // namespace amrb
