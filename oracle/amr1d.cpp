// Oracle (test infrastructure only): CPU FP64 restatement of AMRClaw's 1D per-level
// patch-advance path, used as the parity checker of the 1D device path. The GPU product
// (amrclaw_b200) never loads this code.
//
// Each routine follows the reference routine of src/1d named in its comment, with the
// same loop nesting and accumulation order (compile with -ffp-contract=off):
//   patch step      stepgrid.f:1-150, step1.f90:1-96, flux1.f:1-150, inlinelimiter.f
//   level advance   advanc.f:1-110 (advanc), :140-274 (par_advanc)
//   ghost fill      bound.f90:1-82, filpatch.f90:1-255, prefilp.f90:1-197,
//                   intfil.f90:1-216, trimbd.f90:1-49, bc1amr.f90:1-200,
//                   nodget.f (makeBndryList)
//   conservation    saveqc.f:1-100, cstore.f:1-38, icall.f:1-76, preicall.f:1-96,
//                   qad.f:1-183, fluxsv.f:1-63, fluxad.f:1-47, update.f:1-162,
//                   upbnd.f:1-107, prepf.f:1-36, prepc.f:1-102, setuse.f:1-64, putsp.f:1-40
//   regrid          regrid.f:1-161, grdfit1.f:1-130, flglvl1.f:1-90, flagger.f:1-151,
//                   flagregions1.f90, flag2refine1.f90, bufnst1.f:1-150, projec1.f:1-80,
//                   shiftset.f:1-55, setdomflags.f:1-152, griddomshrink.f, griddomup.f,
//                   griddomcopy.f, setPhysBndryFlags.f, setIndices.f, coarseGridFlagSet.f,
//                   colate1.f:1-120, flagcheck.f, drivesort.f, quick_sort1.f, smartbis.f,
//                   signs.f, findcut.f, moment.f, nestck1.f, baseCheck.f, birect.f,
//                   gfixup.f:1-197, filval.f90:1-222, intcopy.f, preintcopy.f
//   driver          amr1.f90, domain.f, setgrd.f, ginit.f, stst1.f, tick.f, conck.f
//   output          valout.f90 (1D header), gauges_module.f90 (setbestsrc, update_gauges)
//
// Two places of the reference are undefined behaviour, restated as the reference's intent:
// nestck1.f passes an unset zeroBuff to baseCheck (0 here, as nestck2.f sets it), and the
// first periodic branch of prepc.f:84-90 calls setuse with the argument list of the 2D
// routine, so its kflag is iclo - iregsz, never 1, and it adds no register entries.
#include "common.hpp"
#include "riemann1d.hpp"
#include <algorithm>
#include <functional>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc1 {

using orc::DataFile;
using orc::fmtE;

static const double UNSET = -1.0, DONTFLAG = 0.0, DOFLAG = 2.0, BADPRO = 3.0;
static const double NEEDS_TO_BE_SET = (double)10.e33f;  // default-real literal in amr_module.f90
static const double RINFINITY = (double)10.e32f;
static const int IINFINITY = 999999999;

struct Region1 { int minlevel, maxlevel; double tlow, thi, xlow, xhi; };
struct Sample1 { int level; double t; std::vector<double> v; };
struct Gauge1 { int num; double x, t_start, t_end; std::vector<Sample1> data; };

struct Node1 {
  int ilo = 0, ihi = 0, level = 0, levelptr = 0, nextfree = 0, numflags = 0;
  double xlo = 0, xhi = 0, time = 0;
  std::vector<double> q1, q2;   // store1, store2: (nvar, mitot)
  bool has_q2 = false;
  std::vector<double> ffl;      // svdflx(nvar,2), qc1d(nvar,2)
  bool has_ffl = false;
  std::vector<int> listbc;      // (4, maxsp): i, side, kid, register index
  bool has_cfl = false;
  std::vector<double> flags;    // storeflags (ilo-mbuff:ihi+mbuff)
  std::vector<signed char> dom2;  // domflags2 (ilo-mbuff:ihi+mbuff)
  std::vector<int> bnd;         // bndList in traversal order
};

struct Amr1 {
  // ---------------- input
  double xlower = 0, xupper = 1;
  int nx = 0, nvar = 1, mwaves = 1, naux = 0;
  double t0 = 0;
  int output_style = 1, nout = 0, iout = 0, nstop = IINFINITY;
  double tfinal = 0; bool output_t0 = true;
  std::vector<double> tout;
  int output_format = 1;
  double dt_initial = 0, dt_max = 0, cflv1 = 1, cfl = 0.9;
  int nv1 = 0; bool vtime = true;
  int method[8] = {0};
  int mcapa = 0;
  std::vector<int> mthlim;
  int nghost = 2;
  int mthbc[3] = {0};
  bool xperdom = false;
  int mxnest = 1;
  int intratx[12] = {0}, kratio[12] = {0};
  bool flag_gradient = true;
  double tolsp = 0.05, cut = 0.7;
  int kcheck = 2, ibuff = 2;
  int max1d = 500;
  std::vector<Region1> regions;
  std::vector<Gauge1> gauges;
  ProbParams1 prob;
  std::string problem;
  double beta = 0;

  // ---------------- state
  std::vector<Node1> node;
  int ndfree = 1, mstart = 0, lfine = 1;
  int lstart[12] = {0}, newstl[12] = {0}, numgrids[12] = {0}, listsp[12] = {0}, icheck[12] = {0};
  int iregsz[12] = {0};
  double hxposs[12] = {0}, possk[12] = {0};
  std::vector<int> levelgrids[12];
  double cfl_level = 0, cflmax = 0, rvol = 0, tmass0 = 0;
  int matlabu = 0;
  std::string outdir;
  bool write_output = false, record_gauges = true;
  std::vector<int> mbestsrc;
  double time = 0;
  int ncycle = 0;

  // ================================================================ input
  void read_input(const std::string& dir) {
    DataFile c, a, r, g, s;
    if (!c.load(dir + "/claw.data")) throw std::runtime_error("cannot read claw.data");
    if (!a.load(dir + "/amr.data")) throw std::runtime_error("cannot read amr.data");
    if (c.i("num_dim") != 1) throw std::runtime_error("1D oracle: num_dim must be 1");
    xlower = c.d("lower"); xupper = c.d("upper"); nx = c.i("num_cells");
    nvar = c.i("num_eqn"); mwaves = c.i("num_waves"); naux = c.i("num_aux");
    t0 = c.d("t0");
    output_style = c.i("output_style");
    if (output_style == 1) {
      nout = c.i("num_output_times"); tfinal = c.d("tfinal"); output_t0 = c.b("output_t0");
    } else if (output_style == 2) {
      for (auto& x : c.get("output_times")) tout.push_back(DataFile::tod(x));
      nout = (int)tout.size();
      output_t0 = (tout[0] == t0);
      if (output_t0) { tout.erase(tout.begin()); nout -= 1; }
      tfinal = tout.back();
    } else {
      iout = c.i("output_step_interval"); nstop = c.i("total_steps"); output_t0 = c.b("output_t0");
      nout = 0; tfinal = RINFINITY;
    }
    if (output_style == 1 && nout > 0) {
      tout.resize(nout);
      for (int k = 1; k <= nout; ++k) tout[k - 1] = t0 + k * (tfinal - t0) / (double)nout;
    }
    output_format = c.iget("output_format", 1);
    if (output_format != 1 && output_format != 3) throw std::runtime_error("output_format must be 1 (ASCII) or 3 (binary)");
    dt_initial = c.d("dt_initial"); dt_max = c.d("dt_max");
    cflv1 = c.d("cfl_max"); cfl = c.d("cfl_desired"); nv1 = c.i("steps_max");
    if (output_style != 3) nstop = IINFINITY;
    vtime = c.b("dt_variable");
    method[1] = vtime ? 2 : 1;
    method[2] = c.i("order"); method[3] = c.iget("verbosity", 0); method[4] = c.iget("source_split", 0);
    mcapa = c.i("capa_index");
    if (c.b("use_fwaves")) throw std::runtime_error("1D oracle: f-waves are not restated");
    for (int k = 0; k < mwaves; ++k) mthlim.push_back(c.i("limiter", k));
    nghost = c.i("num_ghost");
    mthbc[1] = c.i("bc_lower"); mthbc[2] = c.i("bc_upper");
    if ((mthbc[1] == 2) != (mthbc[2] == 2)) throw std::runtime_error("periodic boundaries: both sides must be 2");
    xperdom = mthbc[1] == 2 && mthbc[2] == 2;
    mxnest = a.i("amr_levels_max");
    const int nr = std::max(1, mxnest - 1);
    for (int k = 0; k < nr; ++k) { intratx[k + 1] = a.i("refinement_ratios_x", k); kratio[k + 1] = a.i("refinement_ratios_t", k); }
    if (a.b("flag_richardson")) throw std::runtime_error("1D oracle: Richardson estimation is not restated");
    flag_gradient = a.b("flag2refine"); tolsp = a.d("flag2refine_tol");
    kcheck = a.i("regrid_interval"); ibuff = a.i("regrid_buffer_width"); cut = a.d("clustering_cutoff");
    max1d = a.iget("max1d", 500);
    if (naux != 0 || mcapa != 0) throw std::runtime_error("1D oracle: no 1D problem carries aux arrays");
    if (r.load(dir + "/regions.data"))
      for (auto& row : r.rows) {
        if (row.size() < 6) continue;
        regions.push_back(Region1{(int)DataFile::tod(row[0]), (int)DataFile::tod(row[1]), DataFile::tod(row[2]), DataFile::tod(row[3]),
                                  DataFile::tod(row[4]), DataFile::tod(row[5])});
      }
    if (g.load(dir + "/gauges.data"))
      for (auto& row : g.rows) {
        if (row.size() < 4) continue;
        Gauge1 ga;
        ga.num = (int)DataFile::tod(row[0]); ga.x = DataFile::tod(row[1]);
        ga.t_start = DataFile::tod(row[2]); ga.t_end = DataFile::tod(row[3]);
        gauges.push_back(ga);
      }
    if (!s.load(dir + "/setprob.data")) throw std::runtime_error("cannot read setprob.data");
    problem = s.s("problem");
    if (problem == "advection_1d") {
      prob.solver = SOLVER1_ADVECTION; prob.u = s.d("u"); beta = s.d("beta");
    } else if (problem == "acoustics_1d") {
      prob.solver = SOLVER1_ACOUSTICS; prob.rho = s.d("rho"); prob.bulk = s.d("bulk"); beta = s.d("beta");
      prob.cc = std::sqrt(prob.bulk / prob.rho); prob.zz = prob.cc * prob.rho;
    } else if (problem == "euler_1d_wcblast") {
      prob.solver = SOLVER1_EULER; prob.gamma = s.dget("gamma", 1.4); prob.gamma1 = prob.gamma - 1.0;
    } else {
      throw std::runtime_error("1D oracle: unknown problem " + problem);
    }
  }

  // qinit of the reference's 1D regression tests: tests/advection_1d_example1/qinit.f90,
  // tests/acoustics_1d_homogeneous/qinit.f90, tests/euler_1d_wcblast/qinit.f90; q(nvar, mitot)
  void qinit(int mbc, int mx, double xl, double dx, double* q) {
    for (int i = 1; i <= mx; ++i) {
      const double xcell = xl + (i - 0.5) * dx;
      double* v = q + (size_t)nvar * (i + mbc - 1);
      if (prob.solver == SOLVER1_ADVECTION) {
        v[0] = std::exp(-beta * ((xcell - 0.75) * (xcell - 0.75)));
        if (xcell > 0.1 && xcell < 0.4) v[0] = v[0] + 1.0;
      } else if (prob.solver == SOLVER1_ACOUSTICS) {
        v[0] = std::exp(-beta * ((xcell - 0.3) * (xcell - 0.3)));
        v[1] = 0.0;
      } else {
        v[0] = 1.0; v[1] = 0.0;
        if (xcell < 0.1) v[2] = 1.e3 / prob.gamma1;
        else if (xcell < 0.9) v[2] = 1.e-2 / prob.gamma1;
        else v[2] = 1.e2 / prob.gamma1;
      }
    }
  }

  // ================================================================ nodes
  int nodget() {
    if (ndfree == 0) {
      const int old = (int)node.size() - 1;
      node.resize(old + 1 + 10000);
      for (int k = old + 1; k <= old + 10000; ++k) node[k].nextfree = k + 1;
      node[old + 10000].nextfree = 0;
      ndfree = old + 1;
    }
    const int m = ndfree;
    ndfree = node[m].nextfree;
    node[m] = Node1();
    return m;
  }
  void putnod(int m) { node[m].nextfree = ndfree; ndfree = m; }
  int mitot_of(int m) const { return node[m].ihi - node[m].ilo + 1 + 2 * nghost; }
  double& Q(std::vector<double>& q, int m, int i) const { return q[(m - 1) + (size_t)nvar * (i - 1)]; }

  // ================================================================ patch step
  // inlinelimiter.f: the wave limiter in the form flux1.f calls (limiter over i = 1..mx+1,
  // the neighbour dot products of the unlimited waves; philim's MC/minmod/... choices)
  static double philim(double a, double b, int meth) {
    const double r = b / a;
    switch (meth) {
      case 1: return std::max(0.0, std::min(1.0, r));
      case 2: return std::max(0.0, std::max(std::min(1.0, 2.0 * r), std::min(2.0, r)));
      case 3: return (r + std::fabs(r)) / (1.0 + std::fabs(r));
      case 4: { const double c = (1.0 + r) / 2.0; return std::max(0.0, std::min(c, std::min(2.0, 2.0 * r))); }
      case 5: return r;
    }
    return std::max(0.0, std::min(1.0, r));  // the computed GOTO falls through to minmod
  }
  void limiter(int mbc, int mx, Waves1 wave, Slice1 s) {
    for (int mw = 1; mw <= mwaves; ++mw) {
      if (mthlim[mw - 1] == 0) continue;
      double dotr = 0.0;
      for (int i = 0; i <= mx + 1; ++i) {
        double wnorm2 = 0.0;
        const double dotl = dotr;
        dotr = 0.0;
        for (int m = 1; m <= nvar; ++m) {
          wnorm2 = wnorm2 + wave(m, mw, i) * wave(m, mw, i);
          dotr = dotr + wave(m, mw, i) * wave(m, mw, i + 1);
        }
        if (i == 0) continue;
        if (wnorm2 == 0.0) continue;
        const double wlimitr = (s(mw, i) > 0.0) ? philim(wnorm2, dotl, mthlim[mw - 1]) : philim(wnorm2, dotr, mthlim[mw - 1]);
        for (int m = 1; m <= nvar; ++m) wave(m, mw, i) = wlimitr * wave(m, mw, i);
      }
    }
    (void)mbc;
  }
  // step1.f90 + flux1.f over one patch: fm, fp (nvar, mitot); returns cflgrid
  double step1(std::vector<double>& q, int mitot, double dx, double dt, std::vector<double>& fm, std::vector<double>& fp) {
    const int mbc = nghost, mx = mitot - 2 * nghost;
    const int n = mitot;
    std::vector<double> wave((size_t)nvar * mwaves * n), s((size_t)mwaves * n), amdq((size_t)nvar * n), apdq((size_t)nvar * n);
    std::vector<double> faddm((size_t)nvar * n, 0.0), faddp((size_t)nvar * n, 0.0);
    Slice1 q1d{q.data(), nvar, 1 - mbc}, S{s.data(), mwaves, 1 - mbc}, AM{amdq.data(), nvar, 1 - mbc}, AP{apdq.data(), nvar, 1 - mbc};
    Slice1 FAM{faddm.data(), nvar, 1 - mbc}, FAP{faddp.data(), nvar, 1 - mbc};
    Waves1 W{wave.data(), nvar, mwaves, 1 - mbc};
    const double dtdx = dt / dx;
    std::fill(fm.begin(), fm.end(), 0.0);
    std::fill(fp.begin(), fp.end(), 0.0);
    bool limit = false;
    for (int mw = 0; mw < mwaves; ++mw) if (mthlim[mw] > 0) limit = true;
    rp1(prob, nvar, mwaves, mbc, mx, q1d, q1d, W, S, AM, AP);
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= nvar; ++m) {
        FAP(m, i) = FAP(m, i) - AP(m, i);
        FAM(m, i) = FAM(m, i) + AM(m, i);
      }
    double cfl1d = 0.0;
    for (int mw = 1; mw <= mwaves; ++mw)
      for (int i = 1; i <= mx + 1; ++i) cfl1d = std::max(std::max(cfl1d, dtdx * S(mw, i)), -dtdx * S(mw, i));
    if (method[2] != 1) {
      if (limit) limiter(mbc, mx, W, S);
      for (int i = 1; i <= mx + 1; ++i) {
        const double dtdxave = 0.5 * (dtdx + dtdx);
        for (int m = 1; m <= nvar; ++m) {
          double cqxx = 0.0;
          for (int mw = 1; mw <= mwaves; ++mw)
            cqxx = cqxx + std::fabs(S(mw, i)) * (1.0 - std::fabs(S(mw, i)) * dtdxave) * W(m, mw, i);
          FAM(m, i) = FAM(m, i) + 0.5 * cqxx;
          FAP(m, i) = FAP(m, i) + 0.5 * cqxx;
        }
      }
    }
    // step1.f90: fm(:,1:mx+1) += faddm (fm is 1-based over the enlarged patch, cell 1-mbc first)
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= nvar; ++m) {
        const size_t at = (m - 1) + (size_t)nvar * (i + mbc - 1);
        fm[at] = fm[at] + FAM(m, i);
        fp[at] = fp[at] + FAP(m, i);
      }
    return cfl1d;
  }
  // stepgrid.f: the step and the conservative update of the interior
  double stepgrid(std::vector<double>& q, std::vector<double>& fm, std::vector<double>& fp, int mitot, double dt, double dx) {
    const double cflgrid = step1(q, mitot, dx, dt, fm, fp);
    cfl_level = std::max(cfl_level, cflgrid);
    const double dtdx = dt / dx;
    for (int i = nghost + 1; i <= mitot - nghost; ++i)
      for (int m = 1; m <= nvar; ++m)
        Q(q, m, i) = Q(q, m, i) - dtdx * (Q(fm, m, i + 1) - Q(fp, m, i));
    return cflgrid > 0.0 ? dt * cfl / cflgrid : RINFINITY;
  }

  // ================================================================ ghost cells
  // bc1amr.f90: extrapolation (1), periodic (2: nothing here), wall (3)
  void bc1amr(std::vector<double>& val, int nrow, double hx, double xlo_p, double xhi_p) {
    const double hxmarg = hx * .01;
    if (xperdom) return;
    if ((int)val.size() < nvar * nrow) throw std::runtime_error("bc1amr: array shorter than nrow");
    if (xlo_p < xlower - hxmarg) {
      const int nxl = (int)((xlower + hxmarg - xlo_p) / hx);
      if (mthbc[1] == 0) throw std::runtime_error("user boundary conditions are not provided");
      if (mthbc[1] == 1) for (int i = 1; i <= nxl; ++i) for (int m = 1; m <= nvar; ++m) Q(val, m, i) = Q(val, m, nxl + 1);
      if (mthbc[1] == 3) {
        for (int i = 1; i <= nxl; ++i) for (int m = 1; m <= nvar; ++m) Q(val, m, i) = Q(val, m, 2 * nxl + 1 - i);
        for (int i = 1; i <= nxl; ++i) Q(val, 2, i) = -Q(val, 2, i);
      }
    }
    if (xhi_p > xupper + hxmarg) {
      const int nxr = (int)((xhi_p - xupper + hxmarg) / hx);
      const int ibeg = std::max(nrow - nxr + 1, 1);
      if (mthbc[2] == 0) throw std::runtime_error("user boundary conditions are not provided");
      if (mthbc[2] == 1) for (int i = ibeg; i <= nrow; ++i) for (int m = 1; m <= nvar; ++m) Q(val, m, i) = Q(val, m, ibeg - 1);
      if (mthbc[2] == 3) {
        for (int i = ibeg; i <= nrow; ++i) for (int m = 1; m <= nvar; ++m) Q(val, m, i) = Q(val, m, 2 * ibeg - 1 - i);
        for (int i = ibeg; i <= nrow; ++i) Q(val, 2, i) = -Q(val, 2, i);
      }
    }
  }
  // intfil.f90: same-level sources of [ilo,ihi] into val from row nrowst (time-interpolated)
  void intfil(std::vector<double>& val, double t, std::vector<signed char>& flaguse, int nrowst, int ilo, int ihi, int level, int msrc) {
    const double t_epsilon = 1.0e-4;
    const double dt = possk[level];
    std::fill(flaguse.begin(), flaguse.end(), 0);
    auto FU = [&](int i) -> signed char& { return flaguse[i - ilo]; };
    std::vector<int> srcs;
    if (msrc == -1) srcs = levelgrids[level];
    else srcs = node[msrc].bnd;
    for (int mptr : srcs) {
      Node1& g = node[mptr];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi);
      if (ixlo > ixhi) continue;
      const double alphac = (g.time - t) / dt;
      const double alphai = 1.0 - alphac;
      if (alphai < -t_epsilon || alphai > 1.0 + t_epsilon) throw std::runtime_error("intfil: time wanted not available");
      int mode;
      if (std::fabs(alphai - 1.0) < t_epsilon) mode = 1;
      else if (std::fabs(alphai) < t_epsilon) mode = 2;
      else mode = 3;
      if ((mode == 2 || mode == 3) && level == mxnest) throw std::runtime_error("intfil: old values wanted at the finest level");
      for (int ivar = 1; ivar <= nvar; ++ivar)
        for (int i = ixlo; i <= ixhi; ++i) {
          const int at = i - g.ilo + nghost + 1;
          double v;
          if (mode == 1) v = Q(g.q1, ivar, at);
          else if (mode == 2) v = Q(g.q2, ivar, at);
          else v = Q(g.q1, ivar, at) * alphai + Q(g.q2, ivar, at) * alphac;
          Q(val, ivar, i - ilo + nrowst) = v;
          FU(i) = 1;
        }
    }
    if (ilo < 0) for (int i = ilo; i <= std::min(-1, nrowst + ihi - ilo); ++i) if (i <= ihi) FU(i) = 1;
    if (ihi >= iregsz[level]) for (int i = std::max(iregsz[level], ilo); i <= ihi; ++i) FU(i) = 1;
  }
  // trimbd.f90: the first and last unset cell
  static void trimbd(const std::vector<signed char>& used, bool& set, int unset[2]) {
    const int n = (int)used.size();
    int utot = 0;
    for (int i = 0; i < n; ++i) utot += used[i];
    if (utot == n) { set = true; return; }
    set = false;
    int check = 1;
    for (int i = 1; i <= n; ++i) { check = std::min(check, (int)used[i - 1]); unset[0] = i; if (check == 0) break; }
    check = 1;
    for (int i = 1; i <= n; ++i) { check = std::min(check, (int)used[n - i]); unset[1] = n - i + 1; if (check == 0) break; }
  }
  // filpatch.f90 (filrecur): [ilo,ihi] of `level` into valbig from row nrowst
  void filrecur(int level, std::vector<double>& valbig, double t, int nrowst, int ilo, int ihi, bool patchOnly, int msrc) {
    const int mitot_patch = ihi - ilo + 1;
    const double dx_fine = hxposs[level];
    const double xlow_fine = xlower + ilo * dx_fine;
    std::vector<signed char> flaguse(mitot_patch);
    intfil(valbig, t, flaguse, nrowst, ilo, ihi, level, msrc);
    bool set;
    int unset[2];
    trimbd(flaguse, set, unset);
    if (!set) {
      if (level == 1) throw std::runtime_error("filrecur: level 1 cells not covered");
      const double dx_coarse = hxposs[level - 1];
      unset[0] = unset[0] + ilo - 1;
      unset[1] = unset[1] + ilo - 1;
      const int r = intratx[level - 1];
      const int iplo = (unset[0] - r + nghost * r) / r - nghost;
      const int iphi = (unset[1] + r) / r;
      const double xlow_coarse = xlower + iplo * dx_coarse;
      const int mitot_coarse = iphi - iplo + 1;
      if (mitot_coarse > ihi - ilo + 3) throw std::runtime_error("filrecur: coarse patch too large");
      std::vector<double> valcrse((size_t)nvar * mitot_coarse, 0.0);
      if (xperdom && (iplo < 0 || iphi >= iregsz[level - 1]))
        prefilrecur(level - 1, valcrse, t, 1, iplo, iphi, iplo);
      else
        filrecur(level - 1, valcrse, t, 1, iplo, iphi, true, -1);
      const double ratiox = (double)r;
      for (int i_fine = 1; i_fine <= mitot_patch; ++i_fine) {
        const int i_coarse = (int)std::floor((i_fine + ilo - 1) / ratiox) - iplo + 1;
        if (i_coarse < 2 || i_coarse > mitot_coarse - 1) throw std::runtime_error("filrecur: coarse stencil outside its patch");
        const double xcent_coarse = xlow_coarse + (i_coarse - .5) * dx_coarse;
        const double xcent_fine = xlower + (i_fine - 1 + ilo + .5) * dx_fine;
        const double eta1 = (xcent_fine - xcent_coarse) / dx_coarse;
        if (flaguse[i_fine - 1] == 0) {
          for (int n = 1; n <= nvar; ++n) {
            const double valp = Q(valcrse, n, i_coarse + 1), valm = Q(valcrse, n, i_coarse - 1), valc = Q(valcrse, n, i_coarse);
            const double dupc = valp - valc, dumc = valc - valm, ducc = valp - valm;
            double du = std::min(std::fabs(dupc), std::fabs(dumc));
            du = std::min(2.0 * du, 0.5 * std::fabs(ducc));
            const double fu = std::max(0.0, orc1_sign(1.0, dupc * dumc));
            const double uslope = du * orc1_sign(1.0, ducc) * fu;
            Q(valbig, n, i_fine + nrowst - 1) = valc + eta1 * uslope;
          }
        }
      }
    }
    const double xhi_fine = xlower + (ihi + 1) * dx_fine;
    if (patchOnly) bc1amr(valbig, (int)(valbig.size() / nvar), dx_fine, xlow_fine, xhi_fine);
  }
  static double orc1_sign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }
  // prefilp.f90 (prefilrecur): the three pieces of [ilo,ihi] at their periodic places,
  // each filled into a scratch patch and copied into valbig, whose index 1 is cell iglo
  void prefilrecur(int level, std::vector<double>& valbig, double t, int nrowst, int ilo, int ihi, int iglo) {
    (void)nrowst;
    int ist[3], iend[3], ishift[3];
    if (xperdom) {
      ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[level];
      iend[0] = -1; iend[1] = iregsz[level] - 1; iend[2] = ihi;
      ishift[0] = iregsz[level]; ishift[1] = 0; ishift[2] = -iregsz[level];
    } else {
      ist[0] = iregsz[level]; ist[1] = ilo; ist[2] = iregsz[level];
      iend[0] = -1; iend[1] = ihi; iend[2] = -1;
      ishift[0] = ishift[1] = ishift[2] = 0;
    }
    for (int k = 0; k < 3; ++k) {
      const int i1 = std::max(ilo, ist[k]), i2 = std::min(ihi, iend[k]);
      if (i1 > i2) continue;
      const int mi = i2 - i1 + 1;
      std::vector<double> valpatch((size_t)nvar * mi, 0.0);
      filrecur(level, valpatch, t, 1, i1 + ishift[k], i2 + ishift[k], true, -1);
      const int is = i1 - iglo + 1;
      for (int ii = 1; ii <= mi; ++ii) for (int m = 1; m <= nvar; ++m) Q(valbig, m, is + ii - 1) = Q(valpatch, m, ii);
    }
  }
  // bound.f90: the two ghost strips, then the physical boundaries
  void bound(double t, std::vector<double>& valbig, int mitot, int mptr) {
    const Node1& g = node[mptr];
    const int ng = nghost, lev = g.level;
    const double hx = hxposs[lev];
    const double xleft = g.xlo, xright = g.xhi;
    if ((xleft - ng * hx < xlower) && xperdom) prefilrecur(lev, valbig, t, 1, g.ilo - ng, g.ilo - 1, g.ilo - ng);
    else filrecur(lev, valbig, t, 1, g.ilo - ng, g.ilo - 1, false, mptr);
    if ((xright + ng * hx > xupper) && xperdom) prefilrecur(lev, valbig, t, mitot - ng + 1, g.ihi + 1, g.ihi + ng, g.ilo - ng);
    else filrecur(lev, valbig, t, mitot - ng + 1, g.ihi + 1, g.ihi + ng, false, mptr);
    bc1amr(valbig, mitot, hx, xleft - ng * hx, xright + ng * hx);
  }

  // ================================================================ copies from a level
  // icall.f / intcopy.f: store1 of the grids of `level` over [ilo,ihi] into val from iputst
  void icall(std::vector<double>& val, int ilo, int ihi, int level, int iputst) {
    for (int mptr = lstart[level]; mptr != 0; mptr = node[mptr].levelptr) {
      Node1& g = node[mptr];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi);
      if (ixlo > ixhi) continue;
      for (int i = ixlo; i <= ixhi; ++i)
        for (int ivar = 1; ivar <= nvar; ++ivar) Q(val, ivar, i - ilo + iputst) = Q(g.q1, ivar, i - g.ilo + nghost + 1);
    }
  }
  // preicall.f / preintcopy.f: icall over the three pieces with periodic shifts
  void preicall(std::vector<double>& val, int ilo, int ihi, int level, bool intcopy_form) {
    int ist[3], iend[3], ishift[3];
    if (xperdom) {
      ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[level];
      iend[0] = -1; iend[1] = iregsz[level] - 1; iend[2] = ihi;
      ishift[0] = iregsz[level]; ishift[1] = 0; ishift[2] = -iregsz[level];
    } else {
      ist[0] = iregsz[level]; ist[1] = ilo; ist[2] = iregsz[level];
      iend[0] = intcopy_form ? -1 : -nghost; iend[1] = ihi; iend[2] = intcopy_form ? -1 : -nghost;
      ishift[0] = ishift[1] = ishift[2] = 0;
    }
    for (int k = 0; k < 3; ++k) {
      const int i1 = std::max(ilo, ist[k]), i2 = std::min(ihi, iend[k]);
      if (i1 <= i2) icall(val, i1 + ishift[k], i2 + ishift[k], level, i1 - ilo + 1);
    }
  }

  // ================================================================ coarse/fine conservation
  // saveqc.f + cstore.f: the coarse values next to each fine grid of `level`
  void saveqc(int level) {
    const int levc = level - 1;
    const double hxc = hxposs[levc];
    for (int mkid = lstart[level]; mkid != 0; mkid = node[mkid].levelptr) {
      Node1& k = node[mkid];
      const int iclo = k.ilo / intratx[level - 1] - 1, ichi = (k.ihi + 1) / intratx[level - 1];
      const int nrow = ichi - iclo + 1;
      const double xl = k.xlo - hxc, xr = k.xhi + hxc;
      std::vector<double> tmp((size_t)nvar * nrow, 0.0);
      const bool sticksout = iclo < 0 || ichi == iregsz[levc];
      if (sticksout && xperdom) preicall(tmp, iclo, ichi, level - 1, false);
      else icall(tmp, iclo, ichi, level - 1, 1);
      bc1amr(tmp, nrow, hxc, xl, xr);
      // cstore.f: qc1d(:,1) = qc(:,1), qc1d(:,2) = qc(:,nrow)
      for (int iv = 1; iv <= nvar; ++iv) {
        k.ffl[(size_t)2 * nvar + (iv - 1)] = Q(tmp, iv, 1);
        k.ffl[(size_t)2 * nvar + nvar + (iv - 1)] = Q(tmp, iv, nrow);
      }
    }
  }
  // qad.f: the coarse/fine Riemann problems at the fine grid's two ends, into svdflx
  void qad(std::vector<double>& valbig, int mitot, std::vector<double>& ffl, double delt) {
    const int mbc = nghost;
    // rp1 over a one-interface row: arrays of 2 cells from index 1-mbc (mx = 2-2*mbc)
    auto solve = [&](const double* left, const double* right, double* am, double* ap) {
      const int mx = 2 - 2 * mbc;
      std::vector<double> ql((size_t)nvar * 2), qr((size_t)nvar * 2), wave((size_t)nvar * mwaves * 2), s((size_t)mwaves * 2),
          amdq((size_t)nvar * 2), apdq((size_t)nvar * 2);
      for (int m = 0; m < nvar; ++m) { qr[m] = left[m]; ql[nvar + m] = right[m]; }
      rp1(prob, nvar, mwaves, mbc, mx, Slice1{ql.data(), nvar, 1 - mbc}, Slice1{qr.data(), nvar, 1 - mbc},
          Waves1{wave.data(), nvar, mwaves, 1 - mbc}, Slice1{s.data(), mwaves, 1 - mbc}, Slice1{amdq.data(), nvar, 1 - mbc},
          Slice1{apdq.data(), nvar, 1 - mbc});
      for (int m = 0; m < nvar; ++m) { am[m] = amdq[nvar + m]; ap[m] = apdq[nvar + m]; }
    };
    std::vector<double> am(nvar), ap(nvar), l(nvar), r(nvar);
    // left end: coarse qc1d(:,1) | fine valbig(:,nghost)
    for (int m = 0; m < nvar; ++m) { l[m] = ffl[(size_t)2 * nvar + m]; r[m] = Q(valbig, m + 1, nghost); }
    solve(l.data(), r.data(), am.data(), ap.data());
    for (int m = 0; m < nvar; ++m) ffl[m] = ffl[m] + am[m] * delt + ap[m] * delt;
    // right end: fine valbig(:,mitot-nghost+1) | coarse qc1d(:,2)
    for (int m = 0; m < nvar; ++m) { l[m] = Q(valbig, m + 1, mitot - nghost + 1); r[m] = ffl[(size_t)3 * nvar + m]; }
    solve(l.data(), r.data(), am.data(), ap.data());
    for (int m = 0; m < nvar; ++m) ffl[nvar + m] = ffl[nvar + m] - am[m] * delt - ap[m] * delt;
  }
  // fluxsv.f: coarse fluxes next to a kid into the kid's register
  void fluxsv(int mptr, const std::vector<double>& fm, const std::vector<double>& fp, double dtc) {
    Node1& g = node[mptr];
    const int maxsp = listsp[g.level];
    for (int ispot = 1; ispot <= maxsp; ++ispot) {
      const int* e = &g.listbc[(size_t)4 * (ispot - 1)];
      if (e[0] == 0) break;
      const int mkid = e[2], intopl = e[3], i = e[0];
      Node1& k = node[mkid];
      double* dst = &k.ffl[(size_t)nvar * (intopl - 1)];
      if (e[1] == 1) for (int iv = 1; iv <= nvar; ++iv) dst[iv - 1] = -fp[(iv - 1) + (size_t)nvar * (i - 1)] * dtc;
      if (e[1] == 2) for (int iv = 1; iv <= nvar; ++iv) dst[iv - 1] = -fm[(iv - 1) + (size_t)nvar * i] * dtc;
    }
  }
  // fluxad.f: the fine grid's own boundary fluxes into its register
  void fluxad(const std::vector<double>& fm, const std::vector<double>& fp, std::vector<double>& ffl, int mitot, double dtf) {
    const int ng = nghost;
    for (int iv = 1; iv <= nvar; ++iv) ffl[iv - 1] = ffl[iv - 1] + fm[(iv - 1) + (size_t)nvar * ng] * dtf;
    for (int iv = 1; iv <= nvar; ++iv) ffl[nvar + iv - 1] = ffl[nvar + iv - 1] + fp[(iv - 1) + (size_t)nvar * (mitot - ng)] * dtf;
  }

  // ================================================================ level substep
  void update_gauges(std::vector<double>& q, double xlow, int mitot, int mptr);
  double par_advanc(int mptr) {
    Node1& g = node[mptr];
    const int level = g.level;
    const double hx = hxposs[level], delt = possk[level];
    const int nxg = g.ihi - g.ilo + 1, mitot = nxg + 2 * nghost;
    if (level < mxnest) g.q2 = g.q1;
    const double xlow = g.xlo - nghost * hx;
    rvol = rvol + nxg;
    if (g.has_ffl) qad(g.q1, mitot, g.ffl, delt);
    if (!gauges.empty()) update_gauges(g.q1, xlow, mitot, mptr);
    std::vector<double> fm((size_t)nvar * mitot), fp((size_t)nvar * mitot);
    const double dtnew = stepgrid(g.q1, fm, fp, mitot, delt, hx);
    if (g.has_cfl) fluxsv(mptr, fm, fp, delt);
    if (g.has_ffl) fluxad(fm, fp, g.ffl, mitot, delt);
    g.time = g.time + delt;
    return dtnew;
  }
  void advanc(int level, double& dtlevnew) {
    for (int mptr : levelgrids[level]) {
      Node1& g = node[mptr];
      bound(g.time, g.q1, mitot_of(mptr), mptr);
    }
    if (level + 1 <= mxnest && lstart[level + 1] != 0) saveqc(level + 1);
    dtlevnew = RINFINITY;
    cfl_level = 0.0;
    for (int mptr : levelgrids[level]) dtlevnew = std::min(dtlevnew, par_advanc(mptr));
    cflmax = std::max(cflmax, cfl_level);
  }

  // ================================================================ level sync
  // upbnd.f: the register corrections of a coarse grid, each coarse cell once per side
  void upbnd(int mptr) {
    Node1& g = node[mptr];
    const int mitot = mitot_of(mptr);
    std::vector<int> iused(mitot + 1, 0);
    const double area = hxposs[g.level];
    const int maxsp = listsp[g.level];
    for (int ispot = 1; ispot <= maxsp; ++ispot) {
      const int* e = &g.listbc[(size_t)4 * (ispot - 1)];
      const int icrse = e[0];
      if (icrse == 0) break;
      const int iside = e[1];
      const int norm = 1 << (iside - 1);
      if ((iused[icrse] / norm) % 2 == 1) continue;
      const int mkid = e[2], lkid = e[3];
      const double sgnm = (iside == 2) ? -1. : 1.;
      const double* reg = &node[mkid].ffl[(size_t)nvar * (lkid - 1)];
      for (int iv = 1; iv <= nvar; ++iv) Q(g.q1, iv, icrse) = Q(g.q1, iv, icrse) + sgnm * reg[iv - 1] / area;
      iused[icrse] = iused[icrse] + norm;
    }
  }
  // update.f: registers, then the fine averages over every coarse cell a kid covers
  void update(int level) {
    for (int mptr : levelgrids[level]) {
      Node1& g = node[mptr];
      if (g.has_cfl) upbnd(mptr);
      for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        Node1& k = node[mkid];
        const int iclo = k.ilo / intratx[level], ichi = k.ihi / intratx[level];
        const int iplo = std::max(g.ilo, iclo), iphi = std::min(g.ihi, ichi);
        if (iplo > iphi) continue;
        int iff = iplo * intratx[level] - k.ilo + nghost + 1;
        const double totrat = intratx[level];
        for (int i = iplo - g.ilo + nghost + 1; i <= iphi - g.ilo + nghost + 1; ++i) {
          for (int iv = 1; iv <= nvar; ++iv) Q(g.q1, iv, i) = 0.0;
          for (int ico = 1; ico <= intratx[level]; ++ico)
            for (int iv = 1; iv <= nvar; ++iv) Q(g.q1, iv, i) = Q(g.q1, iv, i) + Q(k.q1, iv, iff + ico - 1);
          for (int iv = 1; iv <= nvar; ++iv) Q(g.q1, iv, i) = Q(g.q1, iv, i) / totrat;
          iff = iff + intratx[level];
        }
      }
    }
  }
  // prepf.f: zeroed registers (svdflx, qc1d) for every grid of `level`
  void prepf(int level) {
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
      node[m].ffl.assign((size_t)4 * nvar, 0.0);
      node[m].has_ffl = true;
    }
  }
  // setuse.f: the parent cells just outside a kid's coarsened extent [iclo,ichi]
  void setuse(std::vector<int>& lb, int& ispot, int mkid, int ilo, int ihi, int iclo, int ichi, int kflag) {
    const int ist = iclo - 1, iend = ichi + 1;
    if (!(ist < ilo || kflag != 1)) {
      ++ispot;
      lb.insert(lb.end(), {ist - ilo + nghost + 1, 2, mkid, 1});
    }
    if (!(iend > ihi || kflag != 1)) {
      ++ispot;
      lb.insert(lb.end(), {iend - ilo + nghost + 1, 1, mkid, 2});
    }
  }
  // prepc.f: each parent's list of cells next to kids (with the periodic images of
  // prepc.f:84-100: the first branch adds nothing, see the file's header)
  void prepc(int level) {
    int maxsp = 0;
    for (int m = lstart[level + 1]; m != 0; m = node[m].levelptr) maxsp += 2;
    listsp[level] = maxsp;
    if (maxsp == 0) return;
    const int imax = iregsz[level] - 1;
    for (int mpar = lstart[level]; mpar != 0; mpar = node[mpar].levelptr) {
      Node1& p = node[mpar];
      int ispot = 0;
      p.listbc.clear();
      p.has_cfl = true;
      for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        const Node1& k = node[mkid];
        const int iclo = k.ilo / intratx[level], ichi = k.ihi / intratx[level];
        const int iplo = std::max(p.ilo, iclo), iphi = std::min(p.ihi, ichi);
        if (iplo <= iphi + 1) setuse(p.listbc, ispot, mkid, p.ilo, p.ihi, iclo, ichi, 1);
        if (xperdom && iclo == 0 && p.ihi == imax)
          setuse(p.listbc, ispot, mkid, p.ilo, p.ihi, iclo + iregsz[level], ichi + iregsz[level], 1);
      }
      p.listbc.resize((size_t)4 * maxsp, 0);
    }
  }
  // putsp.f
  void putsp(int lbase, int level) {
    if (level != lfine)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].listbc.clear(); node[m].has_cfl = false; }
    if (level == lbase) return;
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].ffl.clear(); node[m].has_ffl = false; }
  }

  // ================================================================ grid lists
  // nodget.f (makeGridList): the grid lists of levels lbase+1..lfine
  void makeGridList(int lbase) {
    for (int lev = lbase + 1; lev <= lfine; ++lev) {
      levelgrids[lev].clear();
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) levelgrids[lev].push_back(m);
    }
  }
  // nodget.f (makeBndryList): the same-level grids meeting each grid grown by nghost, in
  // the order the prepended list is walked (last found first)
  void makeBndryList(int level) {
    const std::vector<int>& G = levelgrids[level];
    for (size_t n = 0; n < G.size(); ++n) {
      Node1& g = node[G[n]];
      g.bnd.clear();
      const int imin = g.ilo - nghost, imax = g.ihi + nghost;
      for (size_t k = 0; k < G.size(); ++k) {
        if (k == n) continue;
        const Node1& s = node[G[k]];
        if (std::max(s.ilo, imin) <= std::min(s.ihi, imax)) g.bnd.insert(g.bnd.begin(), G[k]);
      }
    }
  }
  // quick_sort1.f (qsorti), step by step: tie order decides the grid order
  static void qsorti(std::vector<int>& ord, int n, const std::vector<long long>& a) {
    int poplst[2][64];
    int ndeep = 0, u1 = n, l1 = 1;
    for (int i = 1; i <= n; ++i) ord[i] = i;
    int l, u, p, q, ix, iz, yp, ip, iq;
    long long x, z, xx, zz, y;
  L2:
    if (u1 <= l1) return;
  L3:
    l = l1; u = u1;
  L4:
    p = l; q = u;
    x = a[ord[p]]; z = a[ord[q]];
    if (!(x <= z)) { y = x; x = z; z = y; yp = ord[p]; ord[p] = ord[q]; ord[q] = yp; }
    if (u - l <= 1) goto L15;
    xx = x; ix = p; zz = z; iz = q;
  L6:
    p = p + 1;
    if (p >= q) goto L7;
    x = a[ord[p]];
    if (x >= xx) goto L8;
    goto L6;
  L7:
    p = q - 1;
    goto L13;
  L8:
    q = q - 1;
    if (q <= p) goto L9;
    z = a[ord[q]];
    if (z <= zz) goto L10;
    goto L8;
  L9:
    q = p; p = p - 1; z = x; x = a[ord[p]];
  L10:
    if (!(x <= z)) { y = x; x = z; z = y; ip = ord[p]; ord[p] = ord[q]; ord[q] = ip; }
    if (!(x <= xx)) { xx = x; ix = p; }
    if (!(z >= zz)) { zz = z; iz = q; }
    goto L6;
  L13:
    if (p != ix && x != xx) { ip = ord[p]; ord[p] = ord[ix]; ord[ix] = ip; }
    if (q != iz && z != zz) { iq = ord[q]; ord[q] = ord[iz]; ord[iz] = iq; }
  L15:
    if (u - q <= p - l) goto L16;
    l1 = l; u1 = p - 1; l = q + 1;
    goto L17;
  L16:
    u1 = u; l1 = q + 1; u = p - 1;
  L17:
    if (u1 <= l1) goto L18;
    ndeep = ndeep + 1;
    poplst[0][ndeep] = u; poplst[1][ndeep] = l;
    goto L3;
  L18:
    if (u > l) goto L4;
    if (ndeep == 0) goto L2;
    u = poplst[0][ndeep]; l = poplst[1][ndeep]; ndeep = ndeep - 1;
    goto L18;
  }
  // regrid.f (arrangeGrids): the level's grids by decreasing size
  void arrangeGrids(int level, int numg) {
    std::vector<int> listgrids(numg + 1), index(numg + 1);
    std::vector<long long> cost(numg + 1);
    int mptr = lstart[level];
    for (int i = 1; i <= numg; ++i) {
      listgrids[i] = mptr;
      cost[i] = node[mptr].ihi - node[mptr].ilo + 1;
      mptr = node[mptr].levelptr;
    }
    qsorti(index, numg, cost);
    lstart[level] = listgrids[index[numg]];
    int prev = listgrids[index[numg]];
    for (int i = 1; i <= numg - 1; ++i) {
      node[prev].levelptr = listgrids[index[numg - i]];
      prev = listgrids[index[numg - i]];
    }
    node[prev].levelptr = 0;
  }
  // birect.f: halve grids wider than max1d (with ghost cells) at a multiple of the ratio
  void birect(int mptr1) {
    int mptr = mptr1;
    const int level = node[mptr].level;
    const double hx = hxposs[level];
    while (true) {
      Node1& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1;
      if (nxg + 2 * nghost > max1d) {
        int nxl = nxg / 2;
        const int lratio = level > 1 ? intratx[level - 1] : 2;
        nxl = (nxl / lratio) * lratio;
        const double cxlo = g.xlo, cxhi = g.xhi, cxmid = cxlo + nxl * hx;
        const int mnx = nodget();
        Node1& a = node[mptr];
        Node1& b = node[mnx];
        b.levelptr = a.levelptr; a.levelptr = mnx;
        a.xhi = cxmid;
        b.ihi = a.ihi; a.ihi = a.ilo + nxl - 1; b.ilo = a.ihi + 1;
        b.xlo = cxmid; b.xhi = cxhi; b.time = a.time; b.level = a.level;
        continue;
      }
      mptr = g.levelptr;
      if (mptr == 0) break;
    }
  }

  // ================================================================ flagging
  void flagregions1(int mx, int mbuff, double xl, double dx, int level, double t, double* amrflags) {
    std::vector<int> minlevel(mx + 1, 0), maxlevel(mx + 1, 0);
    const double xu = xl + mx * dx;
    for (const Region1& R : regions) {
      if (t < R.tlow || t > R.thi) continue;
      if (xl >= R.xhi || xu <= R.xlow) continue;
      const int i1 = std::max((int)std::floor((R.xlow - xl) / dx) + 1, 1);
      const int i2 = std::min((int)std::floor((R.xhi - xl) / dx) + 1, mx);
      for (int i = i1; i <= i2; ++i) {
        minlevel[i] = std::max(minlevel[i], R.minlevel);
        maxlevel[i] = std::max(maxlevel[i], R.maxlevel);
      }
    }
    for (int i = 1; i <= mx; ++i) {
      if (minlevel[i] > maxlevel[i]) throw std::runtime_error("flagregions1: minlevel > maxlevel");
      if (maxlevel[i] != 0) {
        if (level < minlevel[i]) amrflags[i + mbuff - 1] = DOFLAG;
        else if (level >= maxlevel[i]) amrflags[i + mbuff - 1] = DONTFLAG;
      }
    }
  }
  // flag2refine1.f90 (the library's, or tests/euler_1d_wcblast/flag2refine1.f90 for the blast:
  // every cell DONTFLAG, then the density difference); amrflags(1-mbuff:mx+mbuff)
  void flag2refine1(int mx, int mbuff, std::vector<double>& q, double* amrflags) {
    auto QQ = [&](int m, int i) { return Q(q, m, i + nghost); };
    if (prob.solver == SOLVER1_EULER) {
      for (int i = 1 - mbuff; i <= mx + mbuff; ++i) amrflags[i + mbuff - 1] = DONTFLAG;
      for (int i = 1; i <= mx; ++i)
        if (std::fabs(QQ(1, i + 1) - QQ(1, i - 1)) > tolsp) amrflags[i + mbuff - 1] = DOFLAG;
      return;
    }
    for (int i = 1; i <= mx; ++i) {
      if (amrflags[i + mbuff - 1] != UNSET) continue;
      for (int m = 1; m <= nvar; ++m) {
        const double dq = std::max(0.0, std::fabs(QQ(m, i + 1) - QQ(m, i - 1)));
        if (dq > tolsp) { amrflags[i + mbuff - 1] = DOFLAG; break; }
      }
    }
  }
  // flagger.f: per grid flags (ilo-mbuff:ihi+mbuff), from store1 after a ghost fill or,
  // at the first step of a run, from store2
  void flagger(int lcheck, double start_time) {
    const int mbuff = std::max(nghost, ibuff + 1);
    for (int mptr : levelgrids[lcheck]) {
      Node1& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1, mitot = nxg + 2 * nghost;
      g.flags.assign(nxg + 2 * mbuff, UNSET);
      std::vector<double>* use;
      std::vector<double> tmpq;
      if (start_time + possk[lcheck] != g.time) {
        bound(g.time, g.q1, mitot, mptr);
        use = &g.q1;
      } else {
        use = &g.q2;
      }
      flagregions1(nxg, mbuff, g.xlo, hxposs[lcheck], lcheck, g.time, g.flags.data());
      bool keep = false;
      for (double f : g.flags) if (f == UNSET) { keep = true; break; }
      if (flag_gradient && keep) flag2refine1(nxg, mbuff, *use, g.flags.data());
    }
  }
  // projec1.f: cells under level lcheck+2's new grids (BADPRO where not flagged)
  void projec1(int level, Node1& g, int mbuff) {
    const int lrat2x = intratx[level] * intratx[level + 1];
    for (int mkid = newstl[level + 2]; mkid != 0; mkid = node[mkid].levelptr) {
      const Node1& k = node[mkid];
      int ist = (int)std::floor((float)k.ilo / (float)lrat2x);  // ikidlo/real(lrat2x): single precision
      int iend = (int)std::ceil((k.ihi + 1.0) / lrat2x) - 1;
      if (ibuff == 0) {
        if (ist * lrat2x == k.ilo) ist = ist - 1;
        if ((iend + 1) * lrat2x == k.ihi + 1) iend = iend + 1;
      }
      const int ixlo = std::max(ist, g.ilo - mbuff), ixhi = std::min(iend, g.ihi + mbuff);
      for (int i = ixlo; i <= ixhi; ++i) {
        double& f = g.flags[i - (g.ilo - mbuff)];
        if (f <= DONTFLAG) f = BADPRO;
      }
    }
  }
  // shiftset.f: every positive interior flag stamped over +-ibuff (the last one wins)
  void shiftset(Node1& g, int mbuff) {
    const int lo = g.ilo - mbuff;
    std::vector<double> copy(g.flags.size(), 0.0);
    for (int i = g.ilo; i <= g.ihi; ++i) {
      const double r = g.flags[i - lo];
      if (r > 0) for (int m = i - ibuff; m <= i + ibuff; ++m) copy[m - lo] = r;
    }
    g.flags = copy;
  }
  // setPhysBndryFlags.f
  void setPhysBndryFlags(std::vector<signed char>& f, int ilo, int ihi, int mbuff, int level) {
    const int lo = ilo - mbuff;
    if (ilo - mbuff < 0 && !xperdom) for (int i = ilo - mbuff; i <= -1; ++i) f[i - lo] = 1;
    if (ihi + mbuff >= iregsz[level] && !xperdom) for (int i = iregsz[level]; i <= ihi + mbuff; ++i) f[i - lo] = 1;
  }
  // griddomshrink.f: a cell stays where it and both neighbours are inside
  void griddomshrink(const std::vector<signed char>& in, int ilo, int ihi, int mbuff, std::vector<signed char>& out, int level) {
    const int lo = ilo - mbuff;
    out.assign(ihi - ilo + 1 + 2 * mbuff, 0);
    for (int i = ilo - mbuff + 1; i <= ihi + mbuff - 1; ++i) {
      out[i - lo] = in[i - lo];
      if (in[i - lo] <= 0 || in[i + 1 - lo] <= 0 || in[i - 1 - lo] <= 0) out[i - lo] = 0;
      out[0] = 0;
      out[ihi + mbuff - lo] = 0;
    }
    setPhysBndryFlags(out, ilo, ihi, mbuff, level);
  }
  // griddomup.f: the coarse domain flags onto the fine index range
  void griddomup(const std::vector<signed char>& c, int ilo, int ihi, int mbuff, int lev, int ilofine, int ihifine,
                 std::vector<signed char>& f) {
    const int lr = intratx[lev], clo = ilo - mbuff, flo = ilofine - mbuff;
    f.assign(ihifine - ilofine + 1 + 2 * mbuff, 0);
    for (int i = ilo; i <= ihi; ++i) {
      const int ifine = i * lr - 1;
      for (int mi = 1; mi <= lr; ++mi) {
        int iset = std::min(ifine + mi, ihifine + mbuff);
        iset = std::max(iset, ilofine - mbuff);
        f[iset - flo] = c[i - clo];
      }
    }
    for (int i = ihifine + 1; i <= ihifine + mbuff; ++i) f[i - flo] = c[i / lr - clo];
    for (int i = ilofine - mbuff; i <= ilofine - 1; ++i) f[i - flo] = c[i / lr - clo];
  }
  // setdomflags.f: the nesting domain of grid g (domflags2) from the base level's grids
  void setdomflags(Node1& g, int mbuff, int lbase, int lcheck) {
    int igridst[12], igridend[12];
    igridst[lcheck] = g.ilo; igridend[lcheck] = g.ihi;
    for (int lc = lcheck - 1; lc >= lbase; --lc) {
      const int ilo_c = (int)std::floor((double)igridst[lc + 1] / intratx[lc]);
      int ihi_c = (int)std::ceil((double)igridend[lc + 1] / intratx[lc]) - 1;
      if (ihi_c * intratx[lc] < igridend[lc + 1]) ihi_c = ihi_c + 1;
      igridend[lc] = ihi_c; igridst[lc] = ilo_c;
    }
    int ilo_c = igridst[lbase], ihi_c = igridend[lbase];
    std::vector<signed char> flags(ihi_c - ilo_c + 1 + 2 * mbuff, 0);
    const int lo = ilo_c - mbuff;
    int ist[3], iend[3], ishift[3];
    if (xperdom) {
      ist[0] = ilo_c - mbuff; ist[1] = 0; ist[2] = iregsz[lbase];
      iend[0] = -1; iend[1] = iregsz[lbase] - 1; iend[2] = ihi_c + mbuff;
      ishift[0] = iregsz[lbase]; ishift[1] = 0; ishift[2] = -iregsz[lbase];
    }
    for (int mb = lstart[lbase]; mb != 0; mb = node[mb].levelptr) {
      const int iblo = node[mb].ilo, ibhi = node[mb].ihi;
      if (xperdom) {
        for (int k = 0; k < 3; ++k) {
          const int i1 = std::max(ilo_c - mbuff, ist[k]), i2 = std::min(ihi_c + mbuff, iend[k]);
          if (!(i1 <= i2)) continue;
          const int ixlo = std::max(iblo, i1 + ishift[k]), ixhi = std::min(ibhi, i2 + ishift[k]);
          if (ixlo > ixhi) continue;
          for (int i = ixlo - ishift[k]; i <= ixhi - ishift[k]; ++i) flags[i - lo] = 1;
        }
      } else {
        const int ixlo = std::max(iblo, ilo_c - mbuff), ixhi = std::min(ibhi, ihi_c + mbuff);
        if (!(ixlo <= ixhi)) continue;
        for (int i = ixlo; i <= ixhi; ++i) flags[i - lo] = 1;
      }
    }
    setPhysBndryFlags(flags, ilo_c, ihi_c, mbuff, lbase);
    std::vector<signed char> icopy = flags;  // griddomcopy.f
    griddomshrink(icopy, ilo_c, ihi_c, mbuff, g.dom2, lbase);
    for (int lev = lbase + 1; lev <= lcheck; ++lev) {
      const int ilofine = igridst[lev], ihifine = igridend[lev];
      griddomup(g.dom2, ilo_c, ihi_c, mbuff, lev - 1, ilofine, ihifine, icopy);
      griddomshrink(icopy, ilofine, ihifine, mbuff, g.dom2, lev);
      ilo_c = ilofine; ihi_c = ihifine;
    }
  }
  // bufnst1.f: projection, buffer, count, nesting domain per grid
  int bufnst1(int lcheck, int lbase) {
    int numbad = 0;
    const int mbuff = std::max(nghost, ibuff + 1);
    for (int mptr : levelgrids[lcheck]) {
      Node1& g = node[mptr];
      if (lcheck + 2 <= mxnest) projec1(lcheck, g, mbuff);
      shiftset(g, mbuff);
      int numflagged = 0;
      for (double f : g.flags) if (f > DONTFLAG) ++numflagged;
      g.numflags = numflagged;
      numbad += numflagged;
      setdomflags(g, mbuff, lbase, lcheck);
    }
    return numbad;
  }
  // colate1.f with flagcheck.f and drivesort.f: flagged cells inside the nesting domain, as
  // cell centres i+.5 (periodic wrap), sorted and unique below level 6
  void colate1(std::vector<double>& badpts, int lcheck) {
    const int mbuff = std::max(nghost, ibuff + 1);
    badpts.clear();
    for (int mptr : levelgrids[lcheck]) {
      Node1& g = node[mptr];
      if (g.numflags != 0) {
        int imin = g.ilo - mbuff, imax = g.ihi + mbuff;
        if (!xperdom) { imin = std::max(imin, 0); imax = std::min(g.ihi + mbuff, iregsz[lcheck] - 1); }
        const int lo = g.ilo - mbuff;
        for (int i = imin; i <= imax; ++i)  // flagcheck.f
          if (g.flags[i - lo] > DONTFLAG && g.dom2[i - lo] != 1) g.flags[i - lo] = 0.;
        for (int i = imin; i <= imax; ++i) {
          if (g.flags[i - lo] < 0) continue;
          if (g.flags[i - lo] <= DONTFLAG) continue;
          int iwrap = i;
          if (xperdom) {
            if (i < 0) iwrap = i + iregsz[lcheck];
            if (i >= iregsz[lcheck]) iwrap = i - iregsz[lcheck];
          }
          badpts.push_back((double)iwrap + .5);
        }
      }
      g.flags.clear(); g.dom2.clear();
    }
    if (lcheck >= 6) return;
    // drivesort.f
    const int npts = (int)badpts.size();
    const int isize = iregsz[lcheck];
    std::vector<long long> iflags(npts + 1);
    std::vector<int> ix(npts + 1);
    for (int k = 1; k <= npts; ++k) iflags[k] = (int)(badpts[k - 1] - .5) + mbuff;
    qsorti(ix, npts, iflags);
    std::vector<double> out;
    int k = 1;
    while (k <= npts) {
      const long long ie = iflags[ix[k]];
      out.push_back((double)(ie % (isize + 2 * mbuff)) + .5 - mbuff);
      k = k + 1;
      while (k <= npts && iflags[ix[k]] == iflags[ix[k - 1]]) k = k + 1;
    }
    badpts = out;
  }

  // ================================================================ clustering
  // moment.f
  static void moment(int rect[2], const double* bp, int npt, double& usage) {
    double emx1 = bp[0], emn1 = emx1;
    for (int p = 0; p < npt; ++p) {
      if (bp[p] > emx1) emx1 = bp[p];
      if (bp[p] < emn1) emn1 = bp[p];
    }
    rect[0] = (int)std::lround(emn1 - .5);
    rect[1] = (int)std::lround(emx1 - .5);
    usage = (double)npt / (double)(rect[1] - rect[0] + 1);
  }
  // signs.f + findcut.f over points [ist, iend) of badpts: index 0 means no cut
  static int findcut(const double* bp, int ist, int iend, int idim) {
    std::vector<int> iscr(idim + 2, 0);
    int ilo = 1, ihi = idim;
    for (int p = ist; p < iend; ++p) { const int iloc = (int)(bp[p] + 1.1); iscr[iloc] += 1; }
    for (int ipt = 1; ipt <= idim; ++ipt) if (iscr[ipt] != 0) { ilo = ipt; break; }
    for (int ipt = 1; ipt <= idim; ++ipt) if (iscr[idim + 1 - ipt] != 0) { ihi = idim + 1 - ipt; break; }
    for (int i = ilo; i <= ihi; ++i) if (iscr[i] == 0) return i;
    int ipre = iscr[ilo];
    for (int i = ilo + 1; i <= ihi - 1; ++i) {
      const int icur = iscr[i];
      iscr[i] = iscr[i + 1] - 2 * icur + ipre;
      ipre = icur;
    }
    int locmaxi = 0, indexi = 0;
    const int imid = (ilo + ihi) / 2;
    for (int i = ilo + 2; i <= ihi - 2 + 1; ++i) {
      const int t1 = iscr[i - 1], t2 = iscr[i];
      const int locdif = std::abs(t1 - t2);
      if (t1 * t2 < 0) {
        if (locdif > locmaxi) { locmaxi = locdif; indexi = i; }
        else if (locdif == locmaxi) { if (std::abs(i - imid) < std::abs(indexi - imid)) indexi = i; }
      }
    }
    return locmaxi < 2 ? 0 : indexi;
  }
  // smartbis.f: bisect clusters until their use is at least cutoff (badpts reordered)
  void smartbis(std::vector<double>& bp, int npts, std::vector<int>& numptc, int& nclust, int idim) {
    nclust = 1;
    numptc.assign(1, npts);
    int icl = 0, ist = 0, iend = npts;  // cluster icl holds points [ist, iend)
    while (true) {
      int rect[2]; double usenew;
      moment(rect, bp.data() + ist, numptc[icl], usenew);
      bool next = usenew >= cut;
      int index = 0;
      if (!next) {
        index = findcut(bp.data(), ist, iend, idim);
        if (index == 0) next = true;
      }
      if (next) {
        ++icl;
        if (icl >= nclust) break;
        ist = iend;
        iend = ist + numptc[icl];
        continue;
      }
      const double fmid = index - .5;
      int itop = ist - 1, ibot = iend, i = ist;
      while (true) {
        if (bp[i] < fmid) {
          ibot = ibot - 1;
          std::swap(bp[ibot], bp[i]);
          if (itop + 1 < ibot) continue;
          break;
        }
        itop = itop + 1;
        if (itop + 1 >= ibot) break;
        i = i + 1;
      }
      numptc[icl] = itop - ist + 1;
      numptc.insert(numptc.begin() + icl + 1, iend - ibot);
      nclust = nclust + 1;
      iend = itop + 1;
    }
  }
  // baseCheck.f: is [ilo,ihi] of a new grid (coarsened to lbase, grown by one) covered by
  // the base level's grids grown by thisBuff (and the physical boundary)?
  bool baseCheck(int mnew, int lbase, int ilo, int ihi, int thisBuff) {
    const int levnew = node[mnew].level;
    const bool borderx = ilo == 0 || ihi == iregsz[levnew] - 1;
    int iclo = ilo, ichi = ihi;
    for (int lev = levnew - 1; lev >= lbase; --lev) {
      iclo = iclo / intratx[lev]; ichi = ichi / intratx[lev];
      iclo = iclo - 1; ichi = ichi + 1;
    }
    if (!(xperdom && borderx)) { iclo = std::max(iclo, 0); ichi = std::min(ichi, iregsz[lbase] - 1); }
    std::vector<double> a(ichi - iclo + 1, 0.0);
    auto A = [&](int i) -> double& { return a[i - iclo]; };
    if (ilo == 0 && !xperdom) { A(iclo) = 1.; A(iclo + 1) = 1.; }
    if (ihi == iregsz[levnew] - 1 && !xperdom) { A(ichi) = 1.; A(ichi - 1) = 1.; }
    for (int mptr = lstart[lbase]; mptr != 0; mptr = node[mptr].levelptr) {
      const int iblo = node[mptr].ilo - thisBuff, ibhi = node[mptr].ihi + thisBuff;
      if (!(xperdom && borderx)) {
        const int ixlo = std::max(iclo, iblo), ixhi = std::min(ichi, ibhi);
        for (int ix = ixlo; ix <= ixhi; ++ix) A(ix) = 1.;
        continue;
      }
      int ist[3] = {iclo, 0, iregsz[lbase]}, iend[3] = {-1, iregsz[lbase] - 1, ichi};
      int ishift[3] = {iregsz[lbase], 0, -iregsz[lbase]};  // setIndices.f (periodic)
      for (int k = 0; k < 3; ++k) {
        const int i1 = std::max(iclo, ist[k]), i2 = std::min(ichi, iend[k]);
        if (!(i1 <= i2)) continue;
        const int ixlo = std::max(i1 + ishift[k], iblo), ixhi = std::min(i2 + ishift[k], ibhi);
        for (int ix = ixlo; ix <= ixhi; ++ix) A(ix - ishift[k]) = 1.;
      }
    }
    for (int i = iclo; i <= ichi; ++i) if (A(i) == 0) return false;
    return true;
  }
  // nestck1.f: a new grid not nested in the base level splits its cluster in two
  bool nestck1(int mnew, int lbase, double* bp, int npts, std::vector<int>& numptc, int icl, int& nclust) {
    if (lbase == 1) return true;
    const int levnew = node[mnew].level;
    const int lratiox = intratx[levnew - 1];
    if (baseCheck(mnew, lbase, node[mnew].ilo, node[mnew].ihi, 0)) return true;
    if (npts <= 1) throw std::runtime_error("nestck1: a cluster of one point is not nested");
    double rmid = (node[mnew].ihi + node[mnew].ilo + 1) / 2.;
    rmid = rmid / lratiox;
    int ipt = 0, ntop = npts - 1;  // 0-based
    while (true) {
      if (bp[ipt] < rmid) {
        ipt = ipt + 1;
        if (ipt <= ntop) continue;
        break;
      }
      std::swap(bp[ipt], bp[ntop]);
      ntop = ntop - 1;
      if (ipt <= ntop) continue;
      break;
    }
    const int nlow = ntop + 1;
    numptc.insert(numptc.begin() + icl + 1, npts - nlow);
    numptc[icl] = nlow;
    nclust = nclust + 1;
    return false;
  }
  // grdfit1.f: flag, cluster and fit the new grids of level lcheck+1
  void grdfit(int lbase, int lcheck, double t, double start_time) {
    flagger(lcheck, start_time);
    const int numbad = bufnst1(lcheck, lbase);
    std::vector<double> bp;
    if (numbad > 0) colate1(bp, lcheck);
    else for (int m : levelgrids[lcheck]) { node[m].flags.clear(); node[m].dom2.clear(); }
    const int npts = (int)bp.size();
    if (npts == 0) return;
    const int levnew = lcheck + 1;
    const double hxfine = hxposs[levnew];
    std::vector<int> numptc;
    int nclust = 0;
    smartbis(bp, npts, numptc, nclust, iregsz[lcheck]);
    int ibase = 0, icl = 0, prvptr = 0;
    while (icl < nclust) {
      const int mnew = nodget();
      while (true) {
        int rect[2]; double usage;
        moment(rect, bp.data() + ibase, numptc[icl], usage);
        Node1& n = node[mnew];
        n.ilo = rect[0] * intratx[lcheck];
        n.ihi = (rect[1] + 1) * intratx[lcheck] - 1;
        n.xlo = n.ilo * hxfine + xlower;
        n.xhi = (n.ihi + 1) * hxfine + xlower;
        n.level = levnew;
        n.time = t;
        if (nestck1(mnew, lbase, bp.data() + ibase, numptc[icl], numptc, icl, nclust)) break;
      }
      if (newstl[levnew] == 0) newstl[levnew] = mnew;
      else node[prvptr].levelptr = mnew;
      prvptr = mnew;
      ibase = ibase + numptc[icl];
      icl = icl + 1;
    }
    birect(newstl[levnew]);
  }

  // filval.f90: a new grid's values, the old grids' where they were, else interpolated
  void filval(int mptr, int level, double t) {
    Node1& g = node[mptr];
    const int r = intratx[level - 1];
    const double dx = hxposs[level], dx_coarse = dx * r;
    const double xl = g.xlo - dx_coarse, xr = g.xhi + dx_coarse;
    const int iclo = g.ilo / r - 1, ichi = (g.ihi + 1) / r - 1 + 1;
    const int mic = (g.ihi - g.ilo + 1) / r + 2;
    const int mitot = mitot_of(mptr);
    std::vector<double> valc((size_t)nvar * mic, 0.0);
    const bool sticksoutxfine = g.ilo < 0 || g.ihi >= iregsz[level];
    const bool sticksoutxcrse = iclo < 0 || ichi >= iregsz[level - 1];
    if (xperdom && sticksoutxcrse) preicall(valc, iclo, ichi, level - 1, true);
    else icall(valc, iclo, ichi, level - 1, 1);
    bc1amr(valc, mic, dx_coarse, xl, xr);
    std::vector<double>& val = g.q1;
    for (int i = 1; i <= mitot; ++i) Q(val, 1, i) = NEEDS_TO_BE_SET;
    if (xperdom && sticksoutxfine) preicall(val, g.ilo - nghost, g.ihi + nghost, level, true);
    else icall(val, g.ilo - nghost, g.ihi + nghost, level, 1);
    std::vector<double> setflags(mitot + 1);
    for (int i = 1; i <= mitot; ++i) setflags[i] = Q(val, 1, i);
    for (int i = 2; i <= mic - 1; ++i)
      for (int iv = 1; iv <= nvar; ++iv) {
        const double s1p = Q(valc, iv, i + 1) - Q(valc, iv, i), s1m = Q(valc, iv, i) - Q(valc, iv, i - 1);
        double slopex = std::min(std::fabs(s1p), std::fabs(s1m)) * orc1_sign(1.0, Q(valc, iv, i + 1) - Q(valc, iv, i - 1));
        if (s1m * s1p <= 0.0) slopex = 0.0;
        for (int ico = 1; ico <= r; ++ico) {
          const double xoff = ((double)ico - 0.5) / r - 0.5;
          const int ifine = (i - 2) * r + nghost + ico;
          if (setflags[ifine] == NEEDS_TO_BE_SET) Q(val, iv, ifine) = Q(valc, iv, i) + xoff * slopex;
        }
      }
  }
  // gfixup.f: registers and old stores released, new grids filled, old grids dropped
  void gfixup(int lbase, int lfnew) {
    putsp(lbase, lbase);
    for (int level = lbase + 1; level <= lfine; ++level) {
      putsp(lbase, level);
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].q2.clear(); node[m].has_q2 = false; }
    }
    const double t = node[lstart[lbase]].time;
    for (int lcheck = lbase + 1; lcheck <= mxnest; ++lcheck) {
      std::vector<int> nl;
      for (int m = newstl[lcheck]; m != 0; m = node[m].levelptr) nl.push_back(m);
      for (int m : nl) node[m].q1.assign((size_t)nvar * mitot_of(m), 0.0);
      for (int m : nl) filval(m, lcheck, t);
      int mptr = lstart[lcheck];
      while (mptr != 0) {
        const int mold = mptr;
        mptr = node[mptr].levelptr;
        node[mold].q1.clear(); node[mold].bnd.clear();
        putnod(mold);
      }
      lstart[lcheck] = newstl[lcheck];
    }
    lfine = lfnew;
    const int levend = std::min(lfine, mxnest - 1);
    for (int level = lbase + 1; level <= levend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        node[m].q2.assign((size_t)nvar * mitot_of(m), 0.0);
        node[m].has_q2 = true;
      }
  }
  // regrid.f
  void regrid(int lbase, double start_time) {
    int lcheck = std::min(lfine, mxnest - 1);
    int lfnew = lbase;
    for (int i = 1; i <= mxnest; ++i) newstl[i] = 0;
    const double t = node[lstart[lbase]].time;
    while (lcheck >= lbase) {
      grdfit(lbase, lcheck, t, start_time);
      if (newstl[lcheck + 1] != 0) lfnew = std::max(lcheck + 1, lfnew);
      lcheck = lcheck - 1;
    }
    gfixup(lbase, lfnew);
    for (int level = lbase; level <= lfine - 1; ++level) { prepf(level + 1); prepc(level); }
    for (int levnew = lbase + 1; levnew <= mxnest; ++levnew) {
      int ng = 0;
      for (int m = lstart[levnew]; m != 0; m = node[m].levelptr) ++ng;
      numgrids[levnew] = ng;
      if (ng > 1) arrangeGrids(levnew, ng);
    }
    makeGridList(lbase);
    for (int levnew = lbase + 1; levnew <= lfine; ++levnew) makeBndryList(levnew);
  }

  // ================================================================ start-up
  // ginit.f: storage and initial values of the grids msave..; first: new grids
  void ginit(int msave, bool first, double start_time) {
    if (msave == 0) return;
    for (int mptr = msave; mptr != 0; mptr = node[mptr].levelptr) {
      Node1& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1, mitot = nxg + 2 * nghost;
      std::vector<double>* dst;
      if (first) {
        g.q1.assign((size_t)nvar * mitot, 0.0);
        if (g.level < mxnest) { g.q2.assign((size_t)nvar * mitot, 0.0); g.has_q2 = true; }
        g.time = start_time;
        dst = &g.q1;
      } else {
        dst = &g.q2;
      }
      qinit(nghost, nxg, g.xlo, hxposs[g.level], dst->data());
    }
  }
  // domain.f
  void domain(double start_time) {
    mstart = nodget();
    Node1& g = node[mstart];
    g.xlo = xlower; g.xhi = xupper; g.level = 1; g.levelptr = 0;
    lstart[1] = mstart;
    g.ilo = 0; g.ihi = nx - 1;
    lfine = 1;
    birect(mstart);
    ginit(mstart, true, start_time);
    int ng = 0;
    for (int m = lstart[1]; m != 0; m = node[m].levelptr) ++ng;
    numgrids[1] = ng;
    if (ng > 1) arrangeGrids(1, ng);
    makeGridList(0);
    makeBndryList(1);
    iregsz[1] = nx;
    for (int level = 2; level <= mxnest; ++level) {
      iregsz[level] = iregsz[level - 1] * intratx[level - 1];
      possk[level] = possk[level - 1] / (double)kratio[level - 1];
    }
  }
  // setgrd.f (no Richardson estimation)
  void setgrd(double start_time) {
    if (mxnest == 1) return;
    int levnew = 2;
    const double t = start_time;
    while (levnew <= mxnest) {
      const int levold = levnew - 1;
      if (lstart[levold] == 0) break;
      const int lbase = levold;
      int lfnew = lbase;
      grdfit(lbase, levold, t, start_time);
      if (newstl[levnew] != 0) lfnew = levnew;
      ginit(newstl[levnew], true, start_time);
      lstart[levnew] = newstl[levnew];
      lfine = lfnew;
      ginit(lstart[levold], false, start_time);
      int ng = 0;
      for (int m = lstart[levnew]; m != 0; m = node[m].levelptr) ++ng;
      numgrids[levnew] = ng;
      if (ng > 1) arrangeGrids(levnew, ng);
      makeGridList(lbase);
      makeBndryList(levnew);
      levnew = levnew + 1;
    }
    for (int lev = 1; !(lev == mxnest || lev > lfine); ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
        std::swap(node[m].q1, node[m].q2);
        node[m].time = start_time;
      }
    for (int level = 1; level <= lfine - 1; ++level) update(lfine - level);
    for (int level = 1; level <= lfine - 1; ++level) { prepf(level + 1); prepc(level); }
  }

  // ================================================================ gauges, mass, output
  // gauges_module.f90 (setbestsrc): the last grid, finest level last, that holds the gauge
  void setbestsrc() {
    mbestsrc.assign(gauges.size(), 0);
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr)
        for (size_t i = 0; i < gauges.size(); ++i)
          if (gauges[i].x >= node[m].xlo && gauges[i].x <= node[m].xhi) mbestsrc[i] = m;
  }
  double conck(int level) {
    double totmass = 0.0;
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
      const int mitot = mitot_of(m);
      for (int i = nghost + 1; i <= mitot - nghost; ++i) totmass = totmass + Q(node[m].q1, 1, i);
    }
    return totmass * hxposs[level];
  }
  // valout.f90 (1D): ASCII fort.q / fort.t, or binary fort.q headers + fort.b whole arrays
  void valout(int lbeg, int lend, double t) {
    const bool binary = output_format == 3;
    if (!binary)
      for (int level = lbeg; level <= lend; ++level)
        for (int m = lstart[level]; m != 0; m = node[m].levelptr)
          for (int i = nghost + 1; i <= mitot_of(m) - nghost; ++i)
            for (int iv = 1; iv <= nvar; ++iv) if (std::fabs(Q(node[m].q1, iv, i)) < 1e-90) Q(node[m].q1, iv, i) = 0.0;
    if (write_output) {
      char fn[64];
      std::snprintf(fn, sizeof(fn), "/fort.q%04d", matlabu);
      FILE* f = std::fopen((outdir + fn).c_str(), "w");
      FILE* b = nullptr;
      if (binary) { std::snprintf(fn, sizeof(fn), "/fort.b%04d", matlabu); b = std::fopen((outdir + fn).c_str(), "wb"); }
      int ngrids = 0;
      for (int level = lbeg; level <= lend; ++level)
        for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
          ++ngrids;
          Node1& g = node[m];
          std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n%6d                 mx\n", m, level, g.ihi - g.ilo + 1);
          std::fprintf(f, "%s    xlow\n%s    dx\n\n", fmtE(g.xlo, 26, 16).c_str(), fmtE(hxposs[level], 26, 16).c_str());
          if (binary) {
            std::fwrite(g.q1.data(), sizeof(double), g.q1.size(), b);
          } else {
            for (int i = nghost + 1; i <= mitot_of(m) - nghost; ++i) {
              for (int iv = 1; iv <= nvar; ++iv) std::fputs(fmtE(Q(g.q1, iv, i), 26, 16).c_str(), f);
              std::fputc('\n', f);
            }
            std::fputs("  \n", f);
          }
        }
      std::fclose(f);
      if (b) std::fclose(b);
      std::snprintf(fn, sizeof(fn), "/fort.t%04d", matlabu);
      f = std::fopen((outdir + fn).c_str(), "w");
      std::fprintf(f, "%s    time\n%6d                 meqn\n%6d                 ngrids\n%6d                 naux\n%6d                 ndim\n%6d                 nghost\n\n",
                   fmtE(t, 18, 8).c_str(), nvar, ngrids, naux, 1, nghost);
      std::fclose(f);
    }
    matlabu = matlabu + 1;
  }

  // ================================================================ tick.f
  bool tick_started = false;
  int tk_nextout = 0, max_cycles = 0;
  double tk_tlevel[12] = {0};
  void tick(double start_time) {
    double dtnew[12];
    double* tlevel = tk_tlevel;
    int ntogo[12];
    int cycles = 0;
    setbestsrc();
    int nextout = 0;
    if (iout == 0) { iout = IINFINITY; nextout = 0; if (nout > 0) nextout = 1; }
    if (tick_started) nextout = tk_nextout;
    if (!tick_started) for (int i = 1; i <= mxnest; ++i) tlevel[i] = time;
    tick_started = true;
    while (!(ncycle >= nstop || time >= tfinal)) {
      const double outtime = nout > 0 ? ((nextout <= nout) ? tout[nextout - 1] : RINFINITY) : tfinal;
      bool dumpout = false;
      if (time < outtime && time + (double)1.001f * possk[1] >= outtime) {
        possk[1] = outtime - time;
        for (int i = 2; i <= mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
        if (nout > 0) { nextout = nextout + 1; dumpout = true; }
      }
      int level = 1;
      ntogo[level] = 1;
      for (int i = 1; i <= 10; ++i) dtnew[i] = RINFINITY;
      while (true) {
        int lbase = -1;
        if (icheck[level] >= kcheck) lbase = level;
        else if (level + 1 >= mxnest) lbase = -1;
        else if (icheck[level + 1] >= kcheck) lbase = level + 1;
        else if (level + 2 >= mxnest) lbase = -1;
        else if (icheck[level + 2] >= kcheck) lbase = level + 2;
        if (lbase > 0) {
          if (!(lbase == mxnest || lbase > lfine)) {
            regrid(lbase, start_time);
            setbestsrc();
          }
          for (int i = lbase; i <= lfine; ++i) icheck[i] = 0;
          for (int i = lbase + 1; i <= lfine; ++i) tlevel[i] = tlevel[lbase];
        }
        double dtlevnew;
        advanc(level, dtlevnew);
        ntogo[level] = ntogo[level] - 1;
        dtnew[level] = std::min(dtnew[level], dtlevnew);
        tlevel[level] = tlevel[level] + possk[level];
        icheck[level] = icheck[level] + 1;
        if (level < lfine) {
          level = level + 1;
          if (((possk[level - 1] - dtnew[level - 1]) / dtnew[level - 1]) > (double)0.05f) {
            const double dttemp = dtnew[level - 1] / kratio[level - 1];
            ntogo[level] = (int)((tlevel[level - 1] - tlevel[level]) / dttemp + (double)0.9f);
          } else {
            ntogo[level] = kratio[level - 1];
          }
          possk[level] = possk[level - 1] / ntogo[level];
          continue;
        }
        bool done = false;
        while (true) {
          if (level == 1) { done = true; break; }
          if (ntogo[level] > 0) {
            while ((possk[level] - dtnew[level]) / dtnew[level] > (double)0.05f) {
              ntogo[level] = ntogo[level] + 1;
              possk[level] = (tlevel[level - 1] - tlevel[level]) / ntogo[level];
            }
            break;
          }
          level = level - 1;
          update(level);
        }
        if (done) break;
      }
      time = time + possk[1];
      ncycle = ncycle + 1;
      conck(1);
      if (vtime) {
        for (int i = 2; i <= lfine; ++i) {
          const int ii = lfine + 1 - i;
          dtnew[ii] = std::min(dtnew[ii], dtnew[ii + 1] * kratio[ii]);
        }
        dtnew[1] = std::min(dtnew[1], dt_max);
        possk[1] = dtnew[1];
        for (int i = 2; i <= mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
      }
      if ((ncycle % iout == 0) || dumpout) valout(1, lfine, time);
      ++cycles;
      if (max_cycles > 0 && cycles >= max_cycles) break;
    }
    tk_nextout = nextout;
  }

  // amr1.f90 start-up
  void init(const std::string& dir) {
    read_input(dir);
    hxposs[1] = (xupper - xlower) / nx;
    matlabu = output_t0 ? 0 : 1;
    possk[1] = dt_initial;
    node.assign(2, Node1());
    node.resize(10001);
    for (int k = 1; k <= 10000; ++k) node[k].nextfree = k + 1;
    node[10000].nextfree = 0;
    ndfree = 1;
    for (int level = 2; level <= mxnest; ++level) hxposs[level] = hxposs[level - 1] / (double)intratx[level - 1];
    domain(t0);
    record_gauges = false;
    setgrd(t0);
    record_gauges = true;
    time = t0;
    tmass0 = conck(1);
    if (output_t0) valout(1, lfine, time);
  }
};

// gauges_module.f90 (update_gauges): linear interpolation between the two cells around
// the gauge, in the grid that is its best source
void Amr1::update_gauges(std::vector<double>& q, double xlow, int mitot, int mptr) {
  (void)mitot;
  if (!record_gauges) return;
  const double tgrid = node[mptr].time;
  const int level = node[mptr].level;
  const double hx = hxposs[level];
  for (size_t i = 0; i < gauges.size(); ++i) {
    Gauge1& g = gauges[i];
    if (mptr != mbestsrc[i]) continue;
    if (tgrid < g.t_start || tgrid > g.t_end) continue;
    const int iindex = (int)(.5 + (g.x - xlow) / hx);
    const double xcent = xlow + (iindex - .5) * hx;
    const double xoff = (g.x - xcent) / hx;
    Sample1 smp; smp.level = level; smp.t = tgrid;
    for (int iv = 1; iv <= nvar; ++iv) {
      double v = (1. - xoff) * Q(q, iv, iindex) + xoff * Q(q, iv, iindex + 1);
      if (std::fabs(v) < 1e-90) v = 0.0;
      smp.v.push_back(v);
    }
    g.data.push_back(smp);
  }
}

}  // namespace orc1

// ============================================================== C entry points (tests only)
using orc1::Amr1;
extern "C" {

void* oracle1d_create(const char* dir, const char* outdir, int write_output) {
  try {
    Amr1* a = new Amr1();
    a->outdir = outdir ? outdir : "";
    a->write_output = write_output != 0;
    a->init(dir);
    return a;
  } catch (std::exception& e) {
    std::fprintf(stderr, "oracle1d_create: %s\n", e.what());
    return nullptr;
  }
}
void oracle1d_destroy(void* h) { delete (Amr1*)h; }
int oracle1d_run(void* h, int max_cycles) {
  Amr1* a = (Amr1*)h;
  try {
    a->max_cycles = max_cycles;
    a->tick(a->t0);
    return 0;
  } catch (std::exception& e) {
    std::fprintf(stderr, "oracle1d_run: %s\n", e.what());
    return 1;
  }
}
double oracle1d_time(void* h) { return ((Amr1*)h)->time; }
double oracle1d_cell_updates(void* h) { return ((Amr1*)h)->rvol; }
double oracle1d_mass(void* h) { return ((Amr1*)h)->conck(1); }
// rows (grid_number, level, ilo, ihi) in output order
int oracle1d_grids(void* h, int* out, int cap) {
  Amr1* a = (Amr1*)h;
  int n = 0;
  for (int level = 1; level <= a->lfine; ++level)
    for (int m = a->lstart[level]; m != 0; m = a->node[m].levelptr) {
      if (out && n < cap) { int* r = out + 4 * n; r[0] = m; r[1] = level; r[2] = a->node[m].ilo; r[3] = a->node[m].ihi; }
      ++n;
    }
  return n;
}
// interior values of every grid in the order of oracle1d_grids, layout [m][i] per grid
long oracle1d_values(void* h, double* out, long cap) {
  Amr1* a = (Amr1*)h;
  long n = 0;
  for (int level = 1; level <= a->lfine; ++level)
    for (int m = a->lstart[level]; m != 0; m = a->node[m].levelptr) {
      const int mitot = a->mitot_of(m), ng = a->nghost;
      for (int iv = 1; iv <= a->nvar; ++iv)
        for (int i = ng + 1; i <= mitot - ng; ++i) {
          if (out && n < cap) out[n] = a->node[m].q1[(iv - 1) + (size_t)a->nvar * (i - 1)];
          ++n;
        }
    }
  return n;
}
// gauge samples: rows (gauge_num, level, t, q1..qnvar)
int oracle1d_gauges(void* h, double* out, int cap_rows) {
  Amr1* a = (Amr1*)h;
  int n = 0;
  const int w = 3 + a->nvar;
  for (auto& g : a->gauges)
    for (auto& s : g.data) {
      if (out && n < cap_rows) {
        double* r = out + (size_t)w * n;
        r[0] = g.num; r[1] = s.level; r[2] = s.t;
        for (int k = 0; k < a->nvar; ++k) r[3 + k] = s.v[k];
      }
      ++n;
    }
  return n;
}

}  // extern "C"
