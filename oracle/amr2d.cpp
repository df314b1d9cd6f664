// Oracle (test infrastructure only): CPU FP64 restatement of AMRClaw's 2D
// per-level patch-advance path, used as the parity checker and the CPU
// baseline. The GPU product (amrclaw_b200) never loads this code.
//
// Each routine follows the reference routine named in its comment, with the
// same loop nesting and accumulation order (compile with -ffp-contract=off so
// no fused multiply-add changes a rounding):
//   patch step      src/2d/stepgrid.f:24-232, step2.f90:7-169, flux2.f:25-237,
//                   inlinelimiter.f:4-108
//   level advance   src/2d/advanc.f:10-142 (advanc), :170-291 (par_advanc)
//   ghost fill      src/2d/bound.f90:51-158, filpatch.f90:71-355,
//                   prefilp.f90:18-276, intfil.f90:98-311, trimbd.f90:32-97,
//                   bc2amr.f90:84-297, init_bndryList.f:50-107
//   conservation    saveqc.f:13-109, cstore.f:4-63, icall.f:8-91,
//                   preicall.f:4-190, qad.f:9-360, fluxsv.f:10-109,
//                   fluxad.f:7-96, update.f:16-189, upbnd.f:18-127,
//                   prepf.f:18-53, prepc.f:11-157, setuse.f:61-213, putsp.f:6-42
//   regrid          regrid.f:4-169, grdfit2.f:20-150, flglvl2.f:24-107,
//                   flagger.f:31-180, flagregions2.f90:40-119,
//                   flag2refine2.f90:53-124, bufnst2.f:15-180, projec2.f:51-220,
//                   shiftset2.f:25-71, setdomflags.f:22-207,
//                   griddomshrink.f:24-82, griddomup.f:16-116,
//                   setPhysBndryFlags.f:28-78, setIndices.f:4-59,
//                   colate2.f:10-200, flagcheck.f:9-40, drivesort.f:7-62,
//                   quick_sort1.f:22-167, smartbis.f:25-177, signs.f:16-71,
//                   findcut.f:7-130, moment.f:16-75, nestck2.f:37-176,
//                   baseCheck.f:19-240, birect.f:10-120, gfixup.f:6-218,
//                   filval.f90:3-214, intcopy.f:12-71, preintcopy.f:4-166,
//                   nodget.f:10-154, putnod.f:5-21
//   driver          amr2.f90:140-625, domain.f:4-110, setgrd.f:4-142,
//                   ginit.f:17-86, stst1.f:4-94, tick.f:4-391, conck.f:6-73
//   output          valout.f90:8-397, gauges_module.f90:255-500
//
// Riemann solvers and problem plugins (qinit, flag2refine variants) are in
// riemann2d.hpp / below; the reference takes those from un-vendored
// clawpack/riemann and per-application sources.
#include "common.hpp"
#include "riemann2d.hpp"
#include <algorithm>
#include <functional>
#include <memory>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const double UNSET = -1.0, DONTFLAG = 0.0, DOFLAG = 2.0, BADPRO = 3.0;
static const double NEEDS_TO_BE_SET = (double)10.e33f;  // default-real literal in amr_module.f90:170
static const double RINFINITY = (double)10.e32f;        // amr_module.f90:171
static const int IINFINITY = 999999999;
static const int HORIZONTAL = 1, VERTICAL = 2;

struct Region { int minlevel, maxlevel; double tlow, thi, xlow, xhi, ylow, yhi; };
struct GaugeSample { int level; double t; std::vector<double> v; };
struct Gauge {
  int num; double x, y, t_start, t_end, last_time, min_inc;
  std::vector<GaugeSample> data;
};

struct Node2 {
  int ilo = 0, ihi = 0, jlo = 0, jhi = 0, level = 0, levelptr = 0, nextfree = 0;
  int numflags = 0;
  double xlo = 0, xhi = 0, ylo = 0, yhi = 0, time = 0;
  std::vector<double> q1, q2, aux;  // store1, store2, storeaux  (nvar, mitot, mjtot)
  bool has_q2 = false;
  std::vector<double> ffl;          // ffluxptr: svdflx(nvar,lenbc) qc1d(nvar,lenbc) auxc1d(naux,lenbc)
  bool has_ffl = false;
  std::vector<int> listbc;          // cfluxptr: listbc(5,maxsp)
  bool has_cfl = false;
  std::vector<double> flags;        // storeflags (mibuff, mjbuff)
  std::vector<signed char> dom1, dom2;  // domflags_base, domflags2
  std::vector<int> bnd;             // bndList traversal order
};

// A Fortran array val(nvar, nrow, ncol) with 1-based indices.
struct FArr {
  double* p; int nvar, nrow, ncol;
  double& operator()(int m, int i, int j) const { return p[(m - 1) + nvar * ((i - 1) + (size_t)nrow * (j - 1))]; }
};

struct Amr2 {
  // ---------------- input (claw.data / amr.data / regions / gauges / setprob)
  double xlower, ylower, xupper, yupper;
  int nx, ny, nvar, mwaves, naux;
  double t0;
  int output_style = 1, nout = 0, iout = 0, nstop = IINFINITY;
  double tfinal = 0; bool output_t0 = true;
  std::vector<double> tout;
  int output_format = 1;
  std::vector<int> output_aux_components;
  bool output_aux_onlyonce = true;
  double dt_initial, dt_max, cflv1, cfl;
  int nv1; bool vtime;
  int method[8] = {0};
  int dimensional_split = 0, mcapa = 0;
  bool use_fwaves = false;
  std::vector<int> mthlim;
  int nghost = 2;
  int mthbc[5] = {0};
  bool xperdom = false, yperdom = false, spheredom = false;
  int mxnest = 1;
  int intratx[12], intraty[12], kratio[12];
  std::vector<std::string> auxtype;
  bool flag_richardson = false, flag_gradient = true;
  double tol = -1, tolsp = 0.05, cut = 0.7;
  int kcheck = 2, ibuff = 3;
  int max1d = 60;
  std::vector<Region> regions;
  std::vector<Gauge> gauges;
  ProbParams prob;
  std::string problem;
  double prob_x0 = 0.1, prob_x1 = 0.6, prob_y0 = 0.1, prob_y1 = 0.6, prob_width = 0.2;
  double ann[8] = {0};  // advection_annulus: A1, beta1, x1, y1, A2, beta2, x2, y2 (setprob.f)
  int flag_component = 0;  // 0 = all components (flag2refine2.f90 default), else one component

  // ---------------- state (amr_module)
  std::vector<Node2> node;
  int ndfree = 1, mstart = 0;
  int lfine = 1;
  int lstart[12] = {0}, newstl[12] = {0}, numgrids[12] = {0}, listsp[12] = {0};
  int iregsz[12], jregsz[12], icheck[12] = {0};
  double hxposs[12], hyposs[12], possk[12];
  std::vector<int> levelgrids[12];   // listOfGrids segments
  double cfl_level = 0, cflmax = 0;
  double rvol = 0, rvoll[12] = {0};
  double tmass0 = 0, lastmass = 0;
  int matlabu = 0;
  std::string outdir;
  bool write_output = false;
  bool record_gauges = true;
  int nthreads = 1;
  std::vector<int> mbestsrc;
  double time = 0;
  int ncycle = 0;

  // ========================================================== input parsing
  void read_input(const std::string& dir) {
    DataFile c, a, r, g, s;
    if (!c.load(dir + "/claw.data")) throw std::runtime_error("cannot read claw.data");
    if (!a.load(dir + "/amr.data")) throw std::runtime_error("cannot read amr.data");
    xlower = c.d("lower", 0); ylower = c.d("lower", 1);
    xupper = c.d("upper", 0); yupper = c.d("upper", 1);
    nx = c.i("num_cells", 0); ny = c.i("num_cells", 1);
    nvar = c.i("num_eqn"); mwaves = c.i("num_waves"); naux = c.i("num_aux");
    t0 = c.d("t0");
    output_style = c.i("output_style");
    if (output_style == 1) {
      nout = c.i("num_output_times"); tfinal = c.d("tfinal"); output_t0 = c.b("output_t0");
      iout = 0;
    } else if (output_style == 2) {
      auto& v = c.get("output_times");
      nout = (int)v.size();
      for (auto& x : v) tout.push_back(DataFile::tod(x));
      output_t0 = (tout[0] == t0);
      if (output_t0) { tout.erase(tout.begin()); nout -= 1; }
      iout = 0; tfinal = tout.back();
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
    if (naux > 0 && c.has("output_aux_components")) {
      for (int k = 0; k < naux; ++k) output_aux_components.push_back(c.i("output_aux_components", k));
      output_aux_onlyonce = c.has("output_aux_onlyonce") ? c.b("output_aux_onlyonce") : true;
    }
    dt_initial = c.d("dt_initial"); dt_max = c.d("dt_max");
    cflv1 = c.d("cfl_max"); cfl = c.d("cfl_desired"); nv1 = c.i("steps_max");
    if (output_style != 3) nstop = IINFINITY;
    vtime = c.b("dt_variable");
    method[1] = vtime ? 2 : 1;
    method[2] = c.i("order"); method[3] = c.i("transverse_waves");
    dimensional_split = c.i("dimensional_split");
    // amr2.f90:258-263: Godunov splitting (1) only; Strang splitting stops the reference
    if (dimensional_split > 1) throw std::runtime_error("Strang splitting is not supported (amrclaw stops)");
    method[4] = c.i("verbosity"); method[5] = c.i("source_split");
    mcapa = c.i("capa_index"); use_fwaves = c.b("use_fwaves");
    for (int k = 0; k < mwaves; ++k) mthlim.push_back(c.i("limiter", k));
    nghost = c.i("num_ghost");
    mthbc[1] = c.i("bc_lower", 0); mthbc[3] = c.i("bc_lower", 1);
    mthbc[2] = c.i("bc_upper", 0); mthbc[4] = c.i("bc_upper", 1);
    xperdom = (mthbc[1] == 2 && mthbc[2] == 2);
    yperdom = (mthbc[3] == 2 && mthbc[4] == 2);
    spheredom = (mthbc[3] == 5 && mthbc[4] == 5);
    mxnest = a.i("amr_levels_max");
    int nr = std::max(1, mxnest - 1);
    for (int k = 0; k < nr; ++k) {
      intratx[k + 1] = a.i("refinement_ratios_x", k);
      intraty[k + 1] = a.i("refinement_ratios_y", k);
      kratio[k + 1] = a.i("refinement_ratios_t", k);
    }
    if (naux > 0) for (int k = 0; k < naux; ++k) auxtype.push_back(a.s("aux_type", k));
    flag_richardson = a.b("flag_richardson"); tol = a.d("flag_richardson_tol");
    flag_gradient = a.b("flag2refine"); tolsp = a.d("flag2refine_tol");
    kcheck = a.i("regrid_interval"); ibuff = a.i("regrid_buffer_width");
    cut = a.d("clustering_cutoff");
    max1d = a.iget("max1d", 60);
    if (r.load(dir + "/regions.data")) {
      for (auto& row : r.rows) {
        if (row.size() < 8) continue;
        Region rg;
        rg.minlevel = (int)DataFile::tod(row[0]); rg.maxlevel = (int)DataFile::tod(row[1]);
        rg.tlow = DataFile::tod(row[2]); rg.thi = DataFile::tod(row[3]);
        rg.xlow = DataFile::tod(row[4]); rg.xhi = DataFile::tod(row[5]);
        rg.ylow = DataFile::tod(row[6]); rg.yhi = DataFile::tod(row[7]);
        regions.push_back(rg);
      }
    }
    if (g.load(dir + "/gauges.data")) {
      for (auto& row : g.rows) {
        if (row.size() < 5) continue;
        Gauge ga;
        ga.num = (int)DataFile::tod(row[0]); ga.x = DataFile::tod(row[1]); ga.y = DataFile::tod(row[2]);
        ga.t_start = DataFile::tod(row[3]); ga.t_end = DataFile::tod(row[4]);
        ga.last_time = ga.t_start; ga.min_inc = row.size() > 5 ? DataFile::tod(row[5]) : 0.0;
        gauges.push_back(ga);
      }
    }
    if (!s.load(dir + "/setprob.data")) throw std::runtime_error("cannot read setprob.data");
    problem = s.s("problem");
    flag_component = s.iget("flag_component", 0);
    if (problem == "advection_square") {
      prob.solver = SOLVER_ADVECTION; prob.ubar = s.d("u"); prob.vbar = s.d("v");
      prob_x0 = s.dget("x0", 0.1); prob_x1 = s.dget("x1", 0.6); prob_y0 = s.dget("y0", 0.1); prob_y1 = s.dget("y1", 0.6);
    } else if (problem == "acoustics_cosine" || problem == "acoustics_gauss") {
      prob.solver = SOLVER_ACOUSTICS; prob.rho = s.d("rho"); prob.bulk = s.d("bulk");
      prob.cc = std::sqrt(prob.bulk / prob.rho); prob.zz = prob.rho * prob.cc;
      prob_width = s.dget("width", problem == "acoustics_cosine" ? 0.2 : 0.05);
      prob_x0 = s.dget("r0", problem == "acoustics_cosine" ? 0.5 : 0.3);
    } else if (problem == "advection_annulus") {
      // tests/advection_2d_annulus/setprob.f: the two Gaussians of qinit.f
      prob.solver = SOLVER_VC_ADVECTION;
      const char* names[8] = {"A1", "beta1", "x1", "y1", "A2", "beta2", "x2", "y2"};
      for (int k = 0; k < 8; ++k) ann[k] = s.d(names[k]);
    } else if (problem == "euler_quadrants") {
      prob.solver = SOLVER_EULER; prob.gamma = s.d("gamma"); prob.gamma1 = prob.gamma - 1.0;
      prob.efix = s.iget("efix", 1) != 0;
      prob_x0 = s.dget("xs", 0.8); prob_y0 = s.dget("ys", 0.8);
    } else {
      throw std::runtime_error("unknown problem " + problem);
    }
  }

  // =================================================== problem plugins (qinit)
  void qinit(int mbc, int mx, int my, double xl, double yl, double dx, double dy, double* q) {
    FArr Q{q, nvar, mx + 2 * mbc, my + 2 * mbc};
    auto at = [&](int m, int i, int j) -> double& { return Q(m, i + mbc, j + mbc); };
    if (problem == "advection_square") {
      // tests/advection_2d_square/qinit.f
      for (int j = 1; j <= my; ++j) {
        double yj = yl + (j - 0.5) * dy;
        for (int i = 1; i <= mx; ++i) {
          double xi = xl + (i - 0.5) * dx;
          at(1, i, j) = (xi > prob_x0 && xi < prob_x1 && yj > prob_y0 && yj < prob_y1) ? 1.0 : 0.1;
        }
      }
    } else if (problem == "acoustics_cosine") {
      // tests/acoustics_2d_radial/qinit.f
      const double pi = 4.0 * std::atan(1.0);
      for (int i = 1; i <= mx; ++i) {
        double xc = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j) {
          double yc = yl + (j - 0.5) * dy;
          double r = std::sqrt(xc * xc + yc * yc);
          double p = (std::fabs(r - prob_x0) <= prob_width) ? 1.0 + std::cos(pi * (r - prob_x0) / prob_width) : 0.0;
          at(1, i, j) = p; at(2, i, j) = 0.0; at(3, i, j) = 0.0;
        }
      }
    } else if (problem == "acoustics_gauss") {
      for (int i = 1; i <= mx; ++i) {
        double xc = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j) {
          double yc = yl + (j - 0.5) * dy;
          double r = std::sqrt(xc * xc + yc * yc);
          double z = (r - prob_x0) / prob_width;
          at(1, i, j) = std::exp(-(z * z)); at(2, i, j) = 0.0; at(3, i, j) = 0.0;
        }
      }
    } else if (problem == "advection_annulus") {
      // tests/advection_2d_annulus/qinit.f: two Gaussians at the physical point of the
      // cell centre (mapc2p.f)
      for (int i = 1; i <= mx; ++i) {
        const double xc = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j) {
          const double yc = yl + (j - 0.5) * dy;
          double xp, yp;
          mapc2p_annulus(xc, yc, xp, yp);
          at(1, i, j) = ann[0] * std::exp(-ann[1] * ((xp - ann[2]) * (xp - ann[2]) + (yp - ann[3]) * (yp - ann[3]))) +
                        ann[4] * std::exp(-ann[5] * ((xp - ann[6]) * (xp - ann[6]) + (yp - ann[7]) * (yp - ann[7])));
        }
      }
    } else if (problem == "euler_quadrants") {
      // examples/euler_2d_quadrants/qinit.f:33-72
      const double rpp[5] = {0, 1.5, 0.3, 0.029032258064516, 0.3};
      const double rpr[5] = {0, 1.5, 0.532258064516129, 0.137992831541219, 0.532258064516129};
      const double rpu[5] = {0, 0.0, 1.206045378311055, 1.206045378311055, 0.0};
      const double rpv[5] = {0, 0.0, 0.0, 1.206045378311055, 1.206045378311055};
      const double g1 = prob.gamma - 1.0;
      for (int i = 1; i <= mx; ++i) {
        double xc = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j) {
          double yc = yl + (j - 0.5) * dy;
          int iq = 1;
          if (xc >= prob_x0 && yc >= prob_y0) iq = 1;
          if (xc < prob_x0 && yc >= prob_y0) iq = 2;
          if (xc < prob_x0 && yc < prob_y0) iq = 3;
          if (xc >= prob_x0 && yc < prob_y0) iq = 4;
          at(1, i, j) = rpr[iq];
          at(2, i, j) = rpr[iq] * rpu[iq];
          at(3, i, j) = rpr[iq] * rpv[iq];
          at(4, i, j) = rpp[iq] / g1 + 0.5 * rpr[iq] * (rpu[iq] * rpu[iq] + rpv[iq] * rpv[iq]);
        }
      }
    }
  }

  // tests/advection_2d_annulus/mapc2p.f: polar coordinates, xc = r, yc = theta
  static void mapc2p_annulus(double xc, double yc, double& xp, double& yp) {
    xp = xc * std::cos(yc);
    yp = xc * std::sin(yc);
  }
  // tests/advection_2d_annulus/stream.f
  static double stream_annulus(double x, double y) { return 3.1415926535897931 * (x * x + y * y); }

  // setaux: aux(naux, 1-mbc:mx+mbc, 1-mbc:my+mbc) of a patch with lower corner (xlow, ylow).
  // tests/advection_2d_annulus/setaux.f: the edge velocities by differencing the stream
  // function between mapped corners, and the capacity kappa = (mapped area) / (dxc*dyc).
  // It sets every cell, so values copied in before (icall) are overwritten.
  void setaux(int mbc, int mx, int my, double xlow, double ylow, double dxc, double dyc, double* aux) const {
    if (problem != "advection_annulus") throw std::runtime_error("setaux: no aux arrays for problem " + problem);
    FArr A{aux, naux, mx + 2 * mbc, my + 2 * mbc};
    for (int j = 1 - mbc; j <= my + mbc; ++j)
      for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        double xc[5], yc[5], xp[5], yp[5];
        xc[0] = xlow + (i - 1) * dxc; yc[0] = ylow + (j - 1) * dyc;
        xc[1] = xc[0]; yc[1] = yc[0] + dyc;
        xc[2] = xc[0] + dxc; yc[2] = yc[0] + dyc;
        xc[3] = xc[0] + dxc; yc[3] = yc[0];
        for (int c = 0; c < 4; ++c) mapc2p_annulus(xc[c], yc[c], xp[c], yp[c]);
        A(1, i + mbc, j + mbc) = (stream_annulus(xp[1], yp[1]) - stream_annulus(xp[0], yp[0])) / dyc;
        A(2, i + mbc, j + mbc) = -(stream_annulus(xp[3], yp[3]) - stream_annulus(xp[0], yp[0])) / dxc;
        xp[4] = xp[0]; yp[4] = yp[0];
        double area = 0.0;
        for (int c = 0; c < 4; ++c) area = area + 0.5 * (yp[c] + yp[c + 1]) * (xp[c + 1] - xp[c]);
        A(3, i + mbc, j + mbc) = area / (dxc * dyc);
      }
  }

  // =================================================== node store (nodget.f)
  int nodget() {
    if (ndfree == 0) {
      int old = (int)node.size() - 1;
      int add = 10000;
      node.resize(old + 1 + add);
      for (int k = old + 1; k <= old + add; ++k) node[k].nextfree = k + 1;
      node[old + add].nextfree = 0;
      ndfree = old + 1;
    }
    int m = ndfree;
    ndfree = node[m].nextfree;
    node[m] = Node2();
    return m;
  }
  void putnod(int m) { node[m].nextfree = ndfree; ndfree = m; }

  int mitot_of(int m) const { return node[m].ihi - node[m].ilo + 1 + 2 * nghost; }
  int mjtot_of(int m) const { return node[m].jhi - node[m].jlo + 1 + 2 * nghost; }

  // ===================================================== patch step (flux2.f)
  void limiter(int maxm, int meqn, int mbc, int mx, Waves wave, Slice s) {
    (void)maxm;
    for (int mw = 1; mw <= mwaves; ++mw) {
      if (mthlim[mw - 1] == 0) continue;
      double dotr = 0.0;
      for (int i = 0; i <= mx + 1; ++i) {
        double wnorm2 = 0.0, dotl = dotr;
        dotr = 0.0;
        for (int m = 1; m <= meqn; ++m) {
          wnorm2 = wnorm2 + wave(m, mw, i) * wave(m, mw, i);
          dotr = dotr + wave(m, mw, i) * wave(m, mw, i + 1);
        }
        if (i == 0) continue;
        if (wnorm2 == 0.0) continue;
        double r = (s(mw, i) > 0.0) ? dotl / wnorm2 : dotr / wnorm2;
        double wl = 0.0;
        switch (mthlim[mw - 1]) {
          case 1: wl = std::max(0.0, std::min(1.0, r)); break;
          case 2: wl = std::max(0.0, std::max(std::min(1.0, 2.0 * r), std::min(2.0, r))); break;
          case 3: wl = (r + std::fabs(r)) / (1.0 + std::fabs(r)); break;
          case 4: { double c = (1.0 + r) / 2.0; wl = std::max(0.0, std::min(c, std::min(2.0, 2.0 * r))); } break;
          case 5: wl = r; break;
        }
        for (int m = 1; m <= meqn; ++m) wave(m, mw, i) = wl * wave(m, mw, i);
      }
    }
    (void)mbc;
  }

  struct Work1d {
    std::vector<double> faddm, faddp, gaddm, gaddp, q1d, aux1, aux2, aux3, dtdx1d;
    std::vector<double> wave, s, amdq, apdq, cqxx, bmasdq, bpasdq;
    void ensure(int maxm, int mbc, int meqn, int mw, int maux) {
      size_t L = maxm + 2 * mbc;
      faddm.assign(meqn * L, 0); faddp.assign(meqn * L, 0);
      gaddm.assign(meqn * L * 2, 0); gaddp.assign(meqn * L * 2, 0);
      q1d.assign(meqn * L, 0);
      aux1.assign(std::max(maux, 1) * L, 0); aux2 = aux1; aux3 = aux1;
      dtdx1d.assign(L, 0);
      wave.assign(meqn * mw * L, 0); s.assign(mw * L, 0);
      amdq.assign(meqn * L, 0); apdq = amdq; cqxx = amdq; bmasdq = amdq; bpasdq = amdq;
    }
  };

  // flux2.f:25-237
  void flux2(int ixy, int maxm, int meqn, int maux, int mbc, int mx, Work1d& W, double& cfl1d) {
    const int base = 1 - mbc;
    const int L = maxm + 2 * mbc;
    Slice q1d{W.q1d.data(), meqn, base};
    Slice aux1{W.aux1.data(), std::max(maux, 1), base}, aux2{W.aux2.data(), std::max(maux, 1), base}, aux3{W.aux3.data(), std::max(maux, 1), base};
    Slice faddm{W.faddm.data(), meqn, base}, faddp{W.faddp.data(), meqn, base};
    auto gaddm = [&](int m, int i, int k) -> double& { return W.gaddm[(m - 1) + meqn * ((i - base) + (size_t)L * (k - 1))]; };
    auto gaddp = [&](int m, int i, int k) -> double& { return W.gaddp[(m - 1) + meqn * ((i - base) + (size_t)L * (k - 1))]; };
    auto dtdx1d = [&](int i) -> double& { return W.dtdx1d[i - base]; };
    Waves wave{W.wave.data(), meqn, mwaves, base};
    Slice s{W.s.data(), mwaves, base};
    Slice amdq{W.amdq.data(), meqn, base}, apdq{W.apdq.data(), meqn, base}, cqxx{W.cqxx.data(), meqn, base};
    Slice bmasdq{W.bmasdq.data(), meqn, base}, bpasdq{W.bpasdq.data(), meqn, base};

    bool limit = false;
    for (int mw = 1; mw <= mwaves; ++mw) if (mthlim[mw - 1] > 0) limit = true;
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
      for (int m = 1; m <= meqn; ++m) {
        faddm(m, i) = 0.0; faddp(m, i) = 0.0;
        gaddm(m, i, 1) = 0.0; gaddp(m, i, 1) = 0.0; gaddm(m, i, 2) = 0.0; gaddp(m, i, 2) = 0.0;
      }
    rpn2(prob, ixy, meqn, mwaves, mbc, mx, q1d, q1d, aux2, aux2, wave, s, amdq, apdq);
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= meqn; ++m) {
        faddp(m, i) = faddp(m, i) - apdq(m, i);
        faddm(m, i) = faddm(m, i) + amdq(m, i);
      }
    cfl1d = 0.0;
    for (int mw = 1; mw <= mwaves; ++mw)
      for (int i = 1; i <= mx + 1; ++i)
        cfl1d = std::max(cfl1d, std::max(dtdx1d(i) * s(mw, i), -dtdx1d(i - 1) * s(mw, i)));
    if (method[2] != 1) {
      if (limit) limiter(maxm, meqn, mbc, mx, wave, s);
      for (int i = 1; i <= mx + 1; ++i) {
        double dtdxave = 0.5 * (dtdx1d(i - 1) + dtdx1d(i));
        for (int m = 1; m <= meqn; ++m) {
          cqxx(m, i) = 0.0;
          for (int mw = 1; mw <= mwaves; ++mw) {
            double abs_sign = use_fwaves ? dsign(1.0, s(mw, i)) : std::fabs(s(mw, i));
            cqxx(m, i) = cqxx(m, i) + abs_sign * (1.0 - std::fabs(s(mw, i)) * dtdxave) * wave(m, mw, i);
          }
          faddm(m, i) = faddm(m, i) + 0.5 * cqxx(m, i);
          faddp(m, i) = faddp(m, i) + 0.5 * cqxx(m, i);
        }
      }
    }
    if (method[3] == 0) return;
    if (method[2] > 1 && method[3] == 2) {
      for (int i = 1; i <= mx + 1; ++i)
        for (int m = 1; m <= meqn; ++m) {
          amdq(m, i) = amdq(m, i) + cqxx(m, i);
          apdq(m, i) = apdq(m, i) - cqxx(m, i);
        }
    }
    rpt2(prob, ixy, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, amdq, bmasdq, bpasdq);
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= meqn; ++m) {
        double gu = 0.5 * dtdx1d(i - 1) * bmasdq(m, i);
        gaddm(m, i - 1, 1) = gaddm(m, i - 1, 1) - gu;
        gaddp(m, i - 1, 1) = gaddp(m, i - 1, 1) - gu;
        gu = 0.5 * dtdx1d(i - 1) * bpasdq(m, i);
        gaddm(m, i - 1, 2) = gaddm(m, i - 1, 2) - gu;
        gaddp(m, i - 1, 2) = gaddp(m, i - 1, 2) - gu;
      }
    rpt2(prob, ixy, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, apdq, bmasdq, bpasdq);
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= meqn; ++m) {
        double gu = 0.5 * dtdx1d(i) * bmasdq(m, i);
        gaddm(m, i, 1) = gaddm(m, i, 1) - gu;
        gaddp(m, i, 1) = gaddp(m, i, 1) - gu;
        gu = 0.5 * dtdx1d(i) * bpasdq(m, i);
        gaddm(m, i, 2) = gaddm(m, i, 2) - gu;
        gaddp(m, i, 2) = gaddp(m, i, 2) - gu;
      }
  }

  // step2.f90:7-169 ; fm,fp,gm,gp are (nvar, mitot, mjtot) 1-based with ghost offset
  void step2(int maxm, int meqn, int maux, int mbc, int mx, int my, const double* qold, const double* aux,
             double dx, double dy, double dt, double& cflgrid, double* fm, double* fp, double* gm, double* gp) {
    const int mitot = mx + 2 * mbc, mjtot = my + 2 * mbc;
    auto Q = [&](int m, int i, int j) { return qold[(m - 1) + meqn * ((i + mbc - 1) + (size_t)mitot * (j + mbc - 1))]; };
    auto A = [&](int m, int i, int j) { return aux[(m - 1) + maux * ((i + mbc - 1) + (size_t)mitot * (j + mbc - 1))]; };
    auto F = [&](double* f, int m, int i, int j) -> double& { return f[(m - 1) + meqn * ((i + mbc - 1) + (size_t)mitot * (j + mbc - 1))]; };
    Work1d W;
    W.ensure(maxm, mbc, meqn, mwaves, maux);
    const int base = 1 - mbc, L = maxm + 2 * mbc;
    cflgrid = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy;
    std::fill(fm, fm + (size_t)meqn * mitot * mjtot, 0.0);
    std::fill(fp, fp + (size_t)meqn * mitot * mjtot, 0.0);
    std::fill(gm, gm + (size_t)meqn * mitot * mjtot, 0.0);
    std::fill(gp, gp + (size_t)meqn * mitot * mjtot, 0.0);
    auto fa = [&](std::vector<double>& v, int m, int i) -> double& { return v[(m - 1) + meqn * (i - base)]; };
    auto ga = [&](std::vector<double>& v, int m, int i, int k) -> double& { return v[(m - 1) + meqn * ((i - base) + (size_t)L * (k - 1))]; };
    for (int j = 0; j <= my + 1; ++j) {
      for (int i = 1 - mbc; i <= mx + mbc; ++i) for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + meqn * (i - base)] = Q(m, i, j);
      if (mcapa > 0) { for (int i = 1 - mbc; i <= mx + mbc; ++i) W.dtdx1d[i - base] = dtdx / A(mcapa, i, j); }
      else std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdx);
      if (maux > 0)
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
          for (int m = 1; m <= maux; ++m) {
            W.aux1[(m - 1) + maux * (i - base)] = A(m, i, j - 1);
            W.aux2[(m - 1) + maux * (i - base)] = A(m, i, j);
            W.aux3[(m - 1) + maux * (i - base)] = A(m, i, j + 1);
          }
      double cfl1d;
      flux2(1, maxm, meqn, maux, mbc, mx, W, cfl1d);
      cflgrid = std::max(cflgrid, cfl1d);
      for (int i = 1; i <= mx + 1; ++i)
        for (int m = 1; m <= meqn; ++m) {
          F(fm, m, i, j) = F(fm, m, i, j) + fa(W.faddm, m, i);
          F(fp, m, i, j) = F(fp, m, i, j) + fa(W.faddp, m, i);
          F(gm, m, i, j) = F(gm, m, i, j) + ga(W.gaddm, m, i, 1);
          F(gp, m, i, j) = F(gp, m, i, j) + ga(W.gaddp, m, i, 1);
          F(gm, m, i, j + 1) = F(gm, m, i, j + 1) + ga(W.gaddm, m, i, 2);
          F(gp, m, i, j + 1) = F(gp, m, i, j + 1) + ga(W.gaddp, m, i, 2);
        }
    }
    for (int i = 0; i <= mx + 1; ++i) {
      for (int j = 1 - mbc; j <= my + mbc; ++j) for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + meqn * (j - base)] = Q(m, i, j);
      if (mcapa > 0) { for (int j = 1 - mbc; j <= my + mbc; ++j) W.dtdx1d[j - base] = dtdy / A(mcapa, i, j); }
      else std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdy);
      if (maux > 0)
        for (int j = 1 - mbc; j <= my + mbc; ++j)
          for (int m = 1; m <= maux; ++m) {
            W.aux1[(m - 1) + maux * (j - base)] = A(m, i - 1, j);
            W.aux2[(m - 1) + maux * (j - base)] = A(m, i, j);
            W.aux3[(m - 1) + maux * (j - base)] = A(m, i + 1, j);
          }
      double cfl1d;
      flux2(2, maxm, meqn, maux, mbc, my, W, cfl1d);
      cflgrid = std::max(cflgrid, cfl1d);
      for (int j = 1; j <= my + 1; ++j)
        for (int m = 1; m <= meqn; ++m) {
          F(gm, m, i, j) = F(gm, m, i, j) + fa(W.faddm, m, j);
          F(gp, m, i, j) = F(gp, m, i, j) + fa(W.faddp, m, j);
          F(fm, m, i, j) = F(fm, m, i, j) + ga(W.gaddm, m, j, 1);
          F(fp, m, i, j) = F(fp, m, i, j) + ga(W.gaddp, m, j, 1);
          F(fm, m, i + 1, j) = F(fm, m, i + 1, j) + ga(W.gaddm, m, j, 2);
          F(fp, m, i + 1, j) = F(fp, m, i + 1, j) + ga(W.gaddp, m, j, 2);
        }
    }
  }

  // stepgrid.f:24-232 ; returns dtnew, accumulates cfl_level
  void stepgrid(double* q, double* fm, double* fp, double* gm, double* gp, int mitot, int mjtot, int mbc, double dt,
                double& dtnew, double dx, double dy, const double* aux, double& cflgrid_out) {
    const int mx = mitot - 2 * mbc, my = mjtot - 2 * mbc;
    const int maxm = std::max(mx, my);
    double cflgrid = 0;
    step2(maxm, nvar, naux, mbc, mx, my, q, aux, dx, dy, dt, cflgrid, fm, fp, gm, gp);
    cflgrid_out = cflgrid;
    const double dtdx = dt / dx, dtdy = dt / dy;
    FArr Q{q, nvar, mitot, mjtot}, FM{fm, nvar, mitot, mjtot}, FP{fp, nvar, mitot, mjtot}, GM{gm, nvar, mitot, mjtot}, GP{gp, nvar, mitot, mjtot};
    for (int j = mbc + 1; j <= mjtot - mbc; ++j)
      for (int i = mbc + 1; i <= mitot - mbc; ++i)
        for (int m = 1; m <= nvar; ++m) {
          if (mcapa == 0) {
            Q(m, i, j) = Q(m, i, j) - dtdx * (FM(m, i + 1, j) - FP(m, i, j)) - dtdy * (GM(m, i, j + 1) - GP(m, i, j));
          } else {
            const double ca = aux[(mcapa - 1) + naux * ((i - 1) + (size_t)mitot * (j - 1))];
            Q(m, i, j) = Q(m, i, j) - (dtdx * (FM(m, i + 1, j) - FP(m, i, j)) + dtdy * (GM(m, i, j + 1) - GP(m, i, j))) / ca;
          }
        }
    if (cflgrid > 0.0) dtnew = dt * cfl / cflgrid;
    else dtnew = RINFINITY;
  }

  // flux2_dimSplit.f: the normal fluctuations, limiter and second-order correction of one
  // slice, without transverse terms (faddm = amdq, faddp = -apdq, then + cqxx/2)
  void flux2_dimSplit(int ixy, int maxm, int meqn, int maux, int mbc, int mx, Work1d& W, double& cfl1d) {
    const int base = 1 - mbc;
    Slice q1d{W.q1d.data(), meqn, base};
    Slice aux2{W.aux2.data(), std::max(maux, 1), base};
    Slice faddm{W.faddm.data(), meqn, base}, faddp{W.faddp.data(), meqn, base};
    auto dtdx1d = [&](int i) -> double& { return W.dtdx1d[i - base]; };
    Waves wave{W.wave.data(), meqn, mwaves, base};
    Slice s{W.s.data(), mwaves, base};
    Slice cqxx{W.cqxx.data(), meqn, base};
    bool limit = false;
    for (int mw = 1; mw <= mwaves; ++mw) if (mthlim[mw - 1] > 0) limit = true;
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
      for (int m = 1; m <= meqn; ++m) { faddm(m, i) = 0.0; faddp(m, i) = 0.0; }
    // rpn2 writes amdq into faddm and apdq into faddp directly (flux2_dimSplit.f:55-57)
    rpn2(prob, ixy, meqn, mwaves, mbc, mx, q1d, q1d, aux2, aux2, wave, s, faddm, faddp);
    for (int i = 1 - mbc; i <= mx + mbc; ++i)
      for (int m = 1; m <= meqn; ++m) faddp(m, i) = -faddp(m, i);
    cfl1d = 0.0;
    for (int mw = 1; mw <= mwaves; ++mw)
      for (int i = 1; i <= mx + 1; ++i)
        cfl1d = std::max(cfl1d, std::max(dtdx1d(i) * s(mw, i), -dtdx1d(i - 1) * s(mw, i)));
    if (method[2] == 1) return;
    if (limit) limiter(maxm, meqn, mbc, mx, wave, s);
    for (int i = 1; i <= mx + 1; ++i) {
      const double dtdxave = 0.5 * (dtdx1d(i - 1) + dtdx1d(i));
      for (int m = 1; m <= meqn; ++m) {
        cqxx(m, i) = 0.0;
        for (int mw = 1; mw <= mwaves; ++mw) {
          const double abs_sign = use_fwaves ? dsign(1.0, s(mw, i)) : std::fabs(s(mw, i));
          cqxx(m, i) = cqxx(m, i) + abs_sign * (1.0 - std::fabs(s(mw, i)) * dtdxave) * wave(m, mw, i);
        }
        faddm(m, i) = faddm(m, i) + 0.5 * cqxx(m, i);
        faddp(m, i) = faddp(m, i) + 0.5 * cqxx(m, i);
      }
    }
  }

  // stepgrid_dimSplit.f:4-201 with step2x.f90 / step2y.f90: Godunov splitting. x-sweeps over
  // every row (ghost rows included), the x-update of every row's interior cells, then
  // y-sweeps over the interior columns of the x-updated values and the y-update.
  void stepgrid_dimSplit(double* q, double* fm, double* fp, double* gm, double* gp, int mitot, int mjtot, int mbc,
                         double dt, double& dtnew, double dx, double dy, const double* aux, double& cflgrid_out) {
    const int mx = mitot - 2 * mbc, my = mjtot - 2 * mbc, meqn = nvar, maux = naux;
    const int maxm = std::max(mx, my);
    const size_t nf = (size_t)meqn * mitot * mjtot;
    auto at = [&](int i, int j) { return (size_t)(i + mbc - 1) + (size_t)mitot * (j + mbc - 1); };
    auto Q = [&](int m, int i, int j) -> double& { return q[(m - 1) + meqn * at(i, j)]; };
    auto F = [&](double* f, int m, int i, int j) -> double& { return f[(m - 1) + meqn * at(i, j)]; };
    auto A = [&](int m, int i, int j) { return aux[(m - 1) + maux * at(i, j)]; };
    Work1d W;
    W.ensure(maxm, mbc, meqn, mwaves, maux);
    const int base = 1 - mbc;
    auto fa = [&](std::vector<double>& v, int m, int i) { return v[(m - 1) + meqn * (i - base)]; };
    double cfl_grid = 0.0;
    // step2x.f90
    double cflx = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy;
    std::fill(fm, fm + nf, 0.0);
    std::fill(fp, fp + nf, 0.0);
    for (int j = 1 - mbc; j <= my + mbc; ++j) {
      for (int i = 1 - mbc; i <= mx + mbc; ++i) for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + meqn * (i - base)] = Q(m, i, j);
      if (mcapa > 0) { for (int i = 1 - mbc; i <= mx + mbc; ++i) W.dtdx1d[i - base] = dtdx / A(mcapa, i, j); }
      else std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdx);
      if (maux > 0)
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
          for (int m = 1; m <= maux; ++m) W.aux2[(m - 1) + maux * (i - base)] = A(m, i, j);
      double cfl1d;
      flux2_dimSplit(1, maxm, meqn, maux, mbc, mx, W, cfl1d);
      cflx = std::max(cflx, cfl1d);
      for (int i = 1; i <= mx + 1; ++i)
        for (int m = 1; m <= meqn; ++m) {
          F(fm, m, i, j) = F(fm, m, i, j) + fa(W.faddm, m, i);
          F(fp, m, i, j) = F(fp, m, i, j) + fa(W.faddp, m, i);
        }
    }
    cfl_grid = std::max(cfl_grid, cflx);
    for (int j = 1 - mbc; j <= my + mbc; ++j)
      for (int i = 1; i <= mx; ++i)
        for (int m = 1; m <= meqn; ++m) {
          if (mcapa == 0) Q(m, i, j) = Q(m, i, j) - dtdx * (F(fm, m, i + 1, j) - F(fp, m, i, j));
          else Q(m, i, j) = Q(m, i, j) - dtdx * (F(fm, m, i + 1, j) - F(fp, m, i, j)) / A(mcapa, i, j);
        }
    // step2y.f90
    double cfly = 0.0;
    std::fill(gm, gm + nf, 0.0);
    std::fill(gp, gp + nf, 0.0);
    for (int i = 1; i <= mx; ++i) {
      for (int j = 1 - mbc; j <= my + mbc; ++j) for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + meqn * (j - base)] = Q(m, i, j);
      if (mcapa > 0) { for (int j = 1 - mbc; j <= my + mbc; ++j) W.dtdx1d[j - base] = dtdy / A(mcapa, i, j); }
      else std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdy);
      if (maux > 0)
        for (int j = 1 - mbc; j <= my + mbc; ++j)
          for (int m = 1; m <= maux; ++m) W.aux2[(m - 1) + maux * (j - base)] = A(m, i, j);
      double cfl1d;
      flux2_dimSplit(2, maxm, meqn, maux, mbc, my, W, cfl1d);
      cfly = std::max(cfly, cfl1d);
      for (int j = 1; j <= my + 1; ++j)
        for (int m = 1; m <= meqn; ++m) {
          F(gm, m, i, j) = F(gm, m, i, j) + fa(W.faddm, m, j);
          F(gp, m, i, j) = F(gp, m, i, j) + fa(W.faddp, m, j);
        }
    }
    cfl_grid = std::max(cfl_grid, cfly);
    for (int j = 1; j <= my; ++j)
      for (int i = 1; i <= mx; ++i)
        for (int m = 1; m <= meqn; ++m) {
          if (mcapa == 0) Q(m, i, j) = Q(m, i, j) - dtdy * (F(gm, m, i, j + 1) - F(gp, m, i, j));
          else Q(m, i, j) = Q(m, i, j) - dtdy * (F(gm, m, i, j + 1) - F(gp, m, i, j)) / A(mcapa, i, j);
        }
    // the level's Courant number decides dtnew (stepgrid_dimSplit.f:171-179); per grid, its
    // own maximum gives the same level minimum
    cflgrid_out = cfl_grid;
    if (cfl_grid > 0.0) dtnew = dt * cfl / cfl_grid;
    else dtnew = RINFINITY;
  }

  // ===================================================== ghost cells: bc2amr
  void bc2amr(double* valp, int nrow, int ncol, double hx, double hy, double xlo_p, double xhi_p, double ylo_p, double yhi_p) {
    FArr val{valp, nvar, nrow, ncol};
    const double hxmarg = hx * 0.01, hymarg = hy * 0.01;
    if (xperdom && (yperdom || spheredom)) return;
    if (xlo_p < xlower - hxmarg) {
      int nxl = (int)((xlower + hxmarg - xlo_p) / hx);
      if (mthbc[1] == 1) {
        for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nxl; ++i) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, nxl + 1, j);
      } else if (mthbc[1] == 3) {
        for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nxl; ++i) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, 2 * nxl + 1 - i, j);
        for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nxl; ++i) val(2, i, j) = -val(2, i, j);
      } else if (mthbc[1] == 0) throw std::runtime_error("user BC not provided");
    }
    if (xhi_p > xupper + hxmarg) {
      int nxr = (int)((xhi_p - xupper + hxmarg) / hx);
      int ibeg = std::max(nrow - nxr + 1, 1);
      if (mthbc[2] == 1) {
        for (int i = ibeg; i <= nrow; ++i) for (int j = 1; j <= ncol; ++j) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, ibeg - 1, j);
      } else if (mthbc[2] == 3) {
        for (int i = ibeg; i <= nrow; ++i) for (int j = 1; j <= ncol; ++j) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, 2 * ibeg - 1 - i, j);
        for (int i = ibeg; i <= nrow; ++i) for (int j = 1; j <= ncol; ++j) val(2, i, j) = -val(2, i, j);
      } else if (mthbc[2] == 0) throw std::runtime_error("user BC not provided");
    }
    if (ylo_p < ylower - hymarg) {
      int nyb = (int)((ylower + hymarg - ylo_p) / hy);
      if (mthbc[3] == 1) {
        for (int j = 1; j <= nyb; ++j) for (int i = 1; i <= nrow; ++i) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, i, nyb + 1);
      } else if (mthbc[3] == 3) {
        for (int j = 1; j <= nyb; ++j) for (int i = 1; i <= nrow; ++i) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, i, 2 * nyb + 1 - j);
        for (int j = 1; j <= nyb; ++j) for (int i = 1; i <= nrow; ++i) val(3, i, j) = -val(3, i, j);
      } else if (mthbc[3] == 0) throw std::runtime_error("user BC not provided");
    }
    if (yhi_p > yupper + hymarg) {
      int nyt = (int)((yhi_p - yupper + hymarg) / hy);
      int jbeg = std::max(ncol - nyt + 1, 1);
      if (mthbc[4] == 1) {
        for (int j = jbeg; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, i, jbeg - 1);
      } else if (mthbc[4] == 3) {
        for (int j = jbeg; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i) for (int m = 1; m <= nvar; ++m) val(m, i, j) = val(m, i, 2 * jbeg - 1 - j);
        for (int j = jbeg; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i) val(3, i, j) = -val(3, i, j);
      } else if (mthbc[4] == 0) throw std::runtime_error("user BC not provided");
    }
  }

  // ===================================================== ghost cells: intfil
  // flaguse is (ilo:ihi, jlo:jhi) column-major
  void intfil(double* valp, int mi, int mj, double t, signed char* flaguse, int nrowst, int ncolst, int ilo, int ihi,
              int jlo, int jhi, int level, int msrc) {
    FArr val{valp, nvar, mi, mj};
    const int nfr = ihi - ilo + 1;
    auto FU = [&](int i, int j) -> signed char& { return flaguse[(i - ilo) + (size_t)nfr * (j - jlo)]; };
    const double dt = possk[level];
    const double t_epsilon = 1.0e-4;
    std::fill(flaguse, flaguse + (size_t)nfr * (jhi - jlo + 1), 0);
    const std::vector<int>& src = (msrc == -1) ? levelgrids[level] : node[msrc].bnd;
    for (int mptr : src) {
      const Node2& g = node[mptr];
      const int imlo = g.ilo, jmlo = g.jlo, imhi = g.ihi, jmhi = g.jhi;
      const int mitot = mitot_of(mptr);
      const int ixlo = std::max(imlo, ilo), ixhi = std::min(imhi, ihi);
      const int jxlo = std::max(jmlo, jlo), jxhi = std::min(jmhi, jhi);
      if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
      const double alphac = (g.time - t) / dt;
      const double alphai = 1.0 - alphac;
      if (alphai < -t_epsilon || alphai > 1.0 + t_epsilon) throw std::runtime_error("intfil: time not available");
      const double* src1 = nullptr;
      const double* src2 = nullptr;
      bool tint = false;
      if (std::fabs(alphai - 1.0) < t_epsilon) src1 = g.q1.data();
      else if (std::fabs(alphai) < t_epsilon) {
        if (level == mxnest) throw std::runtime_error("intfil: old time on finest level");
        src1 = g.q2.data();
      } else {
        if (level == mxnest) throw std::runtime_error("intfil: time interpolation on finest level");
        src1 = g.q1.data(); src2 = g.q2.data(); tint = true;
      }
      auto idx = [&](int ivar, int i, int j) { return (ivar - 1) + (size_t)nvar * ((j - 1) * (size_t)mitot + i - 1); };
      for (int ivar = 1; ivar <= nvar; ++ivar)
        for (int j = jxlo; j <= jxhi; ++j)
          for (int i = ixlo; i <= ixhi; ++i) {
            const size_t k = idx(ivar, i - imlo + nghost + 1, j - jmlo + nghost + 1);
            if (!tint) val(ivar, i - ilo + nrowst, j - jlo + ncolst) = src1[k];
            else val(ivar, i - ilo + nrowst, j - jlo + ncolst) = src1[k] * alphai + src2[k] * alphac;
            FU(i, j) = 1;
          }
    }
    if (jhi >= jregsz[level])
      for (int j = std::max(jregsz[level], jlo); j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) FU(i, j) = 1;
    if (jlo < 0)
      for (int j = jlo; j <= std::min(std::min(-1, ncolst + jhi - jlo), jhi); ++j) for (int i = ilo; i <= ihi; ++i) FU(i, j) = 1;
    if (ilo < 0)
      for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= std::min(std::min(-1, nrowst + ihi - ilo), ihi); ++i) FU(i, j) = 1;
    if (ihi >= iregsz[level])
      for (int j = jlo; j <= jhi; ++j) for (int i = std::max(iregsz[level], ilo); i <= ihi; ++i) FU(i, j) = 1;
  }

  // trimbd.f90:32-97 ; used is (nrow, ncol) 1-based
  void trimbd(const signed char* used, int nrow, int ncol, bool& set, int rect[4]) {
    auto U = [&](int i, int j) { return (int)used[(i - 1) + (size_t)nrow * (j - 1)]; };
    long utot = 0;
    for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i) utot += U(i, j);
    if (utot == (long)nrow * ncol) { set = true; return; }
    set = false;
    for (int i = 1; i <= nrow; ++i) {
      int check = 1;
      for (int j = 1; j <= ncol; ++j) check = std::min(check, U(i, j));
      rect[0] = i; if (check == 0) break;
    }
    for (int i = 1; i <= nrow; ++i) {
      int check = 1;
      for (int j = 1; j <= ncol; ++j) check = std::min(check, U(nrow - i + 1, j));
      rect[1] = nrow - i + 1; if (check == 0) break;
    }
    for (int j = 1; j <= ncol; ++j) {
      int check = 1;
      for (int i = 1; i <= nrow; ++i) check = std::min(check, U(i, j));
      rect[2] = j; if (check == 0) break;
    }
    for (int j = 1; j <= ncol; ++j) {
      int check = 1;
      for (int i = 1; i <= nrow; ++i) check = std::min(check, U(i, ncol - j + 1));
      rect[3] = ncol - j + 1; if (check == 0) break;
    }
  }

  // filpatch.f90:71-355
  void filrecur(int level, double* valbig, int mitot, int mjtot, double t, int nrowst, int ncolst, int ilo, int ihi,
                int jlo, int jhi, bool patchOnly, int msrc) {
    FArr VB{valbig, nvar, mitot, mjtot};
    const int mitot_patch = ihi - ilo + 1, mjtot_patch = jhi - jlo + 1;
    const double dx_fine = hxposs[level], dy_fine = hyposs[level];
    const double xlow_fine = xlower + ilo * dx_fine, ylow_fine = ylower + jlo * dy_fine;
    std::vector<signed char> flaguse((size_t)mitot_patch * mjtot_patch);
    intfil(valbig, mitot, mjtot, t, flaguse.data(), nrowst, ncolst, ilo, ihi, jlo, jhi, level, msrc);
    bool set; int un[4];
    trimbd(flaguse.data(), mitot_patch, mjtot_patch, set, un);
    if (!set) {
      if (level == 1) throw std::runtime_error("filrecur: level 1 not set");
      const double dx_coarse = hxposs[level - 1], dy_coarse = hyposs[level - 1];
      un[0] += ilo - 1; un[1] += ilo - 1; un[2] += jlo - 1; un[3] += jlo - 1;
      const int rx = intratx[level - 1], ry = intraty[level - 1];
      const int iplo = (un[0] - rx + nghost * rx) / rx - nghost;
      const int iphi = (un[1] + rx) / rx;
      const int jplo = (un[2] - ry + nghost * ry) / ry - nghost;
      const int jphi = (un[3] + ry) / ry;
      const double xlow_coarse = xlower + iplo * dx_coarse, ylow_coarse = ylower + jplo * dy_coarse;
      const int mitot_coarse = iphi - iplo + 1, mjtot_coarse = jphi - jplo + 1;
      if (mitot_coarse > ihi - ilo + 3 || mjtot_coarse > jhi - jlo + 3) throw std::runtime_error("filrecur: workspace");
      std::vector<double> valcrse((size_t)(ihi - ilo + 3) * (jhi - jlo + 3) * nvar, 0.0);
      bool sticks = (iplo < 0 || jplo < 0 || iphi >= iregsz[level - 1] || jphi >= jregsz[level - 1]);
      if ((xperdom || (yperdom || spheredom)) && sticks)
        prefilrecur(level - 1, valcrse.data(), mitot_coarse, mjtot_coarse, t, 1, 1, iplo, iphi, jplo, jphi, iplo, iphi, jplo, jphi, true);
      else
        filrecur(level - 1, valcrse.data(), mitot_coarse, mjtot_coarse, t, 1, 1, iplo, iphi, jplo, jphi, true, -1);
      auto CI = [&](int n, int i, int j) { return valcrse[(n - 1) + (size_t)nvar * (i - 1) + (size_t)nvar * mitot_coarse * (j - 1)]; };
      const double ratiox = (double)rx, ratioy = (double)ry;
      for (int jf = 1; jf <= mjtot_patch; ++jf) {
        const int jc = (int)std::floor((jf + jlo - 1) / ratioy) - jplo + 1;
        const double ycc = ylow_coarse + (jc - 0.5) * dy_coarse;
        const double ycf = ylower + (jf - 1 + jlo + 0.5) * dy_fine;
        const double eta2 = (ycf - ycc) / dy_coarse;
        for (int iff = 1; iff <= mitot_patch; ++iff) {
          const int ic = (int)std::floor((iff + ilo - 1) / ratiox) - iplo + 1;
          const double xcc = xlow_coarse + (ic - 0.5) * dx_coarse;
          const double xcf = xlower + (iff - 1 + ilo + 0.5) * dx_fine;
          const double eta1 = (xcf - xcc) / dx_coarse;
          if (flaguse[(iff - 1) + (size_t)mitot_patch * (jf - 1)] == 0) {
            for (int n = 1; n <= nvar; ++n) {
              const double valp10 = CI(n, ic + 1, jc), valm10 = CI(n, ic - 1, jc), valc = CI(n, ic, jc);
              const double valp01 = CI(n, ic, jc + 1), valm01 = CI(n, ic, jc - 1);
              const double dupc = valp10 - valc, dumc = valc - valm10, ducc = valp10 - valm10;
              double du = std::min(std::fabs(dupc), std::fabs(dumc));
              du = std::min(2.0 * du, 0.5 * std::fabs(ducc));
              const double fu = std::max(0.0, dsign(1.0, dupc * dumc));
              const double uslope = du * dsign(1.0, ducc) * fu;
              const double dvpc = valp01 - valc, dvmc = valc - valm01, dvcc = valp01 - valm01;
              double dv = std::min(std::fabs(dvpc), std::fabs(dvmc));
              dv = std::min(2.0 * dv, 0.5 * std::fabs(dvcc));
              const double fv = std::max(0.0, dsign(1.0, dvpc * dvmc));
              const double vslope = dv * dsign(1.0, dvcc) * fv;
              const double valint = valc + eta1 * uslope + eta2 * vslope;
              VB(n, iff + nrowst - 1, jf + ncolst - 1) = valint;
            }
          }
        }
      }
    }
    const double xhi_fine = xlower + (ihi + 1) * dx_fine, yhi_fine = ylower + (jhi + 1) * dy_fine;
    if (patchOnly) bc2amr(valbig, mitot, mjtot, dx_fine, dy_fine, xlow_fine, xhi_fine, ylow_fine, yhi_fine);
  }

  // prefilp.f90:18-214 (non-spherical branch)
  void prefilrecur(int level, double* valbig, int mitot, int mjtot, double t, int nrowst, int ncolst, int ilo, int ihi,
                   int jlo, int jhi, int iglo, int ighi, int jglo, int jghi, bool patchOnly) {
    (void)nrowst; (void)ncolst; (void)ighi; (void)jghi; (void)patchOnly;
    int ist[3], iend[3], jst[3], jend[3], ishift[3], jshift[3];
    if (xperdom) {
      ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[level];
      iend[0] = -1; iend[1] = iregsz[level] - 1; iend[2] = ihi;
      ishift[0] = iregsz[level]; ishift[1] = 0; ishift[2] = -iregsz[level];
    } else {
      ist[0] = iregsz[level]; ist[1] = ilo; ist[2] = iregsz[level];
      iend[0] = -1; iend[1] = ihi; iend[2] = -1;
      ishift[0] = ishift[1] = ishift[2] = 0;
    }
    if (yperdom || spheredom) {
      jst[0] = jlo; jst[1] = 0; jst[2] = jregsz[level];
      jend[0] = -1; jend[1] = jregsz[level] - 1; jend[2] = jhi;
      jshift[0] = jregsz[level]; jshift[1] = 0; jshift[2] = -jregsz[level];
    } else {
      jst[0] = jregsz[level]; jst[1] = jlo; jst[2] = jregsz[level];
      jend[0] = -1; jend[1] = jhi; jend[2] = -1;
      jshift[0] = jshift[1] = jshift[2] = 0;
    }
    FArr VB{valbig, nvar, mitot, mjtot};
    for (int i = 0; i < 3; ++i) {
      const int i1 = std::max(ilo, ist[i]), i2 = std::min(ihi, iend[i]);
      if (i1 > i2) continue;
      for (int j = 0; j < 3; ++j) {
        const int j1 = std::max(jlo, jst[j]), j2 = std::min(jhi, jend[j]);
        if (j1 > j2) continue;
        const int mi = i2 - i1 + 1, mj = j2 - j1 + 1;
        std::vector<double> valPatch((size_t)mi * mj * nvar, 0.0);
        filrecur(level, valPatch.data(), mi, mj, t, 1, 1, i1 + ishift[i], i2 + ishift[i], j1 + jshift[j], j2 + jshift[j], true, -1);
        // patchCopyOut
        const int is = i1 - iglo + 1, js = j1 - jglo + 1;
        FArr VP{valPatch.data(), nvar, mi, mj};
        for (int jj = 1; jj <= mj; ++jj) for (int ii = 1; ii <= mi; ++ii) for (int m = 1; m <= nvar; ++m)
          VB(m, is + ii - 1, js + jj - 1) = VP(m, ii, jj);
      }
    }
  }

  // bound.f90:51-158
  void bound(double t, int ng, double* valbig, int mitot, int mjtot, int mptr) {
    const Node2& g = node[mptr];
    const double xleft = g.xlo, xright = g.xhi, ybot = g.ylo, ytop = g.yhi;
    const int ilo = g.ilo, ihi = g.ihi, jlo = g.jlo, jhi = g.jhi, level = g.level;
    const double hx = hxposs[level], hy = hyposs[level];
    const double xloG = xleft - ng * hx, xhiG = xright + ng * hx, yloG = ybot - ng * hy, yhiG = ytop + ng * hy;
    double xl, xr, yb, yt;
    // left
    xl = xleft - ng * hx;
    if ((xl < xlower) && xperdom)
      prefilrecur(level, valbig, mitot, mjtot, t, 1, ng + 1, ilo - ng, ilo - 1, jlo, jhi, ilo - ng, ihi + ng, jlo - ng, jhi + ng, false);
    else
      filrecur(level, valbig, mitot, mjtot, t, 1, ng + 1, ilo - ng, ilo - 1, jlo, jhi, false, mptr);
    // right
    xr = xright + ng * hx;
    if ((xr > xupper) && xperdom)
      prefilrecur(level, valbig, mitot, mjtot, t, mitot - ng + 1, ng + 1, ihi + 1, ihi + ng, jlo, jhi, ilo - ng, ihi + ng, jlo - ng, jhi + ng, false);
    else
      filrecur(level, valbig, mitot, mjtot, t, mitot - ng + 1, ng + 1, ihi + 1, ihi + ng, jlo, jhi, false, mptr);
    // bottom
    xl = xleft - ng * hx; xr = xright + ng * hx; yb = ybot - ng * hy;
    if (((yb < ylower) && (yperdom || spheredom)) || (((xl < xlower) || (xr > xupper)) && xperdom))
      prefilrecur(level, valbig, mitot, mjtot, t, 1, 1, ilo - ng, ihi + ng, jlo - ng, jlo - 1, ilo - ng, ihi + ng, jlo - ng, jhi + ng, false);
    else
      filrecur(level, valbig, mitot, mjtot, t, 1, 1, ilo - ng, ihi + ng, jlo - ng, jlo - 1, false, mptr);
    // top
    yt = ytop + ng * hy;
    if (((yt > yupper) && (yperdom || spheredom)) || (((xl < xlower) || (xr > xupper)) && xperdom))
      prefilrecur(level, valbig, mitot, mjtot, t, 1, mjtot - ng + 1, ilo - ng, ihi + ng, jhi + 1, jhi + ng, ilo - ng, ihi + ng, jlo - ng, jhi + ng, false);
    else
      filrecur(level, valbig, mitot, mjtot, t, 1, mjtot - ng + 1, ilo - ng, ihi + ng, jhi + 1, jhi + ng, false, mptr);
    bc2amr(valbig, mitot, mjtot, hx, hy, xloG, xhiG, yloG, yhiG);
  }

  // =================================================== same-level copies (icall / intcopy)
  // icall.f: q and (auxp != nullptr) aux of the intersecting grids' interiors
  void icall(double* valp, int nrow, int ncol, int ilo, int ihi, int jlo, int jhi, int level, int iputst, int jputst,
             double* auxp = nullptr) {
    FArr val{valp, nvar, nrow, ncol}, aux{auxp, naux, nrow, ncol};
    for (int mptr = lstart[level]; mptr != 0; mptr = node[mptr].levelptr) {
      const Node2& g = node[mptr];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi), jxlo = std::max(g.jlo, jlo), jxhi = std::min(g.jhi, jhi);
      if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
      const int mitot = mitot_of(mptr);
      for (int j = jxlo; j <= jxhi; ++j)
        for (int i = ixlo; i <= ixhi; ++i) {
          const size_t at = (j - g.jlo + nghost) * (size_t)mitot + (i - g.ilo + nghost);
          for (int ivar = 1; ivar <= nvar; ++ivar) val(ivar, i - ilo + iputst, j - jlo + jputst) = g.q1[(ivar - 1) + (size_t)nvar * at];
          if (auxp)
            for (int ia = 1; ia <= naux; ++ia) aux(ia, i - ilo + iputst, j - jlo + jputst) = g.aux[(ia - 1) + (size_t)naux * at];
        }
    }
  }
  void intcopy(double* valp, int nrow, int ncol, int ilo, int ihi, int jlo, int jhi, int level, int iputst, int jputst) {
    icall(valp, nrow, ncol, ilo, ihi, jlo, jhi, level, iputst, jputst);  // identical for naux = 0
  }
  // preintcopy.f / preicall.f (non-spherical branch; aux with auxp)
  void preintcopy(double* valp, int nrow, int ncol, int ilo, int ihi, int jlo, int jhi, int level, double* auxp = nullptr) {
    int ist[3], iend[3], jst[3], jend[3], ishift[3], jshift[3];
    if (xperdom) {
      ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[level]; iend[0] = -1; iend[1] = iregsz[level] - 1; iend[2] = ihi;
      ishift[0] = iregsz[level]; ishift[1] = 0; ishift[2] = -iregsz[level];
    } else {
      ist[0] = iregsz[level]; ist[1] = ilo; ist[2] = iregsz[level]; iend[0] = -1; iend[1] = ihi; iend[2] = -1;
      ishift[0] = ishift[1] = ishift[2] = 0;
    }
    if (yperdom || spheredom) {
      jst[0] = jlo; jst[1] = 0; jst[2] = jregsz[level]; jend[0] = -1; jend[1] = jregsz[level] - 1; jend[2] = jhi;
      jshift[0] = jregsz[level]; jshift[1] = 0; jshift[2] = -jregsz[level];
    } else {
      jst[0] = jregsz[level]; jst[1] = jlo; jst[2] = jregsz[level]; jend[0] = -1; jend[1] = jhi; jend[2] = -1;
      jshift[0] = jshift[1] = jshift[2] = 0;
    }
    for (int i = 0; i < 3; ++i) {
      const int i1 = std::max(ilo, ist[i]), i2 = std::min(ihi, iend[i]);
      if (i1 > i2) continue;
      for (int j = 0; j < 3; ++j) {
        const int j1 = std::max(jlo, jst[j]), j2 = std::min(jhi, jend[j]);
        if (j1 > j2) continue;
        icall(valp, nrow, ncol, i1 + ishift[i], i2 + ishift[i], j1 + jshift[j], j2 + jshift[j], level, (i1 - ilo) + 1, (j1 - jlo) + 1,
              auxp);
      }
    }
  }

  // ======================================================= saveqc / cstore
  void saveqc(int level) {
    const int levc = level - 1;
    const double hxc = hxposs[levc], hyc = hyposs[levc];
    for (int mkid = lstart[level]; mkid != 0; mkid = node[mkid].levelptr) {
      Node2& k = node[mkid];
      const int nxk = k.ihi - k.ilo + 1, nyk = k.jhi - k.jlo + 1;
      const int ikeep = nxk / intratx[level - 1], jkeep = nyk / intraty[level - 1];
      const int lenbc = 2 * (ikeep + jkeep);
      const double time_k = k.time;
      const int iclo = k.ilo / intratx[level - 1] - 1, jclo = k.jlo / intraty[level - 1] - 1;
      const int ichi = (k.ihi + 1) / intratx[level - 1], jchi = (k.jhi + 1) / intraty[level - 1];
      const int nrow = ichi - iclo + 1, ncol = jchi - jclo + 1;
      const double xl = k.xlo - hxc, yb = k.ylo - hyc, xr = k.xhi + hxc, yt = k.yhi + hyc;
      std::vector<double> tmp((size_t)nrow * ncol * nvar, 0.0), tx((size_t)nrow * ncol * naux, NEEDS_TO_BE_SET);
      double* txp = naux > 0 ? tx.data() : nullptr;
      const bool sticks = (iclo < 0 || ichi == iregsz[levc] || jclo < 0 || jchi == jregsz[levc]);
      if (sticks && (xperdom || yperdom || spheredom)) preintcopy(tmp.data(), nrow, ncol, iclo, ichi, jclo, jchi, level - 1, txp);
      else icall(tmp.data(), nrow, ncol, iclo, ichi, jclo, jchi, level - 1, 1, 1, txp);
      // saveqc.f:86-90: the ring's aux where it leaves the domain
      if (naux > 0 && sticks) setaux(0, nrow, ncol, xl, yb, hxc, hyc, txp);
      bc2amr(tmp.data(), nrow, ncol, hxc, hyc, xl, xr, yb, yt);
      // cstore.f:4-63
      FArr qc{tmp.data(), nvar, nrow, ncol};
      double* qc1d = k.ffl.data() + (size_t)nvar * lenbc;
      int index = 0;
      FArr ac{txp, naux, nrow, ncol};
      double* auxc1d = k.ffl.data() + (size_t)2 * nvar * lenbc;
      auto put = [&](int ii, int jj) {
        ++index;
        for (int iv = 1; iv <= nvar; ++iv) qc1d[(iv - 1) + nvar * (index - 1)] = qc(iv, ii, jj);
        for (int ia = 1; ia <= naux; ++ia) auxc1d[(ia - 1) + naux * (index - 1)] = ac(ia, ii, jj);
      };
      for (int j = 2; j <= ncol - 1; ++j) put(1, j);
      for (int i = 2; i <= nrow - 1; ++i) put(i, ncol);
      for (int j = 2; j <= ncol - 1; ++j) put(nrow, j);
      for (int i = 2; i <= nrow - 1; ++i) put(i, 1);
      (void)time_k;
    }
  }

  // ================================================================== qad
  // qad.f:4-370. aux: the fine grid's aux (naux, mitot, mjtot), auxc1d: the coarse ring's
  // (naux, lenbc); the aux of each Riemann problem comes from the cell of its q, except that
  // a face-type component (xleft / yleft) on the fine grid's lower face takes the fine
  // cell's own face value (qad.f:79-89, 175-185, 246-256, 298-308)
  void qad(double* valbigp, int mitot, int mjtot, double* svdflx, const double* qc1d, int lenbc, int lratiox, int lratioy,
           double hx, double hy, double delt, const double* aux, const double* auxc1d) {
    (void)lenbc;
    FArr valbig{valbigp, nvar, mitot, mjtot};
    const int max1dp1 = std::max(mitot, mjtot) + 2;
    const int mbc = nghost;
    std::vector<double> ql((size_t)nvar * max1dp1, 0.0), qr = ql, amdq = ql, apdq = ql;
    std::vector<double> wave((size_t)nvar * mwaves * max1dp1, 0.0), s((size_t)mwaves * max1dp1, 0.0), auxd(8, 0.0);
    // position p (1-based) <-> solver index p - mbc
    Slice QL{ql.data(), nvar, 1 - mbc + 0}, QR{qr.data(), nvar, 1 - mbc};
    QL.base = 1 - mbc; QR.base = 1 - mbc;
    auto pl = [&](int m, int p) -> double& { return ql[(m - 1) + nvar * (p - 1)]; };
    auto pr = [&](int m, int p) -> double& { return qr[(m - 1) + nvar * (p - 1)]; };
    auto pam = [&](int m, int p) { return amdq[(m - 1) + nvar * (p - 1)]; };
    auto pap = [&](int m, int p) { return apdq[(m - 1) + nvar * (p - 1)]; };
    auto SV = [&](int m, int k) -> double& { return svdflx[(m - 1) + nvar * (k - 1)]; };
    auto QC = [&](int m, int k) { return qc1d[(m - 1) + nvar * (k - 1)]; };
    Slice AM{amdq.data(), nvar, 1 - mbc}, AP{apdq.data(), nvar, 1 - mbc};
    Waves WV{wave.data(), nvar, mwaves, 1 - mbc};
    Slice S{s.data(), mwaves, 1 - mbc};
    (void)auxd;
    const int la = std::max(naux, 1);
    std::vector<double> auxl((size_t)la * max1dp1, 0.0), auxr = auxl;
    Slice AXL{auxl.data(), la, 1 - mbc}, AXR{auxr.data(), la, 1 - mbc};
    auto al = [&](int ma, int p) -> double& { return auxl[(ma - 1) + la * (p - 1)]; };
    auto ar = [&](int ma, int p) -> double& { return auxr[(ma - 1) + la * (p - 1)]; };
    FArr AF{(double*)aux, naux, mitot, mjtot};
    auto AC = [&](int ma, int k) { return auxc1d[(ma - 1) + naux * (k - 1)]; };
    auto is_type = [&](int ma, const char* t) { return auxtype[ma - 1] == t; };
    const int nc = mjtot - 2 * nghost, nr = mitot - 2 * nghost;
    int index = 0;
    // side 1
    for (int j = nghost + 1; j <= mjtot - nghost; ++j) {
      for (int ma = 1; ma <= naux; ++ma) al(ma, j - nghost + 1) = is_type(ma, "xleft") ? AF(ma, nghost + 1, j) : AF(ma, nghost, j);
      for (int iv = 1; iv <= nvar; ++iv) pl(iv, j - nghost + 1) = valbig(iv, nghost, j);
    }
    int lind = 0;
    for (int jc = 1; jc <= (mjtot - 2 * nghost) / lratioy; ++jc) {
      ++index;
      for (int l = 1; l <= lratioy; ++l) {
        ++lind;
        for (int ma = 1; ma <= naux; ++ma) ar(ma, lind) = AC(ma, index);
        for (int iv = 1; iv <= nvar; ++iv) pr(iv, lind) = QC(iv, index);
      }
    }
    rpn2(prob, 1, nvar, mwaves, mbc, nc + 1 - 2 * nghost, QL, QR, AXL, AXR, WV, S, AM, AP);
    int influx = 0;
    for (int j = 1; j <= nc / lratioy; ++j) {
      ++influx;
      const int jfine = (j - 1) * lratioy;
      for (int iv = 1; iv <= nvar; ++iv)
        for (int l = 1; l <= lratioy; ++l)
          SV(iv, influx) = SV(iv, influx) + pam(iv, jfine + l + 1) * hy * delt + pap(iv, jfine + l + 1) * hy * delt;
    }
    // side 2
    if (mjtot != 2 * nghost + 1) {
      for (int i = nghost + 1; i <= mitot - nghost; ++i) {
        for (int ma = 1; ma <= naux; ++ma) ar(ma, i - nghost) = AF(ma, i, mjtot - nghost + 1);
        for (int iv = 1; iv <= nvar; ++iv) pr(iv, i - nghost) = valbig(iv, i, mjtot - nghost + 1);
      }
      lind = 0;
      for (int ic = 1; ic <= (mitot - 2 * nghost) / lratiox; ++ic) {
        ++index;
        for (int l = 1; l <= lratiox; ++l) {
          ++lind;
          for (int ma = 1; ma <= naux; ++ma)
            al(ma, lind + 1) = is_type(ma, "yleft") ? AF(ma, (ic - 1) * lratiox + nghost + l, mjtot - nghost + 1) : AC(ma, index);
          for (int iv = 1; iv <= nvar; ++iv) pl(iv, lind + 1) = QC(iv, index);
        }
      }
      rpn2(prob, 2, nvar, mwaves, mbc, nr + 1 - 2 * nghost, QL, QR, AXL, AXR, WV, S, AM, AP);
      for (int i = 1; i <= nr / lratiox; ++i) {
        ++influx;
        const int ifine = (i - 1) * lratiox;
        for (int iv = 1; iv <= nvar; ++iv)
          for (int l = 1; l <= lratiox; ++l)
            SV(iv, influx) = SV(iv, influx) - pam(iv, ifine + l + 1) * hx * delt - pap(iv, ifine + l + 1) * hx * delt;
      }
    }
    // side 3
    for (int j = nghost + 1; j <= mjtot - nghost; ++j) {
      for (int ma = 1; ma <= naux; ++ma) ar(ma, j - nghost) = AF(ma, mitot - nghost + 1, j);
      for (int iv = 1; iv <= nvar; ++iv) pr(iv, j - nghost) = valbig(iv, mitot - nghost + 1, j);
    }
    lind = 0;
    for (int jc = 1; jc <= (mjtot - 2 * nghost) / lratioy; ++jc) {
      ++index;
      for (int l = 1; l <= lratioy; ++l) {
        ++lind;
        for (int ma = 1; ma <= naux; ++ma)
          al(ma, lind + 1) = is_type(ma, "xleft") ? AF(ma, mitot - nghost + 1, (jc - 1) * lratioy + nghost + l) : AC(ma, index);
        for (int iv = 1; iv <= nvar; ++iv) pl(iv, lind + 1) = QC(iv, index);
      }
    }
    rpn2(prob, 1, nvar, mwaves, mbc, nc + 1 - 2 * nghost, QL, QR, AXL, AXR, WV, S, AM, AP);
    for (int j = 1; j <= nc / lratioy; ++j) {
      ++influx;
      const int jfine = (j - 1) * lratioy;
      for (int iv = 1; iv <= nvar; ++iv)
        for (int l = 1; l <= lratioy; ++l)
          SV(iv, influx) = SV(iv, influx) - pam(iv, jfine + l + 1) * hy * delt - pap(iv, jfine + l + 1) * hy * delt;
    }
    // side 4
    if (mjtot != 2 * nghost + 1) {
      for (int i = nghost + 1; i <= mitot - nghost; ++i) {
        for (int ma = 1; ma <= naux; ++ma) al(ma, i - nghost + 1) = is_type(ma, "yleft") ? AF(ma, i, nghost + 1) : AF(ma, i, nghost);
        for (int iv = 1; iv <= nvar; ++iv) pl(iv, i - nghost + 1) = valbig(iv, i, nghost);
      }
      lind = 0;
      for (int ic = 1; ic <= (mitot - 2 * nghost) / lratiox; ++ic) {
        ++index;
        for (int l = 1; l <= lratiox; ++l) {
          ++lind;
          for (int ma = 1; ma <= naux; ++ma) ar(ma, lind) = AC(ma, index);
          for (int iv = 1; iv <= nvar; ++iv) pr(iv, lind) = QC(iv, index);
        }
      }
      rpn2(prob, 2, nvar, mwaves, mbc, nr + 1 - 2 * nghost, QL, QR, AXL, AXR, WV, S, AM, AP);
      for (int i = 1; i <= nr / lratiox; ++i) {
        ++influx;
        const int ifine = (i - 1) * lratiox;
        for (int iv = 1; iv <= nvar; ++iv)
          for (int l = 1; l <= lratiox; ++l)
            SV(iv, influx) = SV(iv, influx) + pam(iv, ifine + l + 1) * hx * delt + pap(iv, ifine + l + 1) * hx * delt;
      }
    }
  }

  // ================================================================ fluxsv / fluxad
  void fluxsv(int mptr, const double* fm, const double* fp, const double* gm, const double* gp, int mitot, int mjtot, double dtc, double hx, double hy) {
    FArr FM{(double*)fm, nvar, mitot, mjtot}, FP{(double*)fp, nvar, mitot, mjtot}, GM{(double*)gm, nvar, mitot, mjtot}, GP{(double*)gp, nvar, mitot, mjtot};
    const int level = node[mptr].level;
    const int maxsp = listsp[level];
    const std::vector<int>& L = node[mptr].listbc;
    for (int ispot = 1; ispot <= maxsp; ++ispot) {
      auto LB = [&](int k) { return L[(k - 1) + 5 * (ispot - 1)]; };
      if (LB(1) == 0) break;
      const int mkid = LB(4), intopl = LB(5);
      double* svd = node[mkid].ffl.data();
      const int i = LB(1), j = LB(2);
      double* dst = svd + (size_t)nvar * (intopl - 1);
      const int side = LB(3);
      for (int iv = 1; iv <= nvar; ++iv) {
        if (side == 1) dst[iv - 1] = -FP(iv, i, j) * dtc * hy;
        else if (side == 2) dst[iv - 1] = -GM(iv, i, j + 1) * dtc * hx;
        else if (side == 3) dst[iv - 1] = -FM(iv, i + 1, j) * dtc * hy;
        else if (side == 4) dst[iv - 1] = -GP(iv, i, j) * dtc * hx;
      }
    }
  }
  void fluxad(const double* fm, const double* fp, const double* gm, const double* gp, double* svdflx, int mitot, int mjtot,
              int lratiox, int lratioy, int ng, double dtf, double dx, double dy) {
    FArr XM{(double*)fm, nvar, mitot, mjtot}, XP{(double*)fp, nvar, mitot, mjtot}, YM{(double*)gm, nvar, mitot, mjtot}, YP{(double*)gp, nvar, mitot, mjtot};
    auto SV = [&](int m, int k) -> double& { return svdflx[(m - 1) + nvar * (k - 1)]; };
    const int nxf = mitot - 2 * ng, nyf = mjtot - 2 * ng;
    const int nyc = nyf / lratioy, nxc = nxf / lratiox;
    int lind = 0;
    for (int j = 1; j <= nyc; ++j) {
      ++lind; const int jfine = (j - 1) * lratioy + ng;
      for (int iv = 1; iv <= nvar; ++iv) for (int l = 1; l <= lratioy; ++l) SV(iv, lind) = SV(iv, lind) + XM(iv, ng + 1, jfine + l) * dtf * dy;
    }
    for (int i = 1; i <= nxc; ++i) {
      ++lind; const int ifine = (i - 1) * lratiox + ng;
      for (int iv = 1; iv <= nvar; ++iv) for (int l = 1; l <= lratiox; ++l) SV(iv, lind) = SV(iv, lind) + YP(iv, ifine + l, mjtot - ng + 1) * dtf * dx;
    }
    for (int j = 1; j <= nyc; ++j) {
      ++lind; const int jfine = (j - 1) * lratioy + ng;
      for (int iv = 1; iv <= nvar; ++iv) for (int l = 1; l <= lratioy; ++l) SV(iv, lind) = SV(iv, lind) + XP(iv, mitot - ng + 1, jfine + l) * dtf * dy;
    }
    for (int i = 1; i <= nxc; ++i) {
      ++lind; const int ifine = (i - 1) * lratiox + ng;
      for (int iv = 1; iv <= nvar; ++iv) for (int l = 1; l <= lratiox; ++l) SV(iv, lind) = SV(iv, lind) + YM(iv, ifine + l, ng + 1) * dtf * dx;
    }
  }

  // ================================================================ advanc
  struct GridTiming { double seconds = 0; };
  double dtlevnew_last = 0;

  void update_gauges(const double* q, double xlow, double ylow, int mitot, int mjtot, int mptr) {
    if (!record_gauges) return;
    const double tgrid = node[mptr].time;
    const int level = node[mptr].level;
    const double hx = hxposs[level], hy = hyposs[level];
    FArr Q{(double*)q, nvar, mitot, mjtot};
    for (size_t i = 0; i < gauges.size(); ++i) {
      Gauge& g = gauges[i];
      if (mptr != mbestsrc[i]) continue;
      if (tgrid < g.t_start || tgrid > g.t_end) continue;
      if (tgrid - g.last_time < g.min_inc) continue;
      const int ii = (int)(0.5 + (g.x - xlow) / hx);
      const int jj = (int)(0.5 + (g.y - ylow) / hy);
      const double xc = xlow + (ii - 0.5) * hx, yc = ylow + (jj - 0.5) * hy;
      const double xoff = (g.x - xc) / hx, yoff = (g.y - yc) / hy;
      GaugeSample smp; smp.level = level; smp.t = tgrid;
      for (int n = 1; n <= nvar; ++n) {
        double v = (1.0 - xoff) * (1.0 - yoff) * Q(n, ii, jj) + xoff * (1.0 - yoff) * Q(n, ii + 1, jj) +
                   (1.0 - xoff) * yoff * Q(n, ii, jj + 1) + xoff * yoff * Q(n, ii + 1, jj + 1);
        if (std::fabs(v) < 1e-90) v = 0.0;
        smp.v.push_back(v);
      }
      g.data.push_back(smp);
      g.last_time = tgrid;
    }
  }

  void par_advanc(int mptr, double& dtnew, double& cflgrid) {
    Node2& g = node[mptr];
    const int level = g.level;
    const double hx = hxposs[level], hy = hyposs[level], delt = possk[level];
    const int nxg = g.ihi - g.ilo + 1, nyg = g.jhi - g.jlo + 1;
    const int mitot = nxg + 2 * nghost, mjtot = nyg + 2 * nghost;
    if (level < mxnest || dbg_keep_input) g.q2 = g.q1;
    const double xlow = g.xlo - nghost * hx, ylow = g.ylo - nghost * hy;
    if (g.has_ffl) {
      const int lenbc = 2 * (nxg / intratx[level - 1] + nyg / intraty[level - 1]);
      qad(g.q1.data(), mitot, mjtot, g.ffl.data(), g.ffl.data() + (size_t)nvar * lenbc, lenbc, intratx[level - 1], intraty[level - 1], hx, hy, delt,
          g.aux.data(), g.ffl.data() + (size_t)2 * nvar * lenbc);
    }
    if (!gauges.empty()) update_gauges(g.q1.data(), xlow, ylow, mitot, mjtot, mptr);
    const size_t nf = (size_t)nvar * mitot * mjtot;
    std::vector<double> fm(nf), fp(nf), gm(nf), gp(nf);
    // advanc.f:256-270: unsplit or Godunov-split step
    if (dimensional_split == 0)
      stepgrid(g.q1.data(), fm.data(), fp.data(), gm.data(), gp.data(), mitot, mjtot, nghost, delt, dtnew, hx, hy,
               g.aux.data(), cflgrid);
    else
      stepgrid_dimSplit(g.q1.data(), fm.data(), fp.data(), gm.data(), gp.data(), mitot, mjtot, nghost, delt, dtnew, hx,
                        hy, g.aux.data(), cflgrid);
    if (g.has_cfl) fluxsv(mptr, fm.data(), fp.data(), gm.data(), gp.data(), mitot, mjtot, delt, hx, hy);
    if (g.has_ffl) {
      const int lenbc = 2 * (nxg / intratx[level - 1] + nyg / intraty[level - 1]);
      (void)lenbc;
      fluxad(fm.data(), fp.data(), gm.data(), gp.data(), g.ffl.data(), mitot, mjtot, intratx[level - 1], intraty[level - 1], nghost, delt, hx, hy);
    }
    g.time = g.time + delt;
  }

  void advanc(int level, double& dtlevnew) {
    const std::vector<int> grids = levelgrids[level];
    const int n = (int)grids.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int k = 0; k < n; ++k) {
      const int mptr = grids[k];
      Node2& g = node[mptr];
      bound(g.time, nghost, g.q1.data(), mitot_of(mptr), mjtot_of(mptr), mptr);
    }
    if (level + 1 <= mxnest && lstart[level + 1] != 0) saveqc(level + 1);
    dtlevnew = RINFINITY;
    cfl_level = 0.0;
    std::vector<double> dtn(n), cfg(n);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int k = 0; k < n; ++k) par_advanc(grids[k], dtn[k], cfg[k]);
    for (int k = 0; k < n; ++k) {
      const Node2& g = node[grids[k]];
      const double cells = (double)(g.ihi - g.ilo + 1) * (g.jhi - g.jlo + 1);
      rvol += cells; rvoll[level] += cells;
      dtlevnew = std::min(dtlevnew, dtn[k]);
      cfl_level = std::max(cfl_level, cfg[k]);
    }
    cflmax = std::max(cflmax, cfl_level);
  }

  // ================================================================ update / upbnd
  void upbnd(const std::vector<int>& listbc, double* valp, int mitot, int mjtot, int maxsp, int mptr) {
    FArr val{valp, nvar, mitot, mjtot};
    std::vector<int> iused((size_t)mitot * mjtot, 0);
    const int levc = node[mptr].level;
    const double area = hxposs[levc] * hyposs[levc];
    for (int ispot = 1; ispot <= maxsp; ++ispot) {
      auto LB = [&](int k) { return listbc[(k - 1) + 5 * (ispot - 1)]; };
      const int icrse = LB(1);
      if (icrse == 0) break;
      const int jcrse = LB(2), iside = LB(3);
      int iside1 = iside < 5 ? iside : (iside == 5 ? 2 : 4);
      const int norm = 1 << (iside1 - 1);
      int& used = iused[(icrse - 1) + (size_t)mitot * (jcrse - 1)];
      const int iflag = used / norm;
      if (iflag % 2 == 1) continue;
      const int mkid = LB(4), lkid = LB(5);
      double sgnm = (iside == 2 || iside == 3 || iside == 6) ? -1.0 : 1.0;
      // upbnd.f:104-108: with a capacity array the correction is divided by kappa
      if (mcapa > 0) sgnm = sgnm / node[mptr].aux[(mcapa - 1) + (size_t)naux * ((icrse - 1) + (size_t)mitot * (jcrse - 1))];
      const double* svd = node[mkid].ffl.data();
      for (int iv = 1; iv <= nvar; ++iv)
        val(iv, icrse, jcrse) = val(iv, icrse, jcrse) + sgnm * svd[(size_t)nvar * (lkid - 1) + iv - 1] / area;
      used += norm;
    }
  }

  void update(int level) {
    const int lget = level;
    for (int mptr : levelgrids[lget]) {
      Node2& g = node[mptr];
      const int mitot = mitot_of(mptr);
      if (g.has_cfl) upbnd(g.listbc, g.q1.data(), mitot, mjtot_of(mptr), listsp[lget], mptr);
      FArr Q{g.q1.data(), nvar, mitot, mjtot_of(mptr)};
      for (int mkid = lstart[lget + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        const Node2& k = node[mkid];
        const int iclo = k.ilo / intratx[lget], jclo = k.jlo / intraty[lget];
        const int ichi = k.ihi / intratx[lget], jchi = k.jhi / intraty[lget];
        const int mi = k.ihi - k.ilo + 1 + 2 * nghost;
        const int iplo = std::max(g.ilo, iclo), jplo = std::max(g.jlo, jclo);
        const int iphi = std::min(g.ihi, ichi), jphi = std::min(g.jhi, jchi);
        if (iplo > iphi || jplo > jphi) continue;
        int iff = iplo * intratx[lget] - k.ilo + nghost + 1;
        int jff = jplo * intraty[lget] - k.jlo + nghost + 1;
        const double totrat = intratx[lget] * intraty[lget];
        auto F = [&](int iv, int i, int j) { return k.q1[(iv - 1) + (size_t)nvar * ((j - 1) * (size_t)mi + i - 1)]; };
        auto FA = [&](int i, int j) { return k.aux[(mcapa - 1) + (size_t)naux * ((j - 1) * (size_t)mi + i - 1)]; };
        auto CA = [&](int i, int j) { return g.aux[(mcapa - 1) + (size_t)naux * ((j - 1) * (size_t)mitot + i - 1)]; };
        for (int i = iplo - g.ilo + nghost + 1; i <= iphi - g.ilo + nghost + 1; ++i) {
          for (int j = jplo - g.jlo + nghost + 1; j <= jphi - g.jlo + nghost + 1; ++j) {
            for (int iv = 1; iv <= nvar; ++iv) Q(iv, i, j) = 0.0;
            if (mcapa == 0) {
              for (int jco = 1; jco <= intraty[lget]; ++jco)
                for (int ico = 1; ico <= intratx[lget]; ++ico)
                  for (int iv = 1; iv <= nvar; ++iv) Q(iv, i, j) = Q(iv, i, j) + F(iv, iff + ico - 1, jff + jco - 1);
              for (int iv = 1; iv <= nvar; ++iv) Q(iv, i, j) = Q(iv, i, j) / totrat;
            } else {
              // update.f:150-160: kappa-weighted average of the fine cells
              for (int jco = 1; jco <= intraty[lget]; ++jco)
                for (int ico = 1; ico <= intratx[lget]; ++ico) {
                  const double capa = FA(iff + ico - 1, jff + jco - 1);
                  for (int iv = 1; iv <= nvar; ++iv) Q(iv, i, j) = Q(iv, i, j) + F(iv, iff + ico - 1, jff + jco - 1) * capa;
                }
              for (int iv = 1; iv <= nvar; ++iv) Q(iv, i, j) = Q(iv, i, j) / (totrat * CA(i, j));
            }
            jff += intraty[lget];
          }
          iff += intratx[lget];
          jff = jplo * intraty[lget] - k.jlo + nghost + 1;
        }
      }
    }
  }

  // ================================================================ prepf / prepc / setuse
  void prepf(int level) {
    for (int mkid = lstart[level]; mkid != 0; mkid = node[mkid].levelptr) {
      Node2& k = node[mkid];
      const int ikeep = (k.ihi - k.ilo + 1) / intratx[level - 1], jkeep = (k.jhi - k.jlo + 1) / intraty[level - 1];
      const int lenbc = 2 * (ikeep + jkeep);
      k.ffl.assign((size_t)2 * nvar * lenbc + (size_t)naux * lenbc, 0.0);
      k.has_ffl = true;
    }
  }
  void setuse(std::vector<int>& listbc, int maxsp, int& ispot, int mkid, int ilo, int ihi, int jlo, int jhi, int iclo,
              int ichi, int jclo, int jchi, int kflag) {
    auto LB = [&](int k, int sp) -> int& { return listbc[(k - 1) + 5 * (sp - 1)]; };
    (void)maxsp;
    const int ist = iclo - 1, iend = ichi + 1, jst = jclo - 1, jend = jchi + 1;
    if (!(ist < ilo || kflag != 1)) {
      int lkid = std::max(jlo, jclo) - jclo + 1;
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) {
        ++ispot;
        LB(1, ispot) = ist - ilo + nghost + 1; LB(2, ispot) = j - jlo + nghost + 1; LB(3, ispot) = 3;
        LB(4, ispot) = mkid; LB(5, ispot) = lkid; ++lkid;
      }
    }
    if (kflag == 1 && !(jend > jhi)) {
      int lkid = (jchi - jclo + 1) + std::max(ilo, iclo) - iclo + 1;
      for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) {
        ++ispot;
        LB(1, ispot) = i - ilo + nghost + 1; LB(2, ispot) = jend - jlo + nghost + 1; LB(3, ispot) = 4;
        LB(4, ispot) = mkid; LB(5, ispot) = lkid; ++lkid;
      }
    }
    if (!(iend > ihi || kflag != 1)) {
      int lkid = (ichi - iclo + 1) + (jchi - jclo + 1) + std::max(jlo, jclo) - jclo + 1;
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) {
        ++ispot;
        LB(1, ispot) = iend - ilo + nghost + 1; LB(2, ispot) = j - jlo + nghost + 1; LB(3, ispot) = 1;
        LB(4, ispot) = mkid; LB(5, ispot) = lkid; ++lkid;
      }
    }
    if (kflag == 1 && !(jst < jlo)) {
      int lkid = 2 * (jchi - jclo + 1) + (ichi - iclo + 1) + std::max(ilo, iclo) - iclo + 1;
      for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) {
        ++ispot;
        LB(1, ispot) = i - ilo + nghost + 1; LB(2, ispot) = jst - jlo + nghost + 1; LB(3, ispot) = 2;
        LB(4, ispot) = mkid; LB(5, ispot) = lkid; ++lkid;
      }
    }
  }
  void prepc(int level) {
    int maxsp = 0;
    for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
      const Node2& k = node[mkid];
      maxsp += 2 * ((k.ihi - k.ilo + 1) / intratx[level] + (k.jhi - k.jlo + 1) / intraty[level]);
    }
    listsp[level] = maxsp;
    if (maxsp == 0) return;
    const int imax = iregsz[level] - 1, jmax = jregsz[level] - 1;
    for (int mpar = lstart[level]; mpar != 0; mpar = node[mpar].levelptr) {
      int ispot = 0;
      Node2& p = node[mpar];
      const int ilo = p.ilo, jlo = p.jlo, ihi = p.ihi, jhi = p.jhi;
      p.listbc.assign((size_t)5 * maxsp, 0);
      p.has_cfl = true;
      for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        const Node2& k = node[mkid];
        const int iclo = k.ilo / intratx[level], jclo = k.jlo / intraty[level];
        const int ichi = k.ihi / intratx[level], jchi = k.jhi / intraty[level];
        const int iplo = std::max(ilo, iclo), jplo = std::max(jlo, jclo), iphi = std::min(ihi, ichi), jphi = std::min(jhi, jchi);
        if (iplo <= iphi + 1 && jplo <= jphi + 1) setuse(p.listbc, maxsp, ispot, mkid, ilo, ihi, jlo, jhi, iclo, ichi, jclo, jchi, 1);
        if (xperdom && ilo == 0 && ichi == imax)
          setuse(p.listbc, maxsp, ispot, mkid, ilo, ihi, jlo, jhi, iclo - iregsz[level], ichi - iregsz[level], jclo, jchi, 1);
        if (xperdom && iclo == 0 && ihi == imax)
          setuse(p.listbc, maxsp, ispot, mkid, ilo, ihi, jlo, jhi, iclo + iregsz[level], ichi + iregsz[level], jclo, jchi, 1);
        if (yperdom && jlo == 0 && jchi == jmax)
          setuse(p.listbc, maxsp, ispot, mkid, ilo, ihi, jlo, jhi, iclo, ichi, jclo - jregsz[level], jchi - jregsz[level], 1);
        if (yperdom && jclo == 0 && jhi == jmax)
          setuse(p.listbc, maxsp, ispot, mkid, ilo, ihi, jlo, jhi, iclo, ichi, jclo + jregsz[level], jchi + jregsz[level], 1);
      }
    }
  }
  void putsp(int lbase, int level) {
    if (level != lfine)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].listbc.clear(); node[m].has_cfl = false; }
    if (level == lbase) return;
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].ffl.clear(); node[m].has_ffl = false; }
  }

  // ================================================================ grid lists
  void makeGridList() {
    for (int lev = 1; lev <= mxnest + 1 && lev < 12; ++lev) {
      levelgrids[lev].clear();
      if (lev > mxnest) continue;
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) levelgrids[lev].push_back(m);
      numgrids[lev] = (int)levelgrids[lev].size();
    }
  }
  void makeBndryList(int level) {
    const std::vector<int>& G = levelgrids[level];
    for (size_t n = 0; n < G.size(); ++n) {
      const int mptr = G[n];
      Node2& g = node[mptr];
      g.bnd.clear();
      const int imin = g.ilo - nghost, imax = g.ihi + nghost, jmin = g.jlo - nghost, jmax = g.jhi + nghost;
      std::vector<int> found;
      for (size_t k = 0; k < G.size(); ++k) {
        if (k == n) continue;
        const Node2& s = node[G[k]];
        if (std::max(s.ilo, imin) <= std::min(s.ihi, imax) && std::max(s.jlo, jmin) <= std::min(s.jhi, jmax)) found.push_back(G[k]);
      }
      // pushed onto the front of the linked list: traversal is reverse discovery order
      for (auto it = found.rbegin(); it != found.rend(); ++it) g.bnd.push_back(*it);
    }
  }

  // quick_sort1.f:22-167 (qsorti, non-stable, replicated step by step)
  static void qsorti(std::vector<int>& ord, int n, const std::vector<long long>& a) {
    // ord and a are 1-based views (index 0 unused)
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

  // regrid.f:132-169
  void arrangeGrids(int level, int numg) {
    std::vector<int> listgrids(numg + 1), index(numg + 1);
    std::vector<long long> cost(numg + 1);
    int mptr = lstart[level];
    for (int i = 1; i <= numg; ++i) {
      listgrids[i] = mptr;
      cost[i] = (long long)(node[mptr].ihi - node[mptr].ilo + 3) * (node[mptr].jhi - node[mptr].jlo + 2);
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

  // ================================================================ birect.f
  void birect(int mptr1) {
    int mptr = mptr1;
    const int level = node[mptr].level;
    const double hx = hxposs[level], hy = hyposs[level];
    while (true) {
      const double cxlo = node[mptr].xlo, cxhi = node[mptr].xhi, cylo = node[mptr].ylo, cyhi = node[mptr].yhi;
      const int nxg = node[mptr].ihi - node[mptr].ilo + 1, nyg = node[mptr].jhi - node[mptr].jlo + 1;
      if (nxg + 2 * nghost > max1d) {
        int nxl = nxg / 2;
        const int lratio = level > 1 ? intratx[level - 1] : 2;
        nxl = (nxl / lratio) * lratio;
        const double cxmid = cxlo + nxl * hx;
        const int mn = nodget();
        node[mn].levelptr = node[mptr].levelptr; node[mptr].levelptr = mn;
        node[mptr].xhi = cxmid;
        node[mn].ihi = node[mptr].ihi; node[mptr].ihi = node[mptr].ilo + nxl - 1; node[mn].ilo = node[mptr].ihi + 1;
        node[mn].jhi = node[mptr].jhi; node[mn].jlo = node[mptr].jlo;
        node[mn].xlo = cxmid; node[mn].ylo = cylo; node[mn].yhi = cyhi; node[mn].xhi = cxhi;
        node[mn].time = node[mptr].time; node[mn].level = node[mptr].level;
        continue;
      } else if (nyg + 2 * nghost > max1d) {
        int nyl = nyg / 2;
        const int lratio = level > 1 ? intraty[level - 1] : 2;
        nyl = (nyl / lratio) * lratio;
        const double cymid = cylo + nyl * hy;
        const int mn = nodget();
        node[mn].levelptr = node[mptr].levelptr; node[mptr].levelptr = mn;
        node[mptr].yhi = cymid;
        node[mn].jhi = node[mptr].jhi; node[mptr].jhi = node[mptr].jlo + nyl - 1; node[mn].jlo = node[mptr].jhi + 1;
        node[mn].ihi = node[mptr].ihi; node[mn].ilo = node[mptr].ilo;
        node[mn].xlo = cxlo; node[mn].ylo = cymid; node[mn].yhi = cyhi; node[mn].xhi = cxhi;
        node[mn].level = node[mptr].level; node[mn].time = node[mptr].time;
        continue;
      } else {
        mptr = node[mptr].levelptr;
        if (mptr == 0) break;
      }
    }
  }

  // ================================================================ flagging
  void flagregions2(int mx, int my, int mbuff, double xl, double yl, double dx, double dy, int level, double t, double* amrflags) {
    const int ld = mx + 2 * mbuff;
    auto AF = [&](int i, int j) -> double& { return amrflags[(i + mbuff - 1) + (size_t)ld * (j + mbuff - 1)]; };
    std::vector<int> minl((size_t)mx * my, 0), maxl((size_t)mx * my, 0);
    const double xu = xl + mx * dx, yu = yl + my * dy;
    for (const Region& r : regions) {
      if (t < r.tlow || t > r.thi) continue;
      int i1, i2, j1, j2;
      if (xl >= r.xhi || xu <= r.xlow) continue;
      i1 = std::max((int)std::floor((r.xlow - xl) / dx) + 1, 1);
      i2 = std::min((int)std::floor((r.xhi - xl) / dx) + 1, mx);
      if (yl >= r.yhi || yu <= r.ylow) continue;
      j1 = std::max((int)std::floor((r.ylow - yl) / dy) + 1, 1);
      j2 = std::min((int)std::floor((r.yhi - yl) / dy) + 1, my);
      for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
        minl[(i - 1) + (size_t)mx * (j - 1)] = std::max(minl[(i - 1) + (size_t)mx * (j - 1)], r.minlevel);
        maxl[(i - 1) + (size_t)mx * (j - 1)] = std::max(maxl[(i - 1) + (size_t)mx * (j - 1)], r.maxlevel);
      }
    }
    for (int j = 1; j <= my; ++j) for (int i = 1; i <= mx; ++i) {
      const int mn = minl[(i - 1) + (size_t)mx * (j - 1)], mxl = maxl[(i - 1) + (size_t)mx * (j - 1)];
      if (mn > mxl) throw std::runtime_error("flagregions2: min level > max level");
      if (mxl != 0) {
        if (level < mn) AF(i, j) = DOFLAG;
        else if (level >= mxl) AF(i, j) = DONTFLAG;
      }
    }
  }
  void flag2refine2(int mx, int my, int mbc, int mbuff, const double* q, double tolsp_, double* amrflags) {
    const int ld = mx + 2 * mbuff, mitot = mx + 2 * mbc;
    auto AF = [&](int i, int j) -> double& { return amrflags[(i + mbuff - 1) + (size_t)ld * (j + mbuff - 1)]; };
    auto Q = [&](int m, int i, int j) { return q[(m - 1) + (size_t)nvar * ((i + mbc - 1) + (size_t)mitot * (j + mbc - 1))]; };
    for (int j = 1; j <= my; ++j)
      for (int i = 1; i <= mx; ++i) {
        if (AF(i, j) != UNSET) continue;
        const int m0 = flag_component > 0 ? flag_component : 1, m1 = flag_component > 0 ? flag_component : nvar;
        for (int m = m0; m <= m1; ++m) {
          const double dqi = std::fabs(Q(m, i + 1, j) - Q(m, i - 1, j));
          const double dqj = std::fabs(Q(m, i, j + 1) - Q(m, i, j - 1));
          const double dq = std::max(0.0, std::max(dqi, dqj));
          if (dq > tolsp_) { AF(i, j) = DOFLAG; break; }
        }
      }
  }

  void flagger(int lcheck, double start_time) {
    const int mbuff = std::max(nghost, ibuff + 1);
    for (int mptr : levelgrids[lcheck]) {
      Node2& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1, nyg = g.jhi - g.jlo + 1;
      g.flags.assign((size_t)(nxg + 2 * mbuff) * (nyg + 2 * mbuff), UNSET);
    }
    for (int mptr : levelgrids[lcheck]) {
      Node2& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1, nyg = g.jhi - g.jlo + 1;
      const int mitot = nxg + 2 * nghost, mjtot = nyg + 2 * nghost;
      const double t = g.time;
      const double dx = hxposs[lcheck], dy = hyposs[lcheck];
      const double* use;
      if (start_time + possk[lcheck] != t) {
        bound(t, nghost, g.q1.data(), mitot, mjtot, mptr);
        use = g.q1.data();
      } else {
        use = g.q2.data();
      }
      flagregions2(nxg, nyg, mbuff, g.xlo, g.ylo, dx, dy, lcheck, t, g.flags.data());
      bool keep = false;
      for (double f : g.flags) if (f == UNSET) { keep = true; break; }
      if (flag_gradient && keep) flag2refine2(nxg, nyg, nghost, mbuff, use, tolsp, g.flags.data());
      keep = false;
      for (double f : g.flags) if (f == UNSET) { keep = true; break; }
      // flagger.f:93-105: locbig is a copy of the values just flagged, ghost cells included
      if (flag_richardson && keep) errest(mptr, lcheck, std::vector<double>(use, use + (size_t)nvar * mitot * mjtot), mbuff);
    }
  }

  // errest.f:4-63 for grid mptr of level lcheck: a step of 2*dt on the old values
  // coarsened by 2 (prepbigstep.f:5-64 with copysol.f and coarsen.f:4-33), a regular step
  // on `big` (prepregstep.f:5-36), then errf1.f:40-95 on component 1
  void errest(int mptr, int lcheck, std::vector<double> big, int mbuff) {
    if (naux > 0) throw std::runtime_error("Richardson estimation needs num_aux = 0 (no auxcoarsen)");
    const Node2& g = node[mptr];
    const int nx = g.ihi - g.ilo + 1, ny = g.jhi - g.jlo + 1;
    const int mitot = nx + 2 * nghost, mjtot = ny + 2 * nghost;
    const int mi2tot = nx / 2 + 2 * nghost, mj2tot = ny / 2 + 2 * nghost;
    const int ng2 = 2 * nghost, midub = nx + 4 * nghost, mjdub = ny + 4 * nghost;
    const double hx = hxposs[lcheck], hy = hyposs[lcheck];
    const double hx2 = 2.0 * hx, hy2 = 2.0 * hy;
    const double dt = possk[lcheck], dt2 = 2.0 * dt;  // `2. * dt`: the REAL literal 2. is exact
    const double tpre = g.time - dt;
    // copysol.f: the interior of the old values into an array with twice the ghost width
    std::vector<double> valdub((size_t)nvar * midub * mjdub, 0.0);
    FArr V{valdub.data(), nvar, midub, mjdub};
    const FArr Q2{const_cast<double*>(g.q2.data()), nvar, mitot, mjtot};
    for (int j = nghost + 1; j <= mjtot - nghost; ++j)
      for (int i = nghost + 1; i <= mitot - nghost; ++i)
        for (int m = 1; m <= nvar; ++m) V(m, i - nghost + ng2, j - nghost + ng2) = Q2(m, i, j);
    bound(tpre, ng2, valdub.data(), midub, mjdub, mptr);
    // coarsen.f
    std::vector<double> valbgc((size_t)nvar * mi2tot * mj2tot);
    FArr C{valbgc.data(), nvar, mi2tot, mj2tot};
    for (int j = 1; j <= mj2tot; ++j) {
      const int jf = 2 * (j - 1) + 1;
      for (int i = 1; i <= mi2tot; ++i) {
        const int iff = 2 * (i - 1) + 1;
        for (int m = 1; m <= nvar; ++m) C(m, i, j) = (((V(m, iff, jf) + V(m, iff + 1, jf)) + V(m, iff, jf + 1)) + V(m, iff + 1, jf + 1)) / 4.0;
      }
    }
    double dtnew, cflg;
    {
      const size_t nf = (size_t)nvar * mi2tot * mj2tot;
      std::vector<double> fm(nf), fp(nf), gm(nf), gp(nf);
      stepgrid(valbgc.data(), fm.data(), fp.data(), gm.data(), gp.data(), mi2tot, mj2tot, nghost, dt2, dtnew, hx2, hy2, nullptr, cflg);
    }
    {
      const size_t nf = (size_t)nvar * mitot * mjtot;
      std::vector<double> fm(nf), fp(nf), gm(nf), gp(nf);
      stepgrid(big.data(), fm.data(), fp.data(), gm.data(), gp.data(), mitot, mjtot, nghost, dt, dtnew, hx, hy, nullptr, cflg);
    }
    // errf1.f: the flag array (nx+2*mbuff wide) is indexed with the fine grid's ghost
    // width, as in the reference
    const FArr F{big.data(), nvar, mitot, mjtot};
    const int mib = nx + 2 * mbuff;
    auto RF = [&](int i, int j) -> double& { return node[mptr].flags[(size_t)(i - 1) + (size_t)mib * (j - 1)]; };
    const double order = (double)((1 << (method[2] + 1)) - 2);
    std::vector<double> rflag((size_t)mi2tot * mj2tot, UNSET);
    for (int j = nghost + 1, jf = nghost + 1; j <= mj2tot - nghost; ++j, jf += 2)
      for (int i = nghost + 1, iff = nghost + 1; i <= mi2tot - nghost; ++i, iff += 2) {
        if (RF(iff, jf) == UNSET || RF(iff + 1, jf) == UNSET || RF(iff, jf + 1) == UNSET || RF(iff + 1, jf + 1) == UNSET) {
          const double aval = (((F(1, iff, jf) + F(1, iff + 1, jf)) + F(1, iff + 1, jf + 1)) + F(1, iff, jf + 1)) / 4.0;
          const double est = std::fabs((aval - C(1, i, j)) / order);
          if (est >= tol) rflag[(size_t)(i - 1) + (size_t)mi2tot * (j - 1)] = DOFLAG;
        }
      }
    for (int j = nghost + 1, jf = nghost + 1; j <= mj2tot - nghost; ++j, jf += 2)
      for (int i = nghost + 1, iff = nghost + 1; i <= mi2tot - nghost; ++i, iff += 2)
        if (rflag[(size_t)(i - 1) + (size_t)mi2tot * (j - 1)] == DOFLAG)
          RF(iff, jf) = RF(iff + 1, jf) = RF(iff, jf + 1) = RF(iff + 1, jf + 1) = DOFLAG;
  }

  void setIndices(int ist[3], int iend[3], int jst[3], int jend[3], int ilo, int ihi, int jlo, int jhi, int ishift[3], int jshift[3], int level) {
    ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[level];
    iend[0] = -1; iend[1] = iregsz[level] - 1; iend[2] = ihi;
    jst[0] = jlo; jst[1] = 0; jst[2] = jregsz[level];
    jend[0] = -1; jend[1] = jregsz[level] - 1; jend[2] = jhi;
    if (xperdom) { ishift[0] = iregsz[level]; ishift[1] = 0; ishift[2] = -iregsz[level]; } else { ishift[0] = ishift[1] = ishift[2] = 0; }
    if (yperdom) { jshift[0] = jregsz[level]; jshift[1] = 0; jshift[2] = -jregsz[level]; } else { jshift[0] = jshift[1] = jshift[2] = 0; }
  }

  // projec2.f:51-220 ; rectflags(ilo-mbuff:ihi+mbuff, jlo-mbuff:jhi+mbuff)
  void projec2(int level, double* rf, int ilo, int ihi, int jlo, int jhi, int mbuff) {
    const int ld = ihi - ilo + 1 + 2 * mbuff;
    auto RF = [&](int i, int j) -> double& { return rf[(i - (ilo - mbuff)) + (size_t)ld * (j - (jlo - mbuff))]; };
    const int levpro = level + 2;
    for (int mkid = newstl[levpro]; mkid != 0; mkid = node[mkid].levelptr) {
      const Node2& k = node[mkid];
      int istc = k.ilo / intratx[level + 1] - 1; istc = istc / intratx[level] - 1;
      int jstc = k.jlo / intraty[level + 1] - 1; jstc = jstc / intraty[level] - 1;
      int iendc = k.ihi / intratx[level + 1] + 1; iendc = iendc / intratx[level] + 1;
      int jendc = k.jhi / intraty[level + 1] + 1; jendc = jendc / intraty[level] + 1;
      const bool borderx = (istc <= 0 || iendc >= iregsz[level] - 1);
      const bool bordery = (jstc <= 0 || jendc >= jregsz[level] - 1);
      if (!(xperdom && borderx) && !(yperdom && bordery)) {
        istc = std::max(istc, 0); jstc = std::max(jstc, 0);
        iendc = std::min(iendc, iregsz[level]); jendc = std::min(jendc, jregsz[level]);
        const int ixlo = std::max(istc, ilo - mbuff), ixhi = std::min(iendc, ihi + mbuff);
        const int jxlo = std::max(jstc, jlo - mbuff), jxhi = std::min(jendc, jhi + mbuff);
        if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
        for (int j = jxlo; j <= jxhi; ++j) for (int i = ixlo; i <= ixhi; ++i) if (RF(i, j) <= DONTFLAG) RF(i, j) = BADPRO;
        continue;
      }
      // periodic case. The reference passes undefined locals (iclo,ichi,jclo,jhci)
      // to setIndices here; the projected box (istc..iendc, jstc..jendc) is the evident intent.
      int ist[3], iend[3], jst[3], jend[3], ishift[3], jshift[3];
      setIndices(ist, iend, jst, jend, istc, iendc, jstc, jendc, ishift, jshift, level);
      for (int i = 0; i < 3; ++i) {
        int i1 = std::max(istc, ist[i]), i2 = std::min(iendc, iend[i]);
        for (int j = 0; j < 3; ++j) {
          int j1 = std::max(jstc, jst[j]), j2 = std::min(jendc, jend[j]);
          if (!(i1 <= i2 && j1 <= j2)) continue;
          const int a1 = i1 + ishift[i], a2 = i2 + ishift[i], b1 = j1 + jshift[j], b2 = j2 + jshift[j];
          const int ixlo = std::max(a1, ilo - mbuff), ixhi = std::min(a2, ihi + mbuff);
          const int jxlo = std::max(b1, jlo - mbuff), jxhi = std::min(b2, jhi + mbuff);
          if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
          for (int jx = jxlo; jx <= jxhi; ++jx) for (int ix = ixlo; ix <= ixhi; ++ix) if (RF(ix, jx) <= DONTFLAG) RF(ix, jx) = BADPRO;
        }
      }
    }
  }

  void shiftset2(double* rf, int ilo, int ihi, int jlo, int jhi, int mbuff) {
    const int ld = ihi - ilo + 1 + 2 * mbuff, ldj = jhi - jlo + 1 + 2 * mbuff;
    auto RF = [&](int i, int j) -> double& { return rf[(i - (ilo - mbuff)) + (size_t)ld * (j - (jlo - mbuff))]; };
    std::vector<double> copy((size_t)ld * ldj, 0.0);
    auto CP = [&](int i, int j) -> double& { return copy[(i - (ilo - mbuff)) + (size_t)ld * (j - (jlo - mbuff))]; };
    for (int j = jlo; j <= jhi; ++j)
      for (int i = ilo; i <= ihi; ++i) {
        const double r = RF(i, j);
        if (r > 0) for (int k = j - ibuff; k <= j + ibuff; ++k) for (int m = i - ibuff; m <= i + ibuff; ++m) CP(m, k) = r;
      }
    for (size_t k = 0; k < copy.size(); ++k) rf[k] = copy[k];
  }

  // integer*1 helpers for setdomflags: arrays indexed (ilo-mbuff:ihi+mbuff, jlo-mbuff:jhi+mbuff) over raw storage
  struct I1 {
    signed char* p; int ilo, ihi, jlo, jhi, mbuff;
    signed char& operator()(int i, int j) const {
      return p[(i - (ilo - mbuff)) + (size_t)(ihi - ilo + 1 + 2 * mbuff) * (j - (jlo - mbuff))];
    }
  };
  void setPhysBndryFlags(I1 f, int level) {
    const int ilo = f.ilo, ihi = f.ihi, jlo = f.jlo, jhi = f.jhi, mb = f.mbuff;
    if (ilo - mb < 0 && !xperdom) for (int j = jlo - mb; j <= jhi + mb; ++j) for (int i = ilo - mb; i <= -1; ++i) f(i, j) = 1;
    if (ihi + mb >= iregsz[level] && !xperdom) for (int j = jlo - mb; j <= jhi + mb; ++j) for (int i = iregsz[level]; i <= ihi + mb; ++i) f(i, j) = 1;
    if (jlo - mb < 0 && !yperdom) for (int j = jlo - mb; j <= -1; ++j) for (int i = ilo - mb; i <= ihi + mb; ++i) f(i, j) = 1;
    if (jhi + mb >= jregsz[level] && !yperdom) for (int j = jregsz[level]; j <= jhi + mb; ++j) for (int i = ilo - mb; i <= ihi + mb; ++i) f(i, j) = 1;
  }
  void griddomshrink(I1 in, I1 out, int level) {
    const int ilo = in.ilo, ihi = in.ihi, jlo = in.jlo, jhi = in.jhi, mb = in.mbuff;
    for (int j = jlo - mb + 1; j <= jhi + mb - 1; ++j) {
      for (int i = ilo - mb + 1; i <= ihi + mb - 1; ++i) {
        out(i, j) = in(i, j);
        if (in(i, j) <= 0 || in(i + 1, j) <= 0 || in(i - 1, j) <= 0 || in(i + 1, j + 1) <= 0 || in(i - 1, j + 1) <= 0 ||
            in(i, j - 1) <= 0 || in(i, j + 1) <= 0 || in(i + 1, j - 1) <= 0 || in(i - 1, j - 1) <= 0)
          out(i, j) = 0;
      }
      out(ilo - mb, j) = 0; out(ihi + mb, j) = 0;
    }
    for (int i = ilo - mb; i <= ihi + mb; ++i) { out(i, jlo - mb) = 0; out(i, jhi + mb) = 0; }
    setPhysBndryFlags(out, level);
  }
  void griddomup(I1 c, I1 f, int lev) {
    const int rx = intratx[lev], ry = intraty[lev], mb = c.mbuff;
    for (int j = f.jlo - mb; j <= f.jhi + mb; ++j) for (int i = f.ilo - mb; i <= f.ihi + mb; ++i) f(i, j) = 0;
    for (int j = c.jlo; j <= c.jhi; ++j)
      for (int i = c.ilo; i <= c.ihi; ++i) {
        const int ifine = i * rx - 1, jfine = j * ry - 1;
        for (int mj = 1; mj <= ry; ++mj)
          for (int mi = 1; mi <= rx; ++mi) {
            int iset = std::min(ifine + mi, f.ihi + mb), jset = std::min(jfine + mj, f.jhi + mb);
            iset = std::max(iset, f.ilo - mb); jset = std::max(jset, f.jlo - mb);
            f(iset, jset) = c(i, j);
          }
      }
    for (int j = f.jlo - mb; j <= f.jhi + mb; ++j) {
      for (int i = f.ihi + 1; i <= f.ihi + mb; ++i) f(i, j) = c(i / rx, j / ry);
      for (int i = f.ilo - mb; i <= f.ilo - 1; ++i) f(i, j) = c(i / rx, j / ry);
    }
    for (int i = f.ilo; i <= f.ihi; ++i) {
      for (int j = f.jlo - mb; j <= f.jlo - 1; ++j) f(i, j) = c(i / rx, j / ry);
      for (int j = f.jhi + 1; j <= f.jhi + mb; ++j) f(i, j) = c(i / rx, j / ry);
    }
  }
  void setdomflags(int mptr, int ilo, int ihi, int jlo, int jhi, int mbuff, int lbase, int lcheck, int mibuff, int mjbuff) {
    Node2& g = node[mptr];
    g.dom1.assign((size_t)mibuff * mjbuff, 0);
    g.dom2.assign((size_t)mibuff * mjbuff, 0);
    std::vector<signed char> icopy((size_t)mibuff * mjbuff, 0);
    int igst[12], igend[12], jgst[12], jgend[12];
    igst[lcheck] = ilo; igend[lcheck] = ihi; jgst[lcheck] = jlo; jgend[lcheck] = jhi;
    for (int lc = lcheck - 1; lc >= lbase; --lc) {
      int ilc = (int)std::floor((double)igst[lc + 1] / intratx[lc]);
      int jlc = (int)std::floor((double)jgst[lc + 1] / intraty[lc]);
      int ihc = (int)std::ceil((double)igend[lc + 1] / intratx[lc]) - 1;
      int jhc = (int)std::ceil((double)jgend[lc + 1] / intraty[lc]) - 1;
      if (ihc * intratx[lc] < igend[lc + 1]) ihc = ihc + 1;
      if (jhc * intraty[lc] < jgend[lc + 1]) jhc = jhc + 1;
      igend[lc] = ihc; jgend[lc] = jhc; igst[lc] = ilc; jgst[lc] = jlc;
    }
    int ilc = igst[lbase], ihc = igend[lbase], jlc = jgst[lbase], jhc = jgend[lbase];
    I1 base{g.dom1.data(), ilc, ihc, jlc, jhc, mbuff};
    for (int mb = lstart[lbase]; mb != 0; mb = node[mb].levelptr) {
      const int iblo = node[mb].ilo, ibhi = node[mb].ihi, jblo = node[mb].jlo, jbhi = node[mb].jhi;
      const bool borderx = (ilc <= 0 || ihc >= iregsz[lbase] - 1);
      const bool bordery = (jlc <= 0 || jhc >= jregsz[lbase] - 1);
      if ((xperdom && borderx) || (yperdom && bordery)) {
        int ist[3], iend[3], jst[3], jend[3], ishift[3], jshift[3];
        setIndices(ist, iend, jst, jend, ilc - mbuff, ihc + mbuff, jlc - mbuff, jhc + mbuff, ishift, jshift, lbase);
        for (int i = 0; i < 3; ++i) {
          const int i1 = std::max(ilc - mbuff, ist[i]), i2 = std::min(ihc + mbuff, iend[i]);
          for (int j = 0; j < 3; ++j) {
            const int j1 = std::max(jlc - mbuff, jst[j]), j2 = std::min(jhc + mbuff, jend[j]);
            if (!(i1 <= i2 && j1 <= j2)) continue;
            const int ixlo = std::max(iblo, i1 + ishift[i]), ixhi = std::min(ibhi, i2 + ishift[i]);
            const int jxlo = std::max(jblo, j1 + jshift[j]), jxhi = std::min(jbhi, j2 + jshift[j]);
            if (ixlo > ixhi || jxlo > jxhi) continue;
            for (int jj = jxlo - jshift[j]; jj <= jxhi - jshift[j]; ++jj)
              for (int ii = ixlo - ishift[i]; ii <= ixhi - ishift[i]; ++ii) base(ii, jj) = 1;
          }
        }
      } else {
        const int ixlo = std::max(iblo, ilc - mbuff), ixhi = std::min(ibhi, ihc + mbuff);
        const int jxlo = std::max(jblo, jlc - mbuff), jxhi = std::min(jbhi, jhc + mbuff);
        if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
        for (int jj = jxlo; jj <= jxhi; ++jj) for (int ii = ixlo; ii <= ixhi; ++ii) base(ii, jj) = 1;
      }
    }
    setPhysBndryFlags(base, lbase);
    I1 cp{icopy.data(), ilc, ihc, jlc, jhc, mbuff};
    for (int j = jlc - mbuff; j <= jhc + mbuff; ++j) for (int i = ilc - mbuff; i <= ihc + mbuff; ++i) cp(i, j) = base(i, j);
    I1 d2{g.dom2.data(), ilc, ihc, jlc, jhc, mbuff};
    griddomshrink(cp, d2, lbase);
    for (int lev = lbase + 1; lev <= lcheck; ++lev) {
      const int ilf = igst[lev], ihf = igend[lev], jlf = jgst[lev], jhf = jgend[lev];
      I1 c2{g.dom2.data(), ilc, ihc, jlc, jhc, mbuff};
      I1 fcp{icopy.data(), ilf, ihf, jlf, jhf, mbuff};
      griddomup(c2, fcp, lev - 1);
      I1 fd2{g.dom2.data(), ilf, ihf, jlf, jhf, mbuff};
      griddomshrink(fcp, fd2, lev);
      ilc = ilf; ihc = ihf; jlc = jlf; jhc = jhf;
    }
  }

  void bufnst2(int& numbad, int lcheck, int lbase) {
    numbad = 0;
    for (int mptr : levelgrids[lcheck]) {
      Node2& g = node[mptr];
      const int ilo = g.ilo, ihi = g.ihi, jlo = g.jlo, jhi = g.jhi;
      const int mbuff = std::max(nghost, ibuff + 1);
      const int mibuff = ihi - ilo + 1 + 2 * mbuff, mjbuff = jhi - jlo + 1 + 2 * mbuff;
      if (lcheck + 2 <= mxnest) projec2(lcheck, g.flags.data(), ilo, ihi, jlo, jhi, mbuff);
      shiftset2(g.flags.data(), ilo, ihi, jlo, jhi, mbuff);
      int nf = 0;
      for (double f : g.flags) if (f > DONTFLAG) ++nf;
      g.numflags = nf;
      numbad += nf;
      setdomflags(mptr, ilo, ihi, jlo, jhi, mbuff, lbase, lcheck, mibuff, mjbuff);
    }
  }

  void drivesort(int npts, std::vector<double>& badpts, int level, int& nunique, int mbuff) {
    const int isize = iregsz[level];
    std::vector<long long> key(npts + 1);
    std::vector<int> ix(npts + 1);
    for (int k = 1; k <= npts; ++k) {
      const int i = (int)(badpts[2 * (k - 1)] - 0.5), j = (int)(badpts[2 * (k - 1) + 1] - 0.5);
      key[k] = (long long)(i + mbuff) + (long long)(isize + 2 * mbuff) * (j + mbuff);
    }
    qsorti(ix, npts, key);
    int k = 1, index = 0;
    while (k <= npts) {
      const long long ie = key[ix[k]];
      ++index;
      badpts[2 * (index - 1) + 1] = (double)(ie / (isize + 2 * mbuff)) + 0.5 - mbuff;
      badpts[2 * (index - 1)] = (double)(ie % (isize + 2 * mbuff)) + 0.5 - mbuff;
      ++k;
      while (k <= npts && key[ix[k]] == key[ix[k - 1]]) ++k;
    }
    nunique = index;
  }

  void colate2(std::vector<double>& badpts, int lcheck, int& nunique) {
    const int mbuff = std::max(nghost, ibuff + 1);
    int index = 0;
    for (int mptr = lstart[lcheck]; mptr != 0; mptr = node[mptr].levelptr) {
      Node2& g = node[mptr];
      const int ilo = g.ilo, ihi = g.ihi, jlo = g.jlo, jhi = g.jhi;
      const int mibuff = ihi - ilo + 1 + 2 * mbuff;
      auto RF = [&](int i, int j) -> double& { return g.flags[(i - (ilo - mbuff)) + (size_t)mibuff * (j - (jlo - mbuff))]; };
      if (g.numflags != 0) {
        int jmin = jlo - mbuff, jmax = jhi + mbuff, imin = ilo - mbuff, imax = ihi + mbuff;
        if (!xperdom) { imin = std::max(imin, 0); imax = std::min(ihi + mbuff, iregsz[lcheck] - 1); }
        if (!yperdom) { jmin = std::max(jmin, 0); jmax = std::min(jhi + mbuff, jregsz[lcheck] - 1); }
        I1 d2{g.dom2.data(), ilo, ihi, jlo, jhi, mbuff};
        for (int j = jmin; j <= jmax; ++j) for (int i = imin; i <= imax; ++i) {
          if (RF(i, j) <= DONTFLAG) continue;
          if (d2(i, j) != 1) RF(i, j) = DONTFLAG;
        }
        for (int j = jmin; j <= jmax; ++j) for (int i = imin; i <= imax; ++i) {
          if (RF(i, j) < 0) continue;
          if (RF(i, j) <= DONTFLAG) continue;
          ++index;
          int iw = i, jw = j;
          if (xperdom) { if (i < 0) iw = i + iregsz[lcheck]; if (i >= iregsz[lcheck]) iw = i - iregsz[lcheck]; }
          if (yperdom) { if (j < 0) jw = j + jregsz[lcheck]; if (j >= jregsz[lcheck]) jw = j - jregsz[lcheck]; }
          badpts.push_back((double)iw + 0.5);
          badpts.push_back((double)jw + 0.5);
        }
      }
      g.flags.clear(); g.dom1.clear(); g.dom2.clear();
    }
    const int npts = index;
    drivesort(npts, badpts, lcheck, nunique, mbuff);
    badpts.resize(2 * (size_t)nunique);
    if (std::getenv("AMRB_DEBUG")) {
      std::fprintf(stderr, "FLAGS lcheck=%d npts=%d:", lcheck, nunique);
      for (int k = 0; k < nunique && k < 12; ++k) std::fprintf(stderr, " (%d,%d)", (int)(badpts[2 * k] - 0.5), (int)(badpts[2 * k + 1] - 0.5));
      std::fprintf(stderr, "\n");
    }
  }

  // ================================================================ clustering
  void moment(int rect[4], const double* badpts, int npt, double& usage) {
    const double rn = (double)npt;
    double emx1 = badpts[0], emn1 = emx1, emx2 = badpts[1], emn2 = emx2;
    for (int k = 0; k < npt; ++k) {
      const double a = badpts[2 * k], b = badpts[2 * k + 1];
      if (a > emx1) emx1 = a;
      if (a < emn1) emn1 = a;
      if (b > emx2) emx2 = b;
      if (b < emn2) emn2 = b;
    }
    rect[0] = (int)std::nearbyint(emn1 - 0.5); rect[2] = (int)std::nearbyint(emn2 - 0.5);
    rect[1] = (int)std::nearbyint(emx1 - 0.5); rect[3] = (int)std::nearbyint(emx2 - 0.5);
    const int s1 = rect[1] - rect[0] + 1, s2 = rect[3] - rect[2] + 1;
    usage = rn / (double)(s1 * s2);
  }
  void signs(const double* badpts, int ist, int iend, std::vector<int>& iscr, std::vector<int>& jscr, int idim, int jdim,
             int& ilo, int& ihi, int& jlo, int& jhi) {
    ilo = 1; ihi = idim; jlo = 1; jhi = jdim;
    std::fill(iscr.begin(), iscr.end(), 0); std::fill(jscr.begin(), jscr.end(), 0);
    for (int ipt = ist; ipt <= iend; ++ipt) {
      const int il = (int)(badpts[2 * (ipt - 1)] + 1.1), jl = (int)(badpts[2 * (ipt - 1) + 1] + 1.1);
      iscr[il] += 1; jscr[jl] += 1;
    }
    for (int p = 1; p <= idim; ++p) if (iscr[p] != 0) { ilo = p; break; }
    for (int p = 1; p <= idim; ++p) if (iscr[idim + 1 - p] != 0) { ihi = idim + 1 - p; break; }
    for (int p = 1; p <= jdim; ++p) if (jscr[p] != 0) { jlo = p; break; }
    for (int p = 1; p <= jdim; ++p) if (jscr[jdim + 1 - p] != 0) { jhi = jdim + 1 - p; break; }
  }
  void findcut(std::vector<int>& iscr, std::vector<int>& jscr, int& index, int& iside, int ilo, int ihi, int jlo, int jhi) {
    const int ithres = 2, minoff = 2;
    for (int i = ilo; i <= ihi; ++i) if (iscr[i] == 0) { index = i; iside = HORIZONTAL; return; }
    for (int j = jlo; j <= jhi; ++j) if (jscr[j] == 0) { index = j; iside = VERTICAL; return; }
    int ipre = iscr[ilo];
    for (int i = ilo + 1; i <= ihi - 1; ++i) { const int icur = iscr[i]; iscr[i] = iscr[i + 1] - 2 * icur + ipre; ipre = icur; }
    int locmaxi = 0, indexi = 0;
    const int imid = (ilo + ihi) / 2;
    for (int i = ilo + minoff; i <= ihi - minoff + 1; ++i) {
      const int t1 = iscr[i - 1], t2 = iscr[i];
      const int locdif = std::abs(t1 - t2);
      if (t1 * t2 < 0) {
        if (locdif > locmaxi) { locmaxi = locdif; indexi = i; }
        else if (locdif == locmaxi) { if (std::abs(i - imid) < std::abs(indexi - imid)) indexi = i; }
      }
    }
    int jpre = jscr[jlo];
    for (int j = jlo + 1; j <= jhi - 1; ++j) { const int jcur = jscr[j]; jscr[j] = jscr[j + 1] - 2 * jcur + jpre; jpre = jcur; }
    int locmaxj = 0, indexj = 0;
    const int jmid = (jlo + jhi) / 2;
    for (int j = jlo + minoff; j <= jhi - minoff + 1; ++j) {
      const int t1 = jscr[j - 1], t2 = jscr[j];
      const int locdif = std::abs(t1 - t2);
      if (t1 * t2 < 0) {
        if (locdif > locmaxj) { locmaxj = locdif; indexj = j; }
        else if (locdif == locmaxj) { if (std::abs(j - jmid) < std::abs(indexj - jmid)) indexj = j; }
      }
    }
    int locmax;
    if (locmaxi > locmaxj) { index = indexi; iside = HORIZONTAL; locmax = locmaxi; }
    else if (locmaxi < locmaxj) { index = indexj; iside = VERTICAL; locmax = locmaxj; }
    else if (std::abs(indexi - imid) < std::abs(indexj - jmid)) { index = indexi; iside = HORIZONTAL; locmax = locmaxi; }
    else { index = indexj; iside = VERTICAL; locmax = locmaxj; }
    if (locmax < ithres) index = 0;
  }
  void smartbis(std::vector<double>& badpts, int npts, double cutoff, std::vector<int>& numptc, int& nclust, int idim, int jdim) {
    nclust = 1;
    numptc.assign(2, 0); numptc[1] = npts;
    int icl = 1, ist = 1, iend = numptc[icl];
    std::vector<int> iscr(idim + 2), jscr(jdim + 2);
    int rect[4];
    while (true) {
      double usenew;
      moment(rect, badpts.data() + 2 * (ist - 1), numptc[icl], usenew);
      bool advance = false;
      if (usenew >= cutoff) advance = true;
      else {
        int ilo, ihi, jlo, jhi, index, iside;
        signs(badpts.data(), ist, iend, iscr, jscr, idim, jdim, ilo, ihi, jlo, jhi);
        findcut(iscr, jscr, index, iside, ilo, ihi, jlo, jhi);
        if (index == 0) advance = true;
        else {
          double fmid; int idir;
          if (iside == VERTICAL) { fmid = index - 0.5; idir = 2; } else { fmid = index - 0.5; idir = 1; }
          int itop = ist - 1, ibot = iend + 1, i = ist;
          auto BP = [&](int d, int k) -> double& { return badpts[2 * (k - 1) + (d - 1)]; };
          while (true) {
            if (BP(idir, i) < fmid) {
              ibot = ibot - 1;
              std::swap(BP(1, ibot), BP(1, i));
              std::swap(BP(2, ibot), BP(2, i));
              if (itop + 1 < ibot) continue;
              break;
            } else {
              itop = itop + 1;
              if (itop + 1 >= ibot) break;
              i = i + 1;
            }
          }
          numptc[icl] = itop - ist + 1;
          const int ibump = icl + 1;
          numptc.resize(nclust + 2, 0);
          for (int ico = ibump; ico <= nclust; ++ico) { const int nmove = nclust - ico + ibump; numptc[nmove + 1] = numptc[nmove]; }
          numptc[ibump] = iend - ibot + 1;
          nclust = nclust + 1;
          iend = itop;
          continue;
        }
      }
      if (advance) {
        icl = icl + 1;
        if (icl > nclust) break;
        ist = iend + 1;
        iend = ist + numptc[icl] - 1;
      }
    }
  }

  bool baseCheck(int mnew, int lbase, int ilo, int ihi, int jlo, int jhi, int thisBuff) {
    const int levnew = node[mnew].level;
    const bool borderx = (ilo == 0 || ihi == iregsz[levnew] - 1);
    const bool bordery = (jlo == 0 || jhi == jregsz[levnew] - 1);
    int iclo = ilo, ichi = ihi, jclo = jlo, jchi = jhi;
    for (int lev = levnew - 1; lev >= lbase; --lev) {
      iclo = iclo / intratx[lev]; ichi = ichi / intratx[lev]; jclo = jclo / intraty[lev]; jchi = jchi / intraty[lev];
      iclo -= 1; ichi += 1; jclo -= 1; jchi += 1;
    }
    if (!(xperdom && borderx) && !(yperdom && bordery)) {
      iclo = std::max(iclo, 0); jclo = std::max(jclo, 0);
      ichi = std::min(ichi, iregsz[lbase] - 1); jchi = std::min(jchi, jregsz[lbase] - 1);
    }
    const int leni = ichi - iclo + 1, lenj = jchi - jclo + 1;
    std::vector<double> m((size_t)leni * lenj, 0.0);
    auto M = [&](int i, int j) -> double& { return m[(i - iclo) + (size_t)leni * (j - jclo)]; };
    if (ilo == 0 && !xperdom) for (int j = jclo; j <= jchi; ++j) { M(iclo, j) = 1.; M(iclo + 1, j) = 1.; }
    if (ihi == iregsz[levnew] - 1 && !xperdom) for (int j = jclo; j <= jchi; ++j) { M(ichi, j) = 1.; M(ichi - 1, j) = 1.; }
    if (jlo == 0 && !yperdom) for (int i = iclo; i <= ichi; ++i) { M(i, jclo) = 1.; M(i, jclo + 1) = 1.; }
    if (jhi == jregsz[levnew] - 1 && !yperdom) for (int i = iclo; i <= ichi; ++i) { M(i, jchi) = 1.; M(i, jchi - 1) = 1.; }
    for (int mptr = lstart[lbase]; mptr != 0; mptr = node[mptr].levelptr) {
      const int iblo = node[mptr].ilo - thisBuff, ibhi = node[mptr].ihi + thisBuff;
      const int jblo = node[mptr].jlo - thisBuff, jbhi = node[mptr].jhi + thisBuff;
      if (!(xperdom && borderx) && !(yperdom && bordery)) {
        const int ixlo = std::max(iclo, iblo), ixhi = std::min(ichi, ibhi), jxlo = std::max(jclo, jblo), jxhi = std::min(jchi, jbhi);
        if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
        for (int jx = jxlo; jx <= jxhi; ++jx) for (int ix = ixlo; ix <= ixhi; ++ix) M(ix, jx) = 1.;
        continue;
      }
      int ist[3], iend[3], jst[3], jend[3], ishift[3], jshift[3];
      setIndices(ist, iend, jst, jend, iclo, ichi, jclo, jchi, ishift, jshift, lbase);
      for (int i = 0; i < 3; ++i) {
        const int i1 = std::max(iclo, ist[i]), i2 = std::min(ichi, iend[i]);
        for (int j = 0; j < 3; ++j) {
          const int j1 = std::max(jclo, jst[j]), j2 = std::min(jchi, jend[j]);
          if (!(i1 <= i2 && j1 <= j2)) continue;
          const int ixlo = std::max(i1 + ishift[i], iblo), ixhi = std::min(i2 + ishift[i], ibhi);
          const int jxlo = std::max(j1 + jshift[j], jblo), jxhi = std::min(j2 + jshift[j], jbhi);
          if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
          for (int jx = jxlo; jx <= jxhi; ++jx) for (int ix = ixlo; ix <= ixhi; ++ix) M(ix - ishift[i], jx - jshift[j]) = 1.;
        }
      }
    }
    for (int j = jclo; j <= jchi; ++j) for (int i = iclo; i <= ichi; ++i) if (M(i, j) == 0) return false;
    return true;
  }

  bool nestck2(int mnew, int lbase, double* badpts, int npts, std::vector<int>& numptc, int icl, int& nclust) {
    const int levnew = node[mnew].level;
    const int lratiox = intratx[levnew - 1], lratioy = intraty[levnew - 1];
    bool isNested1, isNested2;
    if (lbase == 1) isNested1 = true;
    else isNested1 = baseCheck(mnew, lbase, node[mnew].ilo, node[mnew].ihi, node[mnew].jlo, node[mnew].jhi, 0);
    const int levToCheck = levnew - 2;
    if (levToCheck <= 1) isNested2 = true;
    else if (levToCheck <= lbase) isNested2 = isNested1;
    else {
      const int mbuff = std::max(nghost, ibuff + 1);
      isNested2 = baseCheck(mnew, levToCheck, node[mnew].ilo, node[mnew].ihi, node[mnew].jlo, node[mnew].jhi, mbuff);
    }
    if (isNested1 && isNested2) return true;
    if (npts <= 1) throw std::runtime_error("nestck2: cannot nest a single point");
    double rmid; int idir;
    if (node[mnew].xhi - node[mnew].xlo > node[mnew].yhi - node[mnew].ylo) {
      rmid = (node[mnew].ihi + node[mnew].ilo + 1) / 2.; rmid = rmid / lratiox; idir = 1;
    } else {
      rmid = (node[mnew].jhi + node[mnew].jlo + 1) / 2.; rmid = rmid / lratioy; idir = 2;
    }
    int ipt = 1, ntop = npts;
    auto BP = [&](int d, int k) -> double& { return badpts[2 * (k - 1) + (d - 1)]; };
    while (true) {
      if (BP(idir, ipt) < rmid) {
        ipt = ipt + 1;
        if (ipt <= ntop) continue;
        break;
      }
      std::swap(BP(1, ipt), BP(1, ntop));
      std::swap(BP(2, ipt), BP(2, ntop));
      ntop = ntop - 1;
      if (ipt <= ntop) continue;
      break;
    }
    numptc.resize(nclust + 2, 0);
    numptc[icl] = npts - ntop;
    for (int i = icl; i <= nclust; ++i) { const int nmove = nclust + icl - i; numptc[nmove + 1] = numptc[nmove]; }
    numptc[icl] = ntop;
    nclust = nclust + 1;
    return false;
  }

  void grdfit(int lbase, int lcheck, double t, double start_time) {
    std::vector<double> badpts;
    // flglvl2.f
    flagger(lcheck, start_time);
    int numbad = 0;
    bufnst2(numbad, lcheck, lbase);
    int npts = 0;
    if (numbad > 0) colate2(badpts, lcheck, npts);
    else {
      for (int mptr = lstart[lcheck]; mptr != 0; mptr = node[mptr].levelptr) { node[mptr].flags.clear(); node[mptr].dom1.clear(); node[mptr].dom2.clear(); }
    }
    if (npts == 0) return;
    const int levnew = lcheck + 1;
    const double hxfine = hxposs[levnew], hyfine = hyposs[levnew];
    std::vector<int> numptc;
    int nclust = 0;
    smartbis(badpts, npts, cut, numptc, nclust, iregsz[lcheck], jregsz[lcheck]);
    int ibase = 0, icl = 1, prv = 0;
    while (icl <= nclust) {
      const int mnew = nodget();
      while (true) {
        int rect[4]; double usage;
        moment(rect, badpts.data() + 2 * ibase, numptc[icl], usage);
        Node2& n = node[mnew];
        n.ilo = rect[0] * intratx[lcheck]; n.jlo = rect[2] * intraty[lcheck];
        n.ihi = (rect[1] + 1) * intratx[lcheck] - 1; n.jhi = (rect[3] + 1) * intraty[lcheck] - 1;
        n.xlo = n.ilo * hxfine + xlower; n.ylo = n.jlo * hyfine + ylower;
        n.xhi = (n.ihi + 1) * hxfine + xlower; n.yhi = (n.jhi + 1) * hyfine + ylower;
        n.level = levnew; n.time = t;
        if (nestck2(mnew, lbase, badpts.data() + 2 * ibase, numptc[icl], numptc, icl, nclust)) break;
      }
      if (newstl[levnew] == 0) newstl[levnew] = mnew;
      else node[prv].levelptr = mnew;
      prv = mnew;
      ibase = ibase + numptc[icl];
      icl = icl + 1;
    }
    birect(newstl[levnew]);
  }

  // filval.f90:3-214 (naux = 0 branch)
  void filval(double* valp, int mitot, int mjtot, double dx, double dy, int level, double t, int mic, int mjc, double xleft,
              double xright, double ybot, double ytop, int ilo, int ihi, int jlo, int jhi, double* auxp) {
    (void)t;
    const int rx = intratx[level - 1], ry = intraty[level - 1];
    const double dxc = dx * rx, dyc = dy * ry;
    const double xl = xleft - dxc, xr = xright + dxc, yb = ybot - dyc, yt = ytop + dyc;
    const int iclo = ilo / rx - 1, jclo = jlo / ry - 1, ichi = (ihi + 1) / rx - 1 + 1, jchi = (jhi + 1) / ry - 1 + 1;
    const bool sxf = (ilo < 0) || (ihi >= iregsz[level]), syf = (jlo < 0) || (jhi >= jregsz[level]);
    const bool sxc = (iclo < 0) || (ichi >= iregsz[level - 1]), syc = (jclo < 0) || (jchi >= jregsz[level - 1]);
    std::vector<double> valc((size_t)nvar * mic * mjc, 0.0), auxc((size_t)naux * mic * mjc, 0.0);
    FArr val{valp, nvar, mitot, mjtot}, VC{valc.data(), nvar, mic, mjc}, AUX{auxp, naux, mitot, mjtot}, AUXC{auxc.data(), naux, mic, mjc};
    if (naux == 0) {
      if ((xperdom && sxc) || (yperdom && syc) || spheredom) preintcopy(valc.data(), mic, mjc, iclo, ichi, jclo, jchi, level - 1);
      else intcopy(valc.data(), mic, mjc, iclo, ichi, jclo, jchi, level - 1, 1, 1);
    } else {
      // filval.f90:75-96: q and aux of the coarse cells, then setaux on the coarse patch
      for (int j = 1; j <= mjc; ++j) for (int i = 1; i <= mic; ++i) AUXC(1, i, j) = NEEDS_TO_BE_SET;
      if ((xperdom && sxc) || (yperdom && syc) || spheredom) preintcopy(valc.data(), mic, mjc, iclo, ichi, jclo, jchi, level - 1, auxc.data());
      else icall(valc.data(), mic, mjc, iclo, ichi, jclo, jchi, level - 1, 1, 1, auxc.data());
      setaux(0, mic, mjc, xl, yb, dxc, dyc, auxc.data());
    }
    bc2amr(valc.data(), mic, mjc, dxc, dyc, xl, xr, yb, yt);
    std::vector<double> setflags((size_t)mitot * mjtot);
    if (naux > 0) {
      // filval.f90:112-130: copy q and aux from the old grids of the level; the first aux
      // component marks the cells still to interpolate; then setaux on the new grid
      for (int j = 1; j <= mjtot; ++j) for (int i = 1; i <= mitot; ++i) AUX(1, i, j) = NEEDS_TO_BE_SET;
      if ((xperdom && sxf) || (yperdom && syf) || spheredom)
        preintcopy(valp, mitot, mjtot, ilo - nghost, ihi + nghost, jlo - nghost, jhi + nghost, level, auxp);
      else icall(valp, mitot, mjtot, ilo - nghost, ihi + nghost, jlo - nghost, jhi + nghost, level, 1, 1, auxp);
      for (int j = 1; j <= mjtot; ++j) for (int i = 1; i <= mitot; ++i) setflags[(i - 1) + (size_t)mitot * (j - 1)] = AUX(1, i, j);
      setaux(nghost, mitot - 2 * nghost, mjtot - 2 * nghost, xleft, ybot, dx, dy, auxp);
    } else {
      for (int j = 1; j <= mjtot; ++j) for (int i = 1; i <= mitot; ++i) val(1, i, j) = NEEDS_TO_BE_SET;
      if ((xperdom && sxf) || (yperdom && syf) || spheredom) preintcopy(valp, mitot, mjtot, ilo - nghost, ihi + nghost, jlo - nghost, jhi + nghost, level);
      else intcopy(valp, mitot, mjtot, ilo - nghost, ihi + nghost, jlo - nghost, jhi + nghost, level, 1, 1);
      for (int j = 1; j <= mjtot; ++j) for (int i = 1; i <= mitot; ++i) setflags[(i - 1) + (size_t)mitot * (j - 1)] = val(1, i, j);
    }
    for (int j = 2; j <= mjc - 1; ++j)
      for (int i = 2; i <= mic - 1; ++i)
        for (int iv = 1; iv <= nvar; ++iv) {
          double s1p = VC(iv, i + 1, j) - VC(iv, i, j), s1m = VC(iv, i, j) - VC(iv, i - 1, j);
          double slopex = std::min(std::fabs(s1p), std::fabs(s1m)) * dsign(1.0, VC(iv, i + 1, j) - VC(iv, i - 1, j));
          if (s1m * s1p <= 0.0) slopex = 0.0;
          s1p = VC(iv, i, j + 1) - VC(iv, i, j); s1m = VC(iv, i, j) - VC(iv, i, j - 1);
          double slopey = std::min(std::fabs(s1p), std::fabs(s1m)) * dsign(1.0, VC(iv, i, j + 1) - VC(iv, i, j - 1));
          if (s1m * s1p <= 0.0) slopey = 0.0;
          for (int jco = 1; jco <= ry; ++jco) {
            const double yoff = ((double)jco - 0.5) / ry - 0.5;
            const int jfine = (j - 2) * ry + nghost + jco;
            for (int ico = 1; ico <= rx; ++ico) {
              const double xoff = ((double)ico - 0.5) / rx - 0.5;
              const int ifine = (i - 2) * rx + nghost + ico;
              if (setflags[(ifine - 1) + (size_t)mitot * (jfine - 1)] == NEEDS_TO_BE_SET)
                val(iv, ifine, jfine) = VC(iv, i, j) + xoff * slopex + yoff * slopey;
            }
          }
        }
    // fixcapaq.f:4-62: conserve kappa*q, not q, over each coarse cell, adjusting only the
    // interpolated fine cells
    if (mcapa != 0)
      for (int ic = 2; ic <= mic - 1; ++ic)
        for (int jc = 2; jc <= mjc - 1; ++jc)
          for (int iv = 1; iv <= nvar; ++iv) {
            double capaqfine = 0.0;
            for (int ico = 1; ico <= rx; ++ico) {
              const int ifine = (ic - 2) * rx + nghost + ico;
              for (int jco = 1; jco <= ry; ++jco) {
                const int jfine = (jc - 2) * ry + nghost + jco;
                capaqfine = capaqfine + AUX(mcapa, ifine, jfine) * val(iv, ifine, jfine);
              }
            }
            const double dcapaq = AUXC(mcapa, ic, jc) * VC(iv, ic, jc) - capaqfine / (double)(rx * ry);
            for (int ico = 1; ico <= rx; ++ico) {
              const int ifine = (ic - 2) * rx + nghost + ico;
              for (int jco = 1; jco <= ry; ++jco) {
                const int jfine = (jc - 2) * ry + nghost + jco;
                if (setflags[(ifine - 1) + (size_t)mitot * (jfine - 1)] == NEEDS_TO_BE_SET)
                  val(iv, ifine, jfine) = val(iv, ifine, jfine) + dcapaq / AUX(mcapa, ifine, jfine);
              }
            }
          }
  }

  void gfixup(int lbase, int lfnew) {
    putsp(lbase, lbase);
    for (int level = lbase + 1; level <= lfine; ++level) {
      putsp(lbase, level);
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].q2.clear(); node[m].has_q2 = false; }
    }
    for (int lcheck = lbase + 1; lcheck <= mxnest; ++lcheck) {
      const double hx = hxposs[lcheck], hy = hyposs[lcheck];
      std::vector<int> lnew;
      for (int m = newstl[lcheck]; m != 0; m = node[m].levelptr) lnew.push_back(m);
      for (int m : lnew) {
        node[m].q1.assign((size_t)nvar * mitot_of(m) * mjtot_of(m), 0.0);
        node[m].aux.assign((size_t)naux * mitot_of(m) * mjtot_of(m), 0.0);
      }
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
      for (int k = 0; k < (int)lnew.size(); ++k) {
        const int m = lnew[k];
        Node2& g = node[m];
        const int nxg = g.ihi - g.ilo + 1, nyg = g.jhi - g.jlo + 1;
        const int mic = nxg / intratx[lcheck - 1] + 2, mjc = nyg / intraty[lcheck - 1] + 2;
        filval(g.q1.data(), mitot_of(m), mjtot_of(m), hx, hy, lcheck, g.time, mic, mjc, g.xlo, g.xhi, g.ylo, g.yhi, g.ilo, g.ihi, g.jlo, g.jhi,
               g.aux.data());
      }
      int mptr = lstart[lcheck];
      while (mptr != 0) {
        const int mold = mptr;
        mptr = node[mptr].levelptr;
        node[mold].q1.clear(); node[mold].q2.clear(); node[mold].aux.clear(); node[mold].bnd.clear();
        putnod(mold);
      }
      lstart[lcheck] = newstl[lcheck];
    }
    lfine = lfnew;
    const int levend = std::min(lfine, mxnest - 1);
    for (int level = lbase + 1; level <= levend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        node[m].q2.assign((size_t)nvar * mitot_of(m) * mjtot_of(m), 0.0);
        node[m].has_q2 = true;
      }
  }

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
      int cnt = 0;
      for (int m = lstart[levnew]; m != 0; m = node[m].levelptr) ++cnt;
      numgrids[levnew] = cnt;
      if (cnt > 1) arrangeGrids(levnew, cnt);
    }
    makeGridList();
    for (int levnew = lbase + 1; levnew <= lfine; ++levnew) makeBndryList(levnew);
  }

  // ================================================================ init
  void ginit(int msave, bool first, double start_time) {
    if (msave == 0) return;
    const int level = node[msave].level;
    const double hx = hxposs[level], hy = hyposs[level];
    for (int mptr = msave; mptr != 0; mptr = node[mptr].levelptr) {
      Node2& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1, nyg = g.jhi - g.jlo + 1;
      const size_t n = (size_t)nvar * (nxg + 2 * nghost) * (nyg + 2 * nghost);
      double* loc;
      if (first) {
        g.q1.assign(n, 0.0);
        if (naux > 0) {  // ginit.f:48-58
          g.aux.assign((size_t)naux * (nxg + 2 * nghost) * (nyg + 2 * nghost), 0.0);
          setaux(nghost, nxg, nyg, g.xlo, g.ylo, hx, hy, g.aux.data());
        }
        if (level < mxnest) { g.q2.assign(n, 0.0); g.has_q2 = true; }
        g.time = start_time;
        loc = g.q1.data();
      } else {
        loc = g.q2.data();
      }
      qinit(nghost, nxg, nyg, g.xlo, g.ylo, hx, hy, loc);
    }
  }

  void domain(double start_time) {
    mstart = nodget();
    Node2& g = node[mstart];
    g.xlo = xlower; g.ylo = ylower; g.yhi = yupper; g.xhi = xupper;
    g.level = 1; g.levelptr = 0;
    lstart[1] = mstart;
    g.ilo = 0; g.jlo = 0; g.ihi = nx - 1; g.jhi = ny - 1;
    lfine = 1;
    birect(mstart);
    ginit(mstart, true, start_time);
    int cnt = 0;
    for (int m = lstart[1]; m != 0; m = node[m].levelptr) ++cnt;
    numgrids[1] = cnt;
    if (cnt > 1) arrangeGrids(1, cnt);
    makeGridList();
    makeBndryList(1);
    iregsz[1] = nx; jregsz[1] = ny;
    for (int level = 2; level <= mxnest; ++level) {
      iregsz[level] = iregsz[level - 1] * intratx[level - 1];
      jregsz[level] = jregsz[level - 1] * intraty[level - 1];
      possk[level] = possk[level - 1] / (double)kratio[level - 1];
    }
  }

  void setgrd(double start_time) {
    if (mxnest == 1) return;
    int levnew = 2;
    const double t = start_time;
    while (levnew <= mxnest) {
      const int levold = levnew - 1;
      if (lstart[levold] == 0) break;
      const int lbase = levold;
      int lfnew = lbase;
      // setgrd.f:41-53: Richardson estimation needs the level one step ahead before it is
      // flagged; that step is not counted as integration work
      if (flag_richardson) {
        double dtlev;
        advanc(levold, dtlev);
        rvol = 0;
        for (double& r : rvoll) r = 0;
      }
      for (int i = 1; i <= mxnest; ++i) newstl[i] = 0;
      grdfit(lbase, levold, t, start_time);
      if (newstl[levnew] != 0) lfnew = levnew;
      ginit(newstl[levnew], true, start_time);
      lstart[levnew] = newstl[levnew];
      lfine = lfnew;
      ginit(lstart[levold], false, start_time);
      int cnt = 0;
      for (int m = lstart[levnew]; m != 0; m = node[m].levelptr) ++cnt;
      numgrids[levnew] = cnt;
      if (cnt > 1) arrangeGrids(levnew, cnt);
      makeGridList();
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

  void setbestsrc() {
    mbestsrc.assign(gauges.size(), 0);
    for (size_t i = 0; i < gauges.size(); ++i) {
      for (int lev = lfine; lev >= 1; --lev) {
        bool found = false;
        for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
          const Node2& g = node[m];
          if (gauges[i].x >= g.xlo && gauges[i].x <= g.xhi && gauges[i].y >= g.ylo && gauges[i].y <= g.yhi) {
            mbestsrc[i] = m; found = true; break;
          }
        }
        if (found) break;
      }
    }
  }

  double conck(int level) {
    const double hx = hxposs[level], hy = hyposs[level];
    double totmass = 0.0;
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
      const Node2& g = node[m];
      const int mitot = mitot_of(m), mjtot = mjtot_of(m);
      for (int j = nghost + 1; j <= mjtot - nghost; ++j)
        for (int i = nghost + 1; i <= mitot - nghost; ++i) {
          const size_t at = (j - 1) * (size_t)mitot + i - 1;
          if (mcapa == 0) totmass = totmass + g.q1[(size_t)nvar * at];
          else totmass = totmass + g.q1[(size_t)nvar * at] * g.aux[(mcapa - 1) + (size_t)naux * at];  // conck.f:55-59
        }
    }
    totmass = totmass * hx * hy;
    return totmass;
  }

  // valout.f90:8-397. ASCII (output_format 1): zeroes |q| < 1e-90 in place like the
  // reference and writes the values into fort.q. Binary (3, valout.f90:172-176): fort.q
  // holds the grid headers only and fort.b every grid's whole array (ghost cells
  // included, q(m,i,j) with m fastest) as raw doubles, nothing zeroed.
  // src/2d/valout.f90:216-286: fort.aNNNN, the aux arrays, when any component is requested
  // (every frame, or only at t0 with output_aux_onlyonce). ASCII: fort.q's headers and
  // layout, after zeroing |aux| < 1e-90 of the interior cells in place; binary: each grid's
  // whole aux array (ghost cells included, aux(m,i,j) with m fastest), nothing zeroed.
  void write_aux(int lbeg, int lend, bool binary) {
    char fn[64];
    std::snprintf(fn, sizeof(fn), "/fort.a%04d", matlabu);
    FILE* f = std::fopen((outdir + fn).c_str(), binary ? "wb" : "w");
    if (!f) throw std::runtime_error("cannot write " + outdir + fn);
    for (int level = lbeg; level <= lend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        Node2& g = node[m];
        if (binary) { std::fwrite(g.aux.data(), sizeof(double), g.aux.size(), f); continue; }
        const int mitot = mitot_of(m), mjtot = mjtot_of(m);
        std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n%6d                 mx\n%6d                 my\n",
                     m, level, g.ihi - g.ilo + 1, g.jhi - g.jlo + 1);
        std::fprintf(f, "%s    xlow\n%s    ylow\n%s    dx\n%s    dy\n\n", fmtE(g.xlo, 26, 16).c_str(), fmtE(g.ylo, 26, 16).c_str(),
                     fmtE(hxposs[level], 26, 16).c_str(), fmtE(hyposs[level], 26, 16).c_str());
        FArr A{g.aux.data(), naux, mitot, mjtot};
        for (int j = nghost + 1; j <= mjtot - nghost; ++j) {
          for (int i = nghost + 1; i <= mitot - nghost; ++i) {
            for (int ia = 1; ia <= naux; ++ia) std::fputs(fmtE(A(ia, i, j), 26, 16).c_str(), f);
            std::fputc('\n', f);
          }
          std::fputs("  \n", f);
        }
      }
    std::fclose(f);
  }
  void zero_tiny_aux(int lbeg, int lend) {
    for (int level = lbeg; level <= lend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        const int mitot = mitot_of(m), mjtot = mjtot_of(m);
        FArr A{node[m].aux.data(), naux, mitot, mjtot};
        for (int j = nghost + 1; j <= mjtot - nghost; ++j)
          for (int i = nghost + 1; i <= mitot - nghost; ++i)
            for (int ia = 1; ia <= naux; ++ia) if (std::fabs(A(ia, i, j)) < 1e-90) A(ia, i, j) = 0.0;
      }
  }

  void valout(int lbeg, int lend, double t) {
    const bool binary = output_format == 3;
    int naux_out = 0;
    for (int x : output_aux_components) naux_out += x;
    const bool out_aux = naux_out > 0 && (!output_aux_onlyonce || std::fabs(t - t0) < 1e-90);
    if (out_aux && !binary) zero_tiny_aux(lbeg, lend);
    if (out_aux && write_output) write_aux(lbeg, lend, binary);
    for (int level = lbeg; level <= lend && !binary; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        Node2& g = node[m];
        const int mitot = mitot_of(m), mjtot = mjtot_of(m);
        FArr Q{g.q1.data(), nvar, mitot, mjtot};
        for (int j = nghost + 1; j <= mjtot - nghost; ++j) for (int i = nghost + 1; i <= mitot - nghost; ++i)
          for (int iv = 1; iv <= nvar; ++iv) if (std::fabs(Q(iv, i, j)) < 1e-90) Q(iv, i, j) = 0.0;
      }
    if (write_output && binary) {
      char fn[64], fb[64];
      std::snprintf(fn, sizeof(fn), "/fort.q%04d", matlabu);
      std::snprintf(fb, sizeof(fb), "/fort.b%04d", matlabu);
      FILE* f = std::fopen((outdir + fn).c_str(), "w");
      FILE* b = std::fopen((outdir + fb).c_str(), "wb");
      int ngrids = 0;
      for (int level = lbeg; level <= lend; ++level)
        for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
          ++ngrids;
          Node2& g = node[m];
          std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n%6d                 mx\n%6d                 my\n",
                       m, level, g.ihi - g.ilo + 1, g.jhi - g.jlo + 1);
          std::fprintf(f, "%s    xlow\n%s    ylow\n%s    dx\n%s    dy\n\n", fmtE(g.xlo, 26, 16).c_str(), fmtE(g.ylo, 26, 16).c_str(),
                       fmtE(hxposs[level], 26, 16).c_str(), fmtE(hyposs[level], 26, 16).c_str());
          std::fwrite(g.q1.data(), sizeof(double), g.q1.size(), b);
        }
      std::fclose(f);
      std::fclose(b);
      std::snprintf(fn, sizeof(fn), "/fort.t%04d", matlabu);
      f = std::fopen((outdir + fn).c_str(), "w");
      std::fprintf(f, "%s    time\n%6d                 meqn\n%6d                 ngrids\n%6d                 naux\n%6d                 ndim\n%6d                 nghost\n\n",
                   fmtE(t, 18, 8).c_str(), nvar, ngrids, naux, 2, nghost);
      std::fclose(f);
    } else if (write_output) {
      char fn[64];
      std::snprintf(fn, sizeof(fn), "/fort.q%04d", matlabu);
      FILE* f = std::fopen((outdir + fn).c_str(), "w");
      int ngrids = 0;
      for (int level = lbeg; level <= lend; ++level)
        for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
          ++ngrids;
          Node2& g = node[m];
          const int mitot = mitot_of(m), mjtot = mjtot_of(m);
          std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n%6d                 mx\n%6d                 my\n",
                       m, level, g.ihi - g.ilo + 1, g.jhi - g.jlo + 1);
          std::fprintf(f, "%s    xlow\n%s    ylow\n%s    dx\n%s    dy\n\n", fmtE(g.xlo, 26, 16).c_str(), fmtE(g.ylo, 26, 16).c_str(),
                       fmtE(hxposs[level], 26, 16).c_str(), fmtE(hyposs[level], 26, 16).c_str());
          FArr Q{g.q1.data(), nvar, mitot, mjtot};
          for (int j = nghost + 1; j <= mjtot - nghost; ++j) {
            for (int i = nghost + 1; i <= mitot - nghost; ++i) {
              for (int iv = 1; iv <= nvar; ++iv) std::fputs(fmtE(Q(iv, i, j), 26, 16).c_str(), f);
              std::fputc('\n', f);
            }
            std::fputs("  \n", f);
          }
        }
      std::fclose(f);
      std::snprintf(fn, sizeof(fn), "/fort.t%04d", matlabu);
      f = std::fopen((outdir + fn).c_str(), "w");
      std::fprintf(f, "%s    time\n%6d                 meqn\n%6d                 ngrids\n%6d                 naux\n%6d                 ndim\n%6d                 nghost\n\n",
                   fmtE(t, 18, 8).c_str(), nvar, ngrids, naux, 2, nghost);
      std::fclose(f);
    }
    matlabu = matlabu + 1;
  }

  // ================================================================ tick.f
  double tick_seconds = 0, regrid_seconds = 0;
  // tick.f runs once per program; here a run may be split by max_cycles, so the
  // scheduler's state (cycle count, output index, level times) persists across calls
  // test hook: stop the scheduler right after the n-th level substep of a call
  struct DebugStop {};
  int dbg_stop = 0, dbg_count = 0;
  bool dbg_keep_input = false;  // test hook: keep store2 on the finest level too (the step's ghost-filled input)
  bool tick_started = false;
  int tk_nextout = 0;
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
    if (!tick_started) {
      tlevel[1] = time;
      for (int i = 2; i <= mxnest; ++i) tlevel[i] = tlevel[1];
    }
    tick_started = true;
    while (!(ncycle >= nstop || time >= tfinal)) {
      double outtime;
      if (nout > 0) outtime = (nextout <= nout) ? tout[nextout - 1] : RINFINITY;
      else outtime = tfinal;
      bool dumpout = false;
      if (time < outtime && time + (double)1.001f * possk[1] >= outtime) {  // 1.001 is a default-REAL literal in tick.f
        possk[1] = outtime - time;
        for (int i = 2; i <= mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
        if (nout > 0) { nextout = nextout + 1; dumpout = true; }
      }
      int level = 1;
      ntogo[level] = 1;
      for (int i = 1; i <= 10; ++i) dtnew[i] = RINFINITY;
      // label 60 / 90 / 105 state machine
      while (true) {
        // 60: regridding time?
        int lbase = -1;
        if (icheck[level] >= kcheck) lbase = level;
        else if (level + 1 >= mxnest) lbase = -1;
        else if (icheck[level + 1] >= kcheck) lbase = level + 1;
        else if (level + 2 >= mxnest) lbase = -1;
        else if (icheck[level + 2] >= kcheck) lbase = level + 2;
        if (lbase > 0) {
          if (!(lbase == mxnest || lbase > lfine)) {
            double t0c = omp_wtime_safe();
            regrid(lbase, start_time);
            regrid_seconds += omp_wtime_safe() - t0c;
            setbestsrc();
          }
          for (int i = lbase; i <= lfine; ++i) icheck[i] = 0;
          for (int i = lbase + 1; i <= lfine; ++i) tlevel[i] = tlevel[lbase];
        }
        // 90
        double dtlevnew;
        advanc(level, dtlevnew);
        if (dbg_stop > 0 && ++dbg_count >= dbg_stop) throw DebugStop();
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
        // 105
        bool done = false;
        while (true) {
          if (level == 1) { done = true; break; }
          if (ntogo[level] > 0) {
            while ((possk[level] - dtnew[level]) / dtnew[level] > (double)0.05f) {
              ntogo[level] = ntogo[level] + 1;
              possk[level] = (tlevel[level - 1] - tlevel[level]) / ntogo[level];
            }
            break;  // go to 60
          } else {
            level = level - 1;
            update(level);
          }
        }
        if (done) break;
      }
      // 110
      time = time + possk[1];
      ncycle = ncycle + 1;
      lastmass = conck(1);
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
  int max_cycles = 0;
  static double omp_wtime_safe() {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
  }

  // ================================================================ amr2.f90 driver
  void init(const std::string& dir) {
    read_input(dir);
    // amr2.f90:398-425: the capacity component is the aux component typed "capacity"
    int mc = 0;
    for (int k = 0; k < naux; ++k) {
      if (auxtype[k] == "leftface") auxtype[k] = "xleft";
      if (auxtype[k] == "bottomface") auxtype[k] = "yleft";
      if (auxtype[k] == "capacity") {
        if (mc != 0) throw std::runtime_error("only 1 capacity allowed");
        mc = k + 1;
      }
      if (auxtype[k] != "xleft" && auxtype[k] != "yleft" && auxtype[k] != "capacity" && auxtype[k] != "center")
        throw std::runtime_error("unknown type for auxiliary variables");
    }
    if (mc != mcapa) throw std::runtime_error("mcapa does not agree with auxtype");
    if (naux > 0 && problem != "advection_annulus")
      throw std::runtime_error("2D oracle: problem " + problem + " has no aux arrays (setaux)");
    hxposs[1] = (xupper - xlower) / nx;
    hyposs[1] = (yupper - ylower) / ny;
    matlabu = output_t0 ? 0 : 1;
    possk[1] = dt_initial;
    node.assign(2, Node2());
    node.resize(10001);
    for (int k = 1; k <= 10000; ++k) node[k].nextfree = k + 1;
    node[10000].nextfree = 0;
    ndfree = 1;
    lfine = 1;
    for (int i = 0; i < 12; ++i) { lstart[i] = 0; icheck[i] = 0; numgrids[i] = 0; }
    for (int level = 2; level <= mxnest; ++level) {
      hxposs[level] = hxposs[level - 1] / (double)intratx[level - 1];
      hyposs[level] = hyposs[level - 1] / (double)intraty[level - 1];
    }
    domain(t0);
    record_gauges = false;
    setgrd(t0);
    record_gauges = true;
    time = t0;
    tmass0 = conck(1);
    if (output_t0) valout(1, lfine, time);
  }
};

}  // namespace orc

// ============================================================== C entry points (tests only)
using orc::Amr2;
extern "C" {

void* oracle2d_create(const char* dir, const char* outdir, int write_output, int nthreads) {
  try {
    Amr2* a = new Amr2();
    a->outdir = outdir ? outdir : "";
    a->write_output = write_output != 0;
    a->nthreads = nthreads > 0 ? nthreads : 1;
    a->init(dir);
    return a;
  } catch (std::exception& e) {
    std::fprintf(stderr, "oracle2d_create: %s\n", e.what());
    return nullptr;
  }
}
void oracle2d_destroy(void* h) { delete (Amr2*)h; }

// Run the scheduler until tfinal (max_cycles > 0 stops after that many coarse steps).
int oracle2d_run(void* h, int max_cycles, double* seconds_out) {
  Amr2* a = (Amr2*)h;
  try {
    a->max_cycles = max_cycles;
    double t0 = Amr2::omp_wtime_safe();
    a->tick(a->t0);
    if (seconds_out) *seconds_out = Amr2::omp_wtime_safe() - t0;
    return 0;
  } catch (std::exception& e) {
    std::fprintf(stderr, "oracle2d_run: %s\n", e.what());
    return 1;
  }
}

double oracle2d_time(void* h) { return ((Amr2*)h)->time; }
double oracle2d_cell_updates(void* h) { return ((Amr2*)h)->rvol; }
double oracle2d_mass(void* h) { return ((Amr2*)h)->conck(1); }
double oracle2d_mass0(void* h) { return ((Amr2*)h)->tmass0; }
int oracle2d_lfine(void* h) { return ((Amr2*)h)->lfine; }
int oracle2d_ncycle(void* h) { return ((Amr2*)h)->ncycle; }

// Hierarchy as rows of (grid_number, level, ilo, ihi, jlo, jhi) in output order (level, list order).
// Test hook: run until the n-th level substep from now (0: no stop), leaving the state
// right after that substep. Returns 1 if it stopped there, 0 if the run ended first.
int oracle2d_run_substeps(void* h, int n) {
  Amr2* a = (Amr2*)h;
  a->dbg_stop = n; a->dbg_count = 0; a->dbg_keep_input = true;
  a->max_cycles = 0;
  int stopped = 0;
  try { a->tick(a->t0); } catch (Amr2::DebugStop&) { stopped = 1; }
  a->dbg_stop = 0;
  return stopped;
}
// Test hook: the enlarged array of grid `grid` (store 1 or 2) as [m][j][i]; returns the
// number of doubles (nvar * mitot * mjtot), 0 if the grid does not exist.
long oracle2d_patch(void* h, int grid, int store, double* out, long cap) {
  Amr2* a = (Amr2*)h;
  if (grid <= 0 || grid >= (int)a->node.size()) return 0;
  const auto& g = a->node[grid];
  const std::vector<double>& q = store == 2 ? g.q2 : g.q1;
  const int mitot = g.ihi - g.ilo + 1 + 2 * a->nghost, mjtot = g.jhi - g.jlo + 1 + 2 * a->nghost;
  const long n = (long)a->nvar * mitot * mjtot;
  if ((long)q.size() < n) return 0;
  if (out)
    for (int m = 0; m < a->nvar && m * (long)mitot * mjtot < cap; ++m)
      for (int j = 0; j < mjtot; ++j)
        for (int i = 0; i < mitot; ++i) {
          const long at = ((long)m * mjtot + j) * mitot + i;
          if (at < cap) out[at] = q[(size_t)m + (size_t)a->nvar * ((size_t)i + (size_t)mitot * j)];
        }
  return n;
}
int oracle2d_grids(void* h, int* out, int cap) {
  Amr2* a = (Amr2*)h;
  int n = 0;
  for (int level = 1; level <= a->lfine; ++level)
    for (int m = a->lstart[level]; m != 0; m = a->node[m].levelptr) {
      if (out && n < cap) {
        const auto& g = a->node[m];
        int* r = out + 6 * n;
        r[0] = m; r[1] = level; r[2] = g.ilo; r[3] = g.ihi; r[4] = g.jlo; r[5] = g.jhi;
      }
      ++n;
    }
  return n;
}
// Interior values of every grid in the order of oracle2d_grids, layout [m][j][i] per grid.
long oracle2d_values(void* h, double* out, long cap) {
  Amr2* a = (Amr2*)h;
  long n = 0;
  for (int level = 1; level <= a->lfine; ++level)
    for (int m = a->lstart[level]; m != 0; m = a->node[m].levelptr) {
      const auto& g = a->node[m];
      const int mitot = a->mitot_of(m), mjtot = a->mjtot_of(m), ng = a->nghost;
      for (int iv = 1; iv <= a->nvar; ++iv)
        for (int j = ng + 1; j <= mjtot - ng; ++j)
          for (int i = ng + 1; i <= mitot - ng; ++i) {
            if (out && n < cap) out[n] = g.q1[(iv - 1) + (size_t)a->nvar * ((j - 1) * (size_t)mitot + i - 1)];
            ++n;
          }
    }
  return n;
}
// Gauge samples: rows (gauge_num, level, t, q1..qnvar)
int oracle2d_gauges(void* h, double* out, int cap_rows) {
  Amr2* a = (Amr2*)h;
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
