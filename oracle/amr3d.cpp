// Oracle (test infrastructure only): CPU FP64 restatement of AMRClaw's 3D
// per-level patch-advance path, used as the parity checker and the CPU
// baseline of the 3D workloads. The GPU product (amrclaw_b200) never loads it.
//
// Each routine follows the reference routine named in its comment, with the
// same loop nesting and accumulation order (compile with -ffp-contract=off):
//   patch step      src/3d/stepgrid.f:4-236, step3.f:3-486, flux3.f:4-633,
//                   limiter.f:4-60, philim.f:4-58
//   level advance   src/3d/advanc.f:4-139 (advanc), :166-303 (par_advanc)
//   ghost fill      src/3d/bound.f:4-211, filpatch.f:4-282, intfil.f:4-263,
//                   trimbd.f:4-99, bc3amr.f90:70-380, init_bndryList.f
//   conservation    saveqc.f:3-111, cstore.f:4-96, icall.f:4-98, intcopy.f:4-72,
//                   qad.f:4-534, fluxsv.f:4-94, fluxad.f:4-155, update.f:4-192,
//                   upbnd.f:4-94, prepf.f:4-41, prepc.f:4-138, setuse.f:4-173
//   regrid          regrid.f:4-159, grdfit.f:4-138, flglvl.f:4-85, spest.f:4-101,
//                   flag2refine.f:3-92, setflags.f:4-33, bufnst.f:4-124,
//                   projec.f:4-101, shiftset.f:4-108, colate.f:4-78,
//                   domprep.f:4-169, domshrink.f:4-93, domup.f:4-185,
//                   domcopy.f:4-82, smartbis.f:4-157, signs.f:4-86,
//                   findcut.f:4-198, moment.f:4-70, nestck.f:4-131,
//                   birect.f:4-172, gfixup.f:4-180, filval.f:4-153
//   driver          amr3.f90, domain.f:4-124, setgrd.f:4-142, ginit.f:4-99,
//                   tick.f (same cycle as src/2d/tick.f:4-391), conck.f:4-87
//   output          valout.f90 (3D header), gauges_module.f90:302-460
//
//   periodic        prefilp.f:1-266 (prefilrecur over 27 regions), preicall.f:1-141,
//                   preintcopy.f, bound.f:60-199, filpatch.f:168-179, saveqc.f:72-91,
//                   filval.f:52-68, prepc.f:84-122, domprep.f, domshrink.f, domup.f,
//                   domcopy.f, shiftset.f (the periodic branches)
#include "common.hpp"
#include "riemann3d.hpp"
#include <algorithm>
#include <functional>
#include <memory>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc3 {
using namespace orc;

static const double RINFINITY3 = (double)10.e32f;  // amr_module.f90 rinfinity (default-REAL literal)
static const int IINFINITY3 = 999999999;
static const double GOODPT = 0.0, BADPT = 2.0, BADPRO = 3.0;  // src/3d/amr_module.f90:53-55
static const int IPLANE = 1, JPLANE = 2, KPLANE = 3;

struct GaugeSample3 { int level; double t; std::vector<double> v; };
struct Gauge3 {
  int num; double x, y, z, t_start, t_end, last_time, min_inc;
  std::vector<GaugeSample3> data;
};

struct Node3 {
  int ilo = 0, ihi = 0, jlo = 0, jhi = 0, klo = 0, khi = 0, level = 0, levelptr = 0, nextfree = 0;
  double xlo = 0, xhi = 0, ylo = 0, yhi = 0, zlo = 0, zhi = 0, time = 0;
  std::vector<double> q1, q2, aux;  // store1, store2, storeaux (var fastest, then i, j, k)
  bool has_q2 = false;
  std::vector<double> ffl;          // ffluxptr: svdflx(nvar,lenbc) qc1d(nvar,lenbc) auxc1d(naux,lenbc)
  bool has_ffl = false;
  std::vector<int> listbc;          // cfluxptr: listbc(6,maxsp)
  bool has_cfl = false;
  std::vector<int> bnd;             // same-level neighbours, bndList traversal order
  std::vector<double> tmp;          // spest.f temporary copy with ghost cells (tempptr)
};

// A Fortran array val(nvar, nrow, ncol, nfil) with 1-based indices.
struct FArr3 {
  double* p; int nvar, nrow, ncol, nfil;
  double& operator()(int m, int i, int j, int k) const {
    return p[(m - 1) + (size_t)nvar * ((i - 1) + (size_t)nrow * ((j - 1) + (size_t)ncol * (k - 1)))];
  }
};
// integer*1 flag array with indices (0:isize+1, 0:jsize+1, 0:ksize+1)
struct I1 {
  std::vector<signed char> v; int is = 0, js = 0, ks = 0;
  void init(int a, int b, int c) { is = a; js = b; ks = c; v.assign((size_t)(a + 2) * (b + 2) * (c + 2), 0); }
  signed char& operator()(int i, int j, int k) { return v[(size_t)i + (size_t)(is + 2) * ((size_t)j + (size_t)(js + 2) * k)]; }
};

struct Amr3 {
  // ---------------- input
  double xlower, ylower, zlower, xupper, yupper, zupper;
  int nx, ny, nz, nvar, mwaves, naux;
  double t0;
  int output_style = 1, nout = 0, iout = 0, nstop = IINFINITY3;
  double tfinal = 0; bool output_t0 = true;
  std::vector<int> output_aux_components;
  bool output_aux_onlyonce = true;
  int output_format = 1;
  std::vector<double> tout;
  double dt_initial, dt_max, cflv1, cfl;
  int nv1; bool vtime;
  int method[8] = {0};
  int dimensional_split = 0, mcapa = 0;
  bool use_fwaves = false;
  std::vector<int> mthlim;
  int nghost = 2;
  int mthbc[7] = {0};
  bool xperdom = false, yperdom = false, zperdom = false;
  int mxnest = 1;
  int intratx[12], intraty[12], intratz[12], kratio[12];
  std::vector<std::string> auxtype;
  bool flag_richardson = false, flag_gradient = true;
  double tol = -1, tolsp = 0.05, cut = 0.7;
  int kcheck = 2, ibuff = 3;
  int max1d = 32;
  std::vector<Gauge3> gauges;
  ProbParams prob;
  std::string problem;
  double blast_x = 0, blast_y = 0, blast_z = 0, blast_r = 0.2, blast_pin = 5.0, blast_pout = 1.0;
  int flag_pressure = 0;  // 1: flag on the pressure difference (euler_3d_radial flag2refine pattern)
  // swirl variants: the initial condition is the reference test's half space (x < 0.5) or a
  // sphere; vel_period > 0 scales the velocities by cos(pi t / vel_period) in b4step3
  bool swirl_sphere = false;
  double sph_x = 0.5, sph_y = 0.25, sph_z = 0.5, sph_r = 0.15, vel_period = 0.0;

  // ---------------- state
  std::vector<Node3> node;
  int ndfree = 1;
  int lfine = 1;
  int lstart[12] = {0}, newstl[12] = {0}, listsp[12] = {0};
  int iregsz[12], jregsz[12], kregsz[12], icheck[12] = {0};
  double hxposs[12], hyposs[12], hzposs[12], possk[12];
  std::vector<int> levelgrids[12];
  double cfl_level = 0, cflmax = 0;
  double rvol = 0, rvoll[12] = {0};
  double tmass0 = 0;
  std::string outdir;
  bool write_output = false;
  bool record_gauges = true;
  int nthreads = 1;
  std::vector<int> mbestsrc;
  double time = 0;
  int ncycle = 0;
  int matlabu = 0;

  // ========================================================== input (amr3.f90)
  void read_input(const std::string& dir) {
    DataFile c, a, g, s;
    if (!c.load(dir + "/claw.data")) throw std::runtime_error("cannot read claw.data");
    if (!a.load(dir + "/amr.data")) throw std::runtime_error("cannot read amr.data");
    xlower = c.d("lower", 0); ylower = c.d("lower", 1); zlower = c.d("lower", 2);
    xupper = c.d("upper", 0); yupper = c.d("upper", 1); zupper = c.d("upper", 2);
    nx = c.i("num_cells", 0); ny = c.i("num_cells", 1); nz = c.i("num_cells", 2);
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
      nout = 0; tfinal = RINFINITY3;
    }
    if (output_style == 1 && nout > 0) {
      tout.resize(nout);
      for (int k = 1; k <= nout; ++k) tout[k - 1] = t0 + k * (tfinal - t0) / (double)nout;
    }
    dt_initial = c.d("dt_initial"); dt_max = c.d("dt_max");
    cflv1 = c.d("cfl_max"); cfl = c.d("cfl_desired"); nv1 = c.i("steps_max");
    if (output_style != 3) nstop = IINFINITY3;
    vtime = c.b("dt_variable");
    method[1] = vtime ? 2 : 1;
    method[2] = c.i("order"); method[3] = c.i("transverse_waves");
    dimensional_split = c.i("dimensional_split");
    method[4] = c.i("verbosity"); method[5] = c.i("source_split");
    mcapa = c.i("capa_index"); use_fwaves = c.b("use_fwaves");
    output_format = c.iget("output_format", 1);
    if (output_format != 1 && output_format != 3) throw std::runtime_error("output_format must be 1 (ASCII) or 3 (binary)");
    // amr2.f90:212-218 (amr3.f90 alike): aux components written to fort.aNNNN
    if (naux > 0 && c.has("output_aux_components")) {
      for (int k = 0; k < naux; ++k) output_aux_components.push_back(c.i("output_aux_components", k));
      output_aux_onlyonce = c.has("output_aux_onlyonce") ? c.b("output_aux_onlyonce") : true;
    }
    for (int k = 0; k < mwaves; ++k) mthlim.push_back(c.i("limiter", k));
    nghost = c.i("num_ghost");
    for (int d = 0; d < 3; ++d) { mthbc[2 * d + 1] = c.i("bc_lower", d); mthbc[2 * d + 2] = c.i("bc_upper", d); }
    xperdom = (mthbc[1] == 2 && mthbc[2] == 2);
    yperdom = (mthbc[3] == 2 && mthbc[4] == 2);
    zperdom = (mthbc[5] == 2 && mthbc[6] == 2);
    // amr3.f90:241-246: Godunov splitting (1) only; Strang splitting stops the reference
    if (dimensional_split > 1) throw std::runtime_error("Strang splitting is not supported (amrclaw stops)");
    if (method[3] < 0) throw std::runtime_error("transverse_waves < 0 (dimensional splitting) is not supported");
    if (mcapa != 0) throw std::runtime_error("capacity functions are not supported in 3D");
    mxnest = a.i("amr_levels_max");
    const int nr = std::max(1, mxnest - 1);
    for (int k = 0; k < nr; ++k) {
      intratx[k + 1] = a.i("refinement_ratios_x", k);
      intraty[k + 1] = a.i("refinement_ratios_y", k);
      intratz[k + 1] = a.i("refinement_ratios_z", k);
      kratio[k + 1] = a.i("refinement_ratios_t", k);
    }
    if (naux > 0) for (int k = 0; k < naux; ++k) auxtype.push_back(a.s("aux_type", k));
    flag_richardson = a.b("flag_richardson"); tol = a.d("flag_richardson_tol");
    if (flag_richardson && naux > 0) throw std::runtime_error("Richardson estimation needs num_aux = 0 (no auxcoarsen)");
    // bufnst.f:21-24 adds store2's first component to the flags whenever tol > 0: without
    // errest.f having written flags there, that would be the old solution
    if (!flag_richardson && tol > 0) throw std::runtime_error("flag_richardson_tol > 0 needs flag_richardson");
    flag_gradient = a.b("flag2refine"); tolsp = a.d("flag2refine_tol");
    kcheck = a.i("regrid_interval"); ibuff = a.i("regrid_buffer_width");
    cut = a.d("clustering_cutoff");
    max1d = a.iget("max1d", 32);
    if (g.load(dir + "/gauges.data")) {
      for (auto& row : g.rows) {
        if (row.size() < 6) continue;
        Gauge3 ga;
        ga.num = (int)DataFile::tod(row[0]);
        ga.x = DataFile::tod(row[1]); ga.y = DataFile::tod(row[2]); ga.z = DataFile::tod(row[3]);
        ga.t_start = DataFile::tod(row[4]); ga.t_end = DataFile::tod(row[5]);
        ga.last_time = ga.t_start; ga.min_inc = row.size() > 6 ? DataFile::tod(row[6]) : 0.0;
        gauges.push_back(ga);
      }
    }
    if (!s.load(dir + "/setprob.data")) throw std::runtime_error("cannot read setprob.data");
    problem = s.s("problem");
    if (problem == "advection_swirl") {
      prob.solver = SOLVER_VC_ADVECTION;
      if (naux != 3) throw std::runtime_error("advection_swirl needs 3 aux components");
      swirl_sphere = s.sget("ic", "halfspace") == "sphere";
      sph_x = s.dget("x0", 0.5); sph_y = s.dget("y0", 0.25); sph_z = s.dget("z0", 0.5); sph_r = s.dget("r0", 0.15);
      vel_period = s.dget("vel_period", 0.0);
    } else if (problem == "euler_blast") {
      prob.solver = SOLVER_EULER; prob.gamma = s.d("gamma"); prob.gamma1 = prob.gamma - 1.0;
      prob.efix = s.iget("efix", 1) != 0;
      blast_x = s.d("x0"); blast_y = s.d("y0"); blast_z = s.d("z0"); blast_r = s.d("r0");
      blast_pin = s.d("pin"); blast_pout = s.d("pout");
      flag_pressure = s.iget("flag_pressure", 1);
    } else {
      throw std::runtime_error("unknown problem " + problem);
    }
  }

  // =================================================== problem plugins
  // qinit.f of the applications: tests/advection_3d_swirl/qinit.f:5-42 (swirl);
  // the Euler blast sets rho = 1, u = v = w = 0, p = pin within r0 of (x0,y0,z0), pout outside.
  void qinit(int mbc, int mx, int my, int mz, double xl, double yl, double zl, double dx, double dy, double dz, double* q) {
    FArr3 Q{q, nvar, mx + 2 * mbc, my + 2 * mbc, mz + 2 * mbc};
    auto at = [&](int m, int i, int j, int k) -> double& { return Q(m, i + mbc, j + mbc, k + mbc); };
    if (problem == "advection_swirl" && swirl_sphere) {
      // q = 1 inside the sphere of radius r0 about (x0, y0, z0), 0 outside
      for (int k = 1; k <= mz; ++k) {
        const double zc = zl + (k - 0.5) * dz;
        for (int j = 1; j <= my; ++j) {
          const double yc = yl + (j - 0.5) * dy;
          for (int i = 1; i <= mx; ++i) {
            const double xc = xl + (i - 0.5) * dx;
            const double ddx = xc - sph_x, ddy = yc - sph_y, ddz = zc - sph_z;
            at(1, i, j, k) = (ddx * ddx + ddy * ddy + ddz * ddz <= sph_r * sph_r) ? 1.0 : 0.0;
          }
        }
      }
    } else if (problem == "advection_swirl") {
      for (int i = 1; i <= mx; ++i) {
        const double x = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j)
          for (int k = 1; k <= mz; ++k) at(1, i, j, k) = (x < 0.5) ? 1.0 : 0.0;
      }
    } else {
      const double g1 = prob.gamma - 1.0;
      for (int k = 1; k <= mz; ++k) {
        const double zc = zl + (k - 0.5) * dz;
        for (int j = 1; j <= my; ++j) {
          const double yc = yl + (j - 0.5) * dy;
          for (int i = 1; i <= mx; ++i) {
            const double xc = xl + (i - 0.5) * dx;
            const double ddx = xc - blast_x, ddy = yc - blast_y, ddz = zc - blast_z;
            const double r = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            const double p = (r <= blast_r) ? blast_pin : blast_pout;
            at(1, i, j, k) = 1.0; at(2, i, j, k) = 0.0; at(3, i, j, k) = 0.0; at(4, i, j, k) = 0.0;
            at(5, i, j, k) = p / g1;
          }
        }
      }
    }
  }
  // tests/advection_3d_swirl/setaux.f:2-85: velocities at the left x-, y- and z-face of each cell
  void setaux(int mbc, int mx, int my, int mz, double xl, double yl, double zl, double dx, double dy, double dz, double* aux) {
    if (naux == 0) return;
    FArr3 A{aux, naux, mx + 2 * mbc, my + 2 * mbc, mz + 2 * mbc};
    const double pi = 4.0 * std::atan(1.0), pi2 = 2.0 * pi;
    const double dx2 = 0.5 * dx, dy2 = 0.5 * dy, dz2 = 0.5 * dz;
    auto su = [&](double x, double y, double z) { double s = std::sin(pi * x); return 2.0 * (s * s) * std::sin(pi2 * y) * std::sin(pi2 * z); };
    auto sv = [&](double x, double y, double z) { double s = std::sin(pi * y); return -std::sin(pi2 * x) * (s * s) * std::sin(pi2 * z); };
    auto sw = [&](double x, double y, double z) { double s = std::sin(pi * z); return -std::sin(pi2 * x) * std::sin(pi2 * y) * (s * s); };
    for (int k = 1 - mbc; k <= mz + mbc; ++k) {
      const double zc = zl + (k - 0.5) * dz;
      for (int j = 1 - mbc; j <= my + mbc; ++j) {
        const double yc = yl + (j - 0.5) * dy;
        for (int i = 1 - mbc; i <= mx + mbc; ++i) {
          const double xc = xl + (i - 0.5) * dx;
          A(1, i + mbc, j + mbc, k + mbc) = su(xc - dx2, yc, zc);
          A(2, i + mbc, j + mbc, k + mbc) = sv(xc, yc - dy2, zc);
          A(3, i + mbc, j + mbc, k + mbc) = sw(xc, yc, zc - dz2);
        }
      }
    }
  }

  // b4step3 (src/3d/b4step3.f90:2-16 is the no-op default; stepgrid.f:113 calls it with the
  // grid's time before step3): the time-modulated swirl sets the face velocities of the
  // whole enlarged patch to setaux's values times cos(pi t / vel_period)
  void b4step3(int mx, int my, int mz, double xl, double yl, double zl, double dx, double dy, double dz, double t, double* aux) {
    if (problem != "advection_swirl" || vel_period <= 0.0) return;
    setaux(nghost, mx, my, mz, xl, yl, zl, dx, dy, dz, aux);
    const double pi = 4.0 * std::atan(1.0);
    const double c = std::cos(pi * t / vel_period);
    const size_t n = (size_t)naux * (mx + 2 * nghost) * (my + 2 * nghost) * (mz + 2 * nghost);
    for (size_t i = 0; i < n; ++i) aux[i] = aux[i] * c;
  }

  // =================================================== node store (nodget.f)
  int nodget() {
    if (ndfree == 0) {
      const int old = (int)node.size() - 1, add = 10000;
      node.resize(old + 1 + add);
      for (int k = old + 1; k <= old + add; ++k) node[k].nextfree = k + 1;
      node[old + add].nextfree = 0;
      ndfree = old + 1;
    }
    const int m = ndfree;
    ndfree = node[m].nextfree;
    node[m] = Node3();
    return m;
  }
  void putnod(int m) { node[m].nextfree = ndfree; ndfree = m; }
  int mitot_of(int m) const { return node[m].ihi - node[m].ilo + 1 + 2 * nghost; }
  int mjtot_of(int m) const { return node[m].jhi - node[m].jlo + 1 + 2 * nghost; }
  int mktot_of(int m) const { return node[m].khi - node[m].klo + 1 + 2 * nghost; }
  size_t qsize(int m) const { return (size_t)nvar * mitot_of(m) * mjtot_of(m) * mktot_of(m); }
  size_t asize(int m) const { return (size_t)naux * mitot_of(m) * mjtot_of(m) * mktot_of(m); }

  // ===================================================== patch step
  // limiter.f:4-60 with philim.f:4-58
  void limiter(int meqn, int mx, Waves wave, Slice s) {
    for (int mw = 1; mw <= mwaves; ++mw) {
      if (mthlim[mw - 1] == 0) continue;
      double dotr = 0.0;
      for (int i = 0; i <= mx + 1; ++i) {
        double wnorm2 = 0.0;
        const double dotl = dotr;
        dotr = 0.0;
        for (int m = 1; m <= meqn; ++m) {
          wnorm2 = wnorm2 + wave(m, mw, i) * wave(m, mw, i);
          dotr = dotr + wave(m, mw, i) * wave(m, mw, i + 1);
        }
        if (i == 0) continue;
        if (wnorm2 == 0.0) continue;
        const double r = (s(mw, i) > 0.0) ? dotl / wnorm2 : dotr / wnorm2;
        double wl = 0.0;
        switch (mthlim[mw - 1]) {
          case 1: wl = std::max(0.0, std::min(1.0, r)); break;
          case 2: wl = std::max(std::max(0.0, std::min(1.0, 2.0 * r)), std::min(2.0, r)); break;
          case 3: wl = (r + std::fabs(r)) / (1.0 + std::fabs(r)); break;
          case 4: { const double c = (1.0 + r) / 2.0; wl = std::max(0.0, std::min(std::min(c, 2.0), 2.0 * r)); } break;
          case 5: wl = r; break;
        }
        for (int m = 1; m <= meqn; ++m) wave(m, mw, i) = wl * wave(m, mw, i);
      }
    }
  }

  // One pencil's work arrays (flux3.f arguments), indices 1-mbc .. maxm+mbc.
  struct Pencil {
    int base = 0, L = 0, meqn = 0, maux = 0, mw = 0;
    std::vector<double> q1d, dtdx1d, aux1, aux2, aux3, faddm, faddp, gadd, hadd, wave, s;
    std::vector<double> v[40];  // amdq, apdq, cqxx, and the transverse work vectors
    void init(int maxm, int mbc, int meqn_, int mwaves, int maux_) {
      base = 1 - mbc; L = maxm + 2 * mbc; meqn = meqn_; maux = std::max(maux_, 1); mw = mwaves;
      q1d.assign((size_t)meqn * L, 0); dtdx1d.assign(L, 0);
      aux1.assign((size_t)maux * L * 3, 0); aux2 = aux1; aux3 = aux1;
      faddm.assign((size_t)meqn * L, 0); faddp = faddm;
      gadd.assign((size_t)meqn * L * 6, 0); hadd = gadd;
      wave.assign((size_t)meqn * mwaves * L, 0); s.assign((size_t)mwaves * L, 0);
      for (auto& x : v) x.assign((size_t)meqn * L, 0);
    }
    Slice sl(std::vector<double>& x) { return Slice{x.data(), meqn, base}; }
    // gadd(m, i, side 1..2, d -1..1)
    double& G(std::vector<double>& x, int m, int i, int side, int d) {
      return x[(m - 1) + (size_t)meqn * ((i - base) + (size_t)L * ((side - 1) + 2 * (d + 1)))];
    }
  };

  // flux3.f:4-633
  void flux3(int ixyz, int meqn, int maux, int mbc, int mx, Pencil& W, double dtdy, double dtdz, double& cfl1d) {
    const int base = W.base;
    Slice q1d = W.sl(W.q1d);
    auto dtdx1d = [&](int i) -> double { return W.dtdx1d[i - base]; };
    AuxSlice3 aux1{W.aux1.data(), W.maux, base, W.L}, aux2{W.aux2.data(), W.maux, base, W.L}, aux3{W.aux3.data(), W.maux, base, W.L};
    Slice aux2c{W.aux2.data() + (size_t)W.maux * W.L, W.maux, base};  // aux2(:, :, 2)
    Slice faddm = W.sl(W.faddm), faddp = W.sl(W.faddp);
    Waves wave{W.wave.data(), meqn, mwaves, base};
    Slice s{W.s.data(), mwaves, base};
    enum { AMDQ, APDQ, CQXX, BMAMDQ, BMAPDQ, BPAMDQ, BPAPDQ, CMAMDQ, CMAPDQ, CPAMDQ, CPAPDQ, CMAMDQ2, CMAPDQ2,
           CPAMDQ2, CPAPDQ2, BMCQXXM, BMCQXXP, BPCQXXM, BPCQXXP, CMCQXXM, CMCQXXP, CPCQXXM, CPCQXXP, BMCMAMDQ,
           BMCMAPDQ, BPCMAMDQ, BPCMAPDQ, BMCPAMDQ, BMCPAPDQ, BPCPAMDQ, BPCPAPDQ };
    auto V = [&](int id) { return W.sl(W.v[id]); };
    Slice amdq = V(AMDQ), apdq = V(APDQ), cqxx = V(CQXX);
    bool limit = false;
    for (int mw = 1; mw <= mwaves; ++mw) if (mthlim[mw - 1] > 0) limit = true;
    for (int m = 1; m <= meqn; ++m)
      for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        faddm(m, i) = 0.0; faddp(m, i) = 0.0;
        for (int side = 1; side <= 2; ++side)
          for (int d = -1; d <= 1; ++d) { W.G(W.gadd, m, i, side, d) = 0.0; W.G(W.hadd, m, i, side, d) = 0.0; }
      }
    int m3, m4;
    if (method[3] < 0) { m3 = -1; m4 = 0; }
    else { m3 = method[3] / 10; m4 = method[3] - 10 * m3; }
    rpn3(prob, ixyz, meqn, mwaves, mbc, mx, q1d, q1d, aux2c, aux2c, wave, s, amdq, apdq);
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
      if (limit) limiter(meqn, mx, wave, s);
      for (int i = 1; i <= mx + 1; ++i) {
        const double dtdxave = 0.5 * (dtdx1d(i - 1) + dtdx1d(i));
        for (int m = 1; m <= meqn; ++m) {
          cqxx(m, i) = 0.0;
          for (int mw = 1; mw <= mwaves; ++mw) {
            const double sg = use_fwaves ? dsign(1.0, s(mw, i)) : std::fabs(s(mw, i));
            cqxx(m, i) = cqxx(m, i) + 0.5 * sg * (1.0 - std::fabs(s(mw, i)) * dtdxave) * wave(m, mw, i);
          }
          faddm(m, i) = faddm(m, i) + cqxx(m, i);
          faddp(m, i) = faddp(m, i) + cqxx(m, i);
        }
      }
    }
    if (m3 <= 0) return;
    rpt3(prob, ixyz, 2, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, amdq, V(BMAMDQ), V(BPAMDQ));
    rpt3(prob, ixyz, 2, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, apdq, V(BMAPDQ), V(BPAPDQ));
    rpt3(prob, ixyz, 3, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, amdq, V(CMAMDQ), V(CPAMDQ));
    rpt3(prob, ixyz, 3, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, apdq, V(CMAPDQ), V(CPAPDQ));
    if (m3 == 2) {
      if (maux > 0) {
        rpt3(prob, ixyz, 2, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, cqxx, V(BMCQXXM), V(BPCQXXM));
        rpt3(prob, ixyz, 2, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, cqxx, V(BMCQXXP), V(BPCQXXP));
        rpt3(prob, ixyz, 3, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, cqxx, V(CMCQXXM), V(CPCQXXM));
        rpt3(prob, ixyz, 3, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, cqxx, V(CMCQXXP), V(CPCQXXP));
      } else {
        rpt3(prob, ixyz, 2, 0, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, cqxx, V(BMCQXXM), V(BPCQXXM));
        rpt3(prob, ixyz, 3, 0, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, cqxx, V(CMCQXXM), V(CPCQXXM));
        for (int i = 0; i <= mx + 2; ++i)
          for (int m = 1; m <= meqn; ++m) {
            V(BMCQXXP)(m, i) = V(BMCQXXM)(m, i); V(BPCQXXP)(m, i) = V(BPCQXXM)(m, i);
            V(CMCQXXP)(m, i) = V(CMCQXXM)(m, i); V(CPCQXXP)(m, i) = V(CPCQXXM)(m, i);
          }
      }
    }
    if (m4 == 1) {
      for (int i = 0; i <= mx + 2; ++i)
        for (int m = 1; m <= meqn; ++m) {
          V(CPAPDQ2)(m, i) = V(CPAPDQ)(m, i); V(CPAMDQ2)(m, i) = V(CPAMDQ)(m, i);
          V(CMAPDQ2)(m, i) = V(CMAPDQ)(m, i); V(CMAMDQ2)(m, i) = V(CMAMDQ)(m, i);
        }
    } else if (m4 == 2) {
      for (int i = 0; i <= mx + 2; ++i)
        for (int m = 1; m <= meqn; ++m) {
          V(CPAPDQ2)(m, i) = V(CPAPDQ)(m, i) - 3.0 * V(CPCQXXP)(m, i);
          V(CPAMDQ2)(m, i) = V(CPAMDQ)(m, i) + 3.0 * V(CPCQXXM)(m, i);
          V(CMAPDQ2)(m, i) = V(CMAPDQ)(m, i) - 3.0 * V(CMCQXXP)(m, i);
          V(CMAMDQ2)(m, i) = V(CMAMDQ)(m, i) + 3.0 * V(CMCQXXM)(m, i);
        }
    }
    if (m4 > 0) {
      rptt3(prob, ixyz, 2, 2, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(CPAPDQ2), V(BMCPAPDQ), V(BPCPAPDQ));
      rptt3(prob, ixyz, 2, 1, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(CPAMDQ2), V(BMCPAMDQ), V(BPCPAMDQ));
      rptt3(prob, ixyz, 2, 2, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(CMAPDQ2), V(BMCMAPDQ), V(BPCMAPDQ));
      rptt3(prob, ixyz, 2, 1, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(CMAMDQ2), V(BMCMAMDQ), V(BPCMAMDQ));
    }
    const double c6 = 1.0 / 6.0;
    auto g = [&](int m, int i, int side, int d) -> double& { return W.G(W.gadd, m, i, side, d); };
    auto h = [&](int m, int i, int side, int d) -> double& { return W.G(W.hadd, m, i, side, d); };
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= meqn; ++m) {
        g(m, i - 1, 1, 0) = g(m, i - 1, 1, 0) - 0.5 * dtdx1d(i - 1) * V(BMAMDQ)(m, i);
        g(m, i - 1, 2, 0) = g(m, i - 1, 2, 0) - 0.5 * dtdx1d(i - 1) * V(BPAMDQ)(m, i);
        g(m, i, 1, 0) = g(m, i, 1, 0) - 0.5 * dtdx1d(i) * V(BMAPDQ)(m, i);
        g(m, i, 2, 0) = g(m, i, 2, 0) - 0.5 * dtdx1d(i) * V(BPAPDQ)(m, i);
        if (m4 > 0) {
          g(m, i, 2, 0) = g(m, i, 2, 0) + c6 * dtdx1d(i - 1) * dtdz * (V(BPCPAPDQ)(m, i) - V(BPCMAPDQ)(m, i));
          g(m, i, 1, 0) = g(m, i, 1, 0) + c6 * dtdx1d(i) * dtdz * (V(BMCPAPDQ)(m, i) - V(BMCMAPDQ)(m, i));
          g(m, i, 2, 1) = g(m, i, 2, 1) - c6 * dtdx1d(i) * dtdz * V(BPCPAPDQ)(m, i);
          g(m, i, 1, 1) = g(m, i, 1, 1) - c6 * dtdx1d(i) * dtdz * V(BMCPAPDQ)(m, i);
          g(m, i, 2, -1) = g(m, i, 2, -1) + c6 * dtdx1d(i) * dtdz * V(BPCMAPDQ)(m, i);
          g(m, i, 1, -1) = g(m, i, 1, -1) + c6 * dtdx1d(i) * dtdz * V(BMCMAPDQ)(m, i);
          g(m, i - 1, 2, 0) = g(m, i - 1, 2, 0) + c6 * dtdx1d(i - 1) * dtdz * (V(BPCPAMDQ)(m, i) - V(BPCMAMDQ)(m, i));
          g(m, i - 1, 1, 0) = g(m, i - 1, 1, 0) + c6 * dtdx1d(i - 1) * dtdz * (V(BMCPAMDQ)(m, i) - V(BMCMAMDQ)(m, i));
          g(m, i - 1, 2, 1) = g(m, i - 1, 2, 1) - c6 * dtdx1d(i - 1) * dtdz * V(BPCPAMDQ)(m, i);
          g(m, i - 1, 1, 1) = g(m, i - 1, 1, 1) - c6 * dtdx1d(i - 1) * dtdz * V(BMCPAMDQ)(m, i);
          g(m, i - 1, 2, -1) = g(m, i - 1, 2, -1) + c6 * dtdx1d(i - 1) * dtdz * V(BPCMAMDQ)(m, i);
          g(m, i - 1, 1, -1) = g(m, i - 1, 1, -1) + c6 * dtdx1d(i - 1) * dtdz * V(BMCMAMDQ)(m, i);
        }
        if (m3 < 2) continue;
        g(m, i, 2, 0) = g(m, i, 2, 0) + dtdx1d(i) * V(BPCQXXP)(m, i);
        g(m, i, 1, 0) = g(m, i, 1, 0) + dtdx1d(i) * V(BMCQXXP)(m, i);
        g(m, i - 1, 2, 0) = g(m, i - 1, 2, 0) - dtdx1d(i - 1) * V(BPCQXXM)(m, i);
        g(m, i - 1, 1, 0) = g(m, i - 1, 1, 0) - dtdx1d(i - 1) * V(BMCQXXM)(m, i);
      }
    if (m4 == 2) {
      for (int i = 0; i <= mx + 2; ++i)
        for (int m = 1; m <= meqn; ++m) {
          V(BPAPDQ)(m, i) = V(BPAPDQ)(m, i) - 3.0 * V(BPCQXXP)(m, i);
          V(BPAMDQ)(m, i) = V(BPAMDQ)(m, i) + 3.0 * V(BPCQXXM)(m, i);
          V(BMAPDQ)(m, i) = V(BMAPDQ)(m, i) - 3.0 * V(BMCQXXP)(m, i);
          V(BMAMDQ)(m, i) = V(BMAMDQ)(m, i) + 3.0 * V(BMCQXXM)(m, i);
        }
    }
    if (m4 > 0) {
      rptt3(prob, ixyz, 3, 2, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(BPAPDQ), V(BMCPAPDQ), V(BPCPAPDQ));
      rptt3(prob, ixyz, 3, 1, 2, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(BPAMDQ), V(BMCPAMDQ), V(BPCPAMDQ));
      rptt3(prob, ixyz, 3, 2, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(BMAPDQ), V(BMCMAPDQ), V(BPCMAPDQ));
      rptt3(prob, ixyz, 3, 1, 1, meqn, mbc, mx, q1d, q1d, aux1, aux2, aux3, V(BMAMDQ), V(BMCMAMDQ), V(BPCMAMDQ));
    }
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= meqn; ++m) {
        h(m, i - 1, 1, 0) = h(m, i - 1, 1, 0) - 0.5 * dtdx1d(i - 1) * V(CMAMDQ)(m, i);
        h(m, i - 1, 2, 0) = h(m, i - 1, 2, 0) - 0.5 * dtdx1d(i - 1) * V(CPAMDQ)(m, i);
        h(m, i, 1, 0) = h(m, i, 1, 0) - 0.5 * dtdx1d(i) * V(CMAPDQ)(m, i);
        h(m, i, 2, 0) = h(m, i, 2, 0) - 0.5 * dtdx1d(i) * V(CPAPDQ)(m, i);
        if (m4 > 0) {
          h(m, i, 2, 0) = h(m, i, 2, 0) + c6 * dtdx1d(i) * dtdy * (V(BPCPAPDQ)(m, i) - V(BPCMAPDQ)(m, i));
          h(m, i, 1, 0) = h(m, i, 1, 0) + c6 * dtdx1d(i) * dtdy * (V(BMCPAPDQ)(m, i) - V(BMCMAPDQ)(m, i));
          h(m, i, 2, 1) = h(m, i, 2, 1) - c6 * dtdx1d(i) * dtdy * V(BPCPAPDQ)(m, i);
          h(m, i, 1, 1) = h(m, i, 1, 1) - c6 * dtdx1d(i) * dtdy * V(BMCPAPDQ)(m, i);
          h(m, i, 2, -1) = h(m, i, 2, -1) + c6 * dtdx1d(i) * dtdy * V(BPCMAPDQ)(m, i);
          h(m, i, 1, -1) = h(m, i, 1, -1) + c6 * dtdx1d(i) * dtdy * V(BMCMAPDQ)(m, i);
          h(m, i - 1, 2, 0) = h(m, i - 1, 2, 0) + c6 * dtdx1d(i - 1) * dtdy * (V(BPCPAMDQ)(m, i) - V(BPCMAMDQ)(m, i));
          h(m, i - 1, 1, 0) = h(m, i - 1, 1, 0) + c6 * dtdx1d(i - 1) * dtdy * (V(BMCPAMDQ)(m, i) - V(BMCMAMDQ)(m, i));
          h(m, i - 1, 2, 1) = h(m, i - 1, 2, 1) - c6 * dtdx1d(i - 1) * dtdy * V(BPCPAMDQ)(m, i);
          h(m, i - 1, 1, 1) = h(m, i - 1, 1, 1) - c6 * dtdx1d(i - 1) * dtdy * V(BMCPAMDQ)(m, i);
          h(m, i - 1, 2, -1) = h(m, i - 1, 2, -1) + c6 * dtdx1d(i - 1) * dtdy * V(BPCMAMDQ)(m, i);
          h(m, i - 1, 1, -1) = h(m, i - 1, 1, -1) + c6 * dtdx1d(i - 1) * dtdy * V(BMCMAMDQ)(m, i);
        }
        if (m3 < 2) continue;
        h(m, i, 2, 0) = h(m, i, 2, 0) + dtdx1d(i) * V(CPCQXXP)(m, i);
        h(m, i, 1, 0) = h(m, i, 1, 0) + dtdx1d(i) * V(CMCQXXP)(m, i);
        h(m, i - 1, 2, 0) = h(m, i - 1, 2, 0) - dtdx1d(i - 1) * V(CPCQXXM)(m, i);
        h(m, i - 1, 1, 0) = h(m, i - 1, 1, 0) - dtdx1d(i - 1) * V(CMCQXXM)(m, i);
      }
  }

  // step3.f:3-486 ; fm..hp are (nvar, mitot, mjtot, mktot) arrays of the enlarged patch
  void step3(int mx, int my, int mz, const double* qold, const double* aux, double dx, double dy, double dz, double dt,
             double& cflgrid, double* fm, double* fp, double* gm, double* gp, double* hm, double* hp) {
    const int mbc = nghost, meqn = nvar, maux = naux;
    const int mitot = mx + 2 * mbc, mjtot = my + 2 * mbc, mktot = mz + 2 * mbc;
    const int maxm = std::max(mx, std::max(my, mz));
    auto at = [&](int i, int j, int k) { return (size_t)(i + mbc - 1) + (size_t)mitot * ((size_t)(j + mbc - 1) + (size_t)mjtot * (k + mbc - 1)); };
    auto Q = [&](int m, int i, int j, int k) { return qold[(m - 1) + (size_t)meqn * at(i, j, k)]; };
    auto A = [&](int m, int i, int j, int k) { return aux[(m - 1) + (size_t)maux * at(i, j, k)]; };
    auto F = [&](double* f, int m, int i, int j, int k) -> double& { return f[(m - 1) + (size_t)meqn * at(i, j, k)]; };
    Pencil W;
    W.init(maxm, mbc, meqn, mwaves, maux);
    const int base = W.base;
    cflgrid = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy, dtdz = dt / dz;
    const size_t n = (size_t)meqn * mitot * mjtot * mktot;
    for (double* f : {fm, fp, gm, gp, hm, hp}) std::fill(f, f + n, 0.0);
    auto fa = [&](std::vector<double>& v, int m, int i) { return v[(m - 1) + (size_t)meqn * (i - base)]; };
    auto ga = [&](std::vector<double>& v, int m, int i, int side, int d) { return W.G(v, m, i, side, d); };
    auto loadaux = [&](int i, int ai, int j1, int k1, int which, int kk) {
      // which: 1,2,3 -> aux1, aux2, aux3 ; kk: 1..3
      std::vector<double>& dst = which == 1 ? W.aux1 : which == 2 ? W.aux2 : W.aux3;
      for (int ma = 1; ma <= maux; ++ma) dst[(ma - 1) + (size_t)W.maux * ((i - base) + (size_t)W.L * (kk - 1))] = A(ma, ai, j1, k1);
    };
    // x-sweeps
    for (int k = 0; k <= mz + 1; ++k)
      for (int j = 0; j <= my + 1; ++j) {
        for (int i = 1 - mbc; i <= mx + mbc; ++i)
          for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + (size_t)meqn * (i - base)] = Q(m, i, j, k);
        std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdx);
        if (maux > 0)
          for (int i = 1 - mbc; i <= mx + mbc; ++i) {
            loadaux(i, i, j - 1, k - 1, 1, 1); loadaux(i, i, j - 1, k, 1, 2); loadaux(i, i, j - 1, k + 1, 1, 3);
            loadaux(i, i, j, k - 1, 2, 1); loadaux(i, i, j, k, 2, 2); loadaux(i, i, j, k + 1, 2, 3);
            loadaux(i, i, j + 1, k - 1, 3, 1); loadaux(i, i, j + 1, k, 3, 2); loadaux(i, i, j + 1, k + 1, 3, 3);
          }
        double cfl1d;
        flux3(1, meqn, maux, mbc, mx, W, dtdy, dtdz, cfl1d);
        cflgrid = std::max(cflgrid, cfl1d);
        for (int i = 1; i <= mx + 1; ++i)
          for (int m = 1; m <= meqn; ++m) {
            F(fm, m, i, j, k) = F(fm, m, i, j, k) + fa(W.faddm, m, i);
            F(fp, m, i, j, k) = F(fp, m, i, j, k) + fa(W.faddp, m, i);
            for (int d = -1; d <= 1; ++d) {
              F(gm, m, i, j, k + d) = F(gm, m, i, j, k + d) + ga(W.gadd, m, i, 1, d);
              F(gp, m, i, j, k + d) = F(gp, m, i, j, k + d) + ga(W.gadd, m, i, 1, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(gm, m, i, j + 1, k + d) = F(gm, m, i, j + 1, k + d) + ga(W.gadd, m, i, 2, d);
              F(gp, m, i, j + 1, k + d) = F(gp, m, i, j + 1, k + d) + ga(W.gadd, m, i, 2, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(hm, m, i, j + d, k) = F(hm, m, i, j + d, k) + ga(W.hadd, m, i, 1, d);
              F(hp, m, i, j + d, k) = F(hp, m, i, j + d, k) + ga(W.hadd, m, i, 1, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(hm, m, i, j + d, k + 1) = F(hm, m, i, j + d, k + 1) + ga(W.hadd, m, i, 2, d);
              F(hp, m, i, j + d, k + 1) = F(hp, m, i, j + d, k + 1) + ga(W.hadd, m, i, 2, d);
            }
          }
      }
    // y-sweeps
    for (int k = 0; k <= mz + 1; ++k)
      for (int i = 0; i <= mx + 1; ++i) {
        for (int j = 1 - mbc; j <= my + mbc; ++j)
          for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + (size_t)meqn * (j - base)] = Q(m, i, j, k);
        std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdy);
        if (maux > 0)
          for (int j = 1 - mbc; j <= my + mbc; ++j) {
            loadaux(j, i - 1, j, k - 1, 1, 1); loadaux(j, i, j, k - 1, 1, 2); loadaux(j, i + 1, j, k - 1, 1, 3);
            loadaux(j, i - 1, j, k, 2, 1); loadaux(j, i, j, k, 2, 2); loadaux(j, i + 1, j, k, 2, 3);
            loadaux(j, i - 1, j, k + 1, 3, 1); loadaux(j, i, j, k + 1, 3, 2); loadaux(j, i + 1, j, k + 1, 3, 3);
          }
        double cfl1d;
        flux3(2, meqn, maux, mbc, my, W, dtdz, dtdx, cfl1d);
        cflgrid = std::max(cflgrid, cfl1d);
        for (int j = 1; j <= my + 1; ++j)
          for (int m = 1; m <= meqn; ++m) {
            F(gm, m, i, j, k) = F(gm, m, i, j, k) + fa(W.faddm, m, j);
            F(gp, m, i, j, k) = F(gp, m, i, j, k) + fa(W.faddp, m, j);
            for (int d = -1; d <= 1; ++d) {
              F(hm, m, i + d, j, k) = F(hm, m, i + d, j, k) + ga(W.gadd, m, j, 1, d);
              F(hp, m, i + d, j, k) = F(hp, m, i + d, j, k) + ga(W.gadd, m, j, 1, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(hm, m, i + d, j, k + 1) = F(hm, m, i + d, j, k + 1) + ga(W.gadd, m, j, 2, d);
              F(hp, m, i + d, j, k + 1) = F(hp, m, i + d, j, k + 1) + ga(W.gadd, m, j, 2, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(fm, m, i, j, k + d) = F(fm, m, i, j, k + d) + ga(W.hadd, m, j, 1, d);
              F(fp, m, i, j, k + d) = F(fp, m, i, j, k + d) + ga(W.hadd, m, j, 1, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(fm, m, i + 1, j, k + d) = F(fm, m, i + 1, j, k + d) + ga(W.hadd, m, j, 2, d);
              F(fp, m, i + 1, j, k + d) = F(fp, m, i + 1, j, k + d) + ga(W.hadd, m, j, 2, d);
            }
          }
      }
    // z-sweeps
    for (int j = 0; j <= my + 1; ++j)
      for (int i = 0; i <= mx + 1; ++i) {
        for (int k = 1 - mbc; k <= mz + mbc; ++k)
          for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + (size_t)meqn * (k - base)] = Q(m, i, j, k);
        std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdz);
        if (maux > 0)
          for (int k = 1 - mbc; k <= mz + mbc; ++k) {
            loadaux(k, i - 1, j - 1, k, 1, 1); loadaux(k, i - 1, j, k, 1, 2); loadaux(k, i - 1, j + 1, k, 1, 3);
            loadaux(k, i, j - 1, k, 2, 1); loadaux(k, i, j, k, 2, 2); loadaux(k, i, j + 1, k, 2, 3);
            loadaux(k, i + 1, j - 1, k, 3, 1); loadaux(k, i + 1, j, k, 3, 2); loadaux(k, i + 1, j + 1, k, 3, 3);
          }
        double cfl1d;
        flux3(3, meqn, maux, mbc, mz, W, dtdx, dtdy, cfl1d);
        cflgrid = std::max(cflgrid, cfl1d);
        for (int k = 1; k <= mz + 1; ++k)
          for (int m = 1; m <= meqn; ++m) {
            F(hm, m, i, j, k) = F(hm, m, i, j, k) + fa(W.faddm, m, k);
            F(hp, m, i, j, k) = F(hp, m, i, j, k) + fa(W.faddp, m, k);
            for (int d = -1; d <= 1; ++d) {
              F(fm, m, i, j + d, k) = F(fm, m, i, j + d, k) + ga(W.gadd, m, k, 1, d);
              F(fp, m, i, j + d, k) = F(fp, m, i, j + d, k) + ga(W.gadd, m, k, 1, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(fm, m, i + 1, j + d, k) = F(fm, m, i + 1, j + d, k) + ga(W.gadd, m, k, 2, d);
              F(fp, m, i + 1, j + d, k) = F(fp, m, i + 1, j + d, k) + ga(W.gadd, m, k, 2, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(gm, m, i + d, j, k) = F(gm, m, i + d, j, k) + ga(W.hadd, m, k, 1, d);
              F(gp, m, i + d, j, k) = F(gp, m, i + d, j, k) + ga(W.hadd, m, k, 1, d);
            }
            for (int d = -1; d <= 1; ++d) {
              F(gm, m, i + d, j + 1, k) = F(gm, m, i + d, j + 1, k) + ga(W.hadd, m, k, 2, d);
              F(gp, m, i + d, j + 1, k) = F(gp, m, i + d, j + 1, k) + ga(W.hadd, m, k, 2, d);
            }
          }
      }
  }

  // flux3_dimSplit.f:4-260: the normal fluctuations, limiter and second-order correction of
  // one pencil, without transverse terms: faddm = amdq, faddp = -apdq, both + cqxx
  void flux3_dimSplit(int ixyz, int meqn, int mbc, int mx, Pencil& W, double& cfl1d) {
    const int base = W.base;
    Slice q1d = W.sl(W.q1d);
    auto dtdx1d = [&](int i) -> double { return W.dtdx1d[i - base]; };
    Slice aux2c{W.aux2.data() + (size_t)W.maux * W.L, W.maux, base};  // aux2(:, :, 2): the pencil's own aux
    Slice faddm = W.sl(W.faddm), faddp = W.sl(W.faddp);
    Waves wave{W.wave.data(), meqn, mwaves, base};
    Slice s{W.s.data(), mwaves, base};
    bool limit = false;
    for (int mw = 1; mw <= mwaves; ++mw) if (mthlim[mw - 1] > 0) limit = true;
    for (int m = 1; m <= meqn; ++m)
      for (int i = 1 - mbc; i <= mx + mbc; ++i) { faddm(m, i) = 0.0; faddp(m, i) = 0.0; }
    // rpn3 writes amdq into faddm and apdq into faddp (flux3_dimSplit.f:150-160)
    rpn3(prob, ixyz, meqn, mwaves, mbc, mx, q1d, q1d, aux2c, aux2c, wave, s, faddm, faddp);
    for (int i = 1; i <= mx + 1; ++i)
      for (int m = 1; m <= meqn; ++m) faddp(m, i) = -faddp(m, i);
    cfl1d = 0.0;
    for (int mw = 1; mw <= mwaves; ++mw)
      for (int i = 1; i <= mx + 1; ++i)
        cfl1d = std::max(cfl1d, std::max(dtdx1d(i) * s(mw, i), -dtdx1d(i - 1) * s(mw, i)));
    if (method[2] == 1) return;
    if (limit) limiter(meqn, mx, wave, s);
    for (int i = 1; i <= mx + 1; ++i) {
      const double dtdxave = 0.5 * (dtdx1d(i - 1) + dtdx1d(i));
      for (int m = 1; m <= meqn; ++m) {
        double cqxx = 0.0;
        for (int mw = 1; mw <= mwaves; ++mw) {
          const double sg = use_fwaves ? dsign(1.0, s(mw, i)) : std::fabs(s(mw, i));
          cqxx = cqxx + 0.5 * sg * (1.0 - std::fabs(s(mw, i)) * dtdxave) * wave(m, mw, i);
        }
        faddm(m, i) = faddm(m, i) + cqxx;
        faddp(m, i) = faddp(m, i) + cqxx;
      }
    }
  }

  // stepgrid_dimSplit.f:4-264 with step3x.f / step3y.f / step3z.f: Godunov splitting. x-sweeps
  // over every (j, k) pencil of the enlarged patch and the x-update of their interior cells;
  // y-sweeps over the interior i, every k, of the x-updated values and the y-update of the
  // interior j; z-sweeps over the interior (i, j) and the z-update of the interior cells.
  void stepgrid_dimSplit(double* q, double* fm, double* fp, double* gm, double* gp, double* hm, double* hp, int mitot,
                         int mjtot, int mktot, double dt, double& dtnew, double dx, double dy, double dz, const double* aux,
                         double& cflgrid_out) {
    const int mbc = nghost, meqn = nvar, maux = naux;
    const int mx = mitot - 2 * mbc, my = mjtot - 2 * mbc, mz = mktot - 2 * mbc;
    const int maxm = std::max(mx, std::max(my, mz));
    auto at = [&](int i, int j, int k) { return (size_t)(i + mbc - 1) + (size_t)mitot * ((size_t)(j + mbc - 1) + (size_t)mjtot * (k + mbc - 1)); };
    auto Q = [&](int m, int i, int j, int k) -> double& { return q[(m - 1) + (size_t)meqn * at(i, j, k)]; };
    auto A = [&](int m, int i, int j, int k) { return aux[(m - 1) + (size_t)maux * at(i, j, k)]; };
    auto F = [&](double* f, int m, int i, int j, int k) -> double& { return f[(m - 1) + (size_t)meqn * at(i, j, k)]; };
    Pencil W;
    W.init(maxm, mbc, meqn, mwaves, maux);
    const int base = W.base;
    auto fa = [&](std::vector<double>& v, int m, int i) { return v[(m - 1) + (size_t)meqn * (i - base)]; };
    auto pencil_in = [&](int n, double dtdn, auto qat, auto aat) {
      for (int x = 1 - mbc; x <= n + mbc; ++x)
        for (int m = 1; m <= meqn; ++m) W.q1d[(m - 1) + (size_t)meqn * (x - base)] = qat(m, x);
      std::fill(W.dtdx1d.begin(), W.dtdx1d.end(), dtdn);
      if (maux > 0)
        for (int x = 1 - mbc; x <= n + mbc; ++x)
          for (int ma = 1; ma <= maux; ++ma) W.aux2[(ma - 1) + (size_t)W.maux * ((x - base) + (size_t)W.L)] = aat(ma, x);
    };
    const size_t nf = (size_t)meqn * mitot * mjtot * mktot;
    double cfl_grid = 0.0;
    const double dtdx = dt / dx, dtdy = dt / dy, dtdz = dt / dz;
    // step3x.f
    std::fill(fm, fm + nf, 0.0); std::fill(fp, fp + nf, 0.0);
    double cflx = 0.0;
    for (int k = 1 - mbc; k <= mz + mbc; ++k)
      for (int j = 1 - mbc; j <= my + mbc; ++j) {
        pencil_in(mx, dtdx, [&](int m, int x) { return Q(m, x, j, k); }, [&](int ma, int x) { return A(ma, x, j, k); });
        double cfl1d;
        flux3_dimSplit(1, meqn, mbc, mx, W, cfl1d);
        cflx = std::max(cflx, cfl1d);
        for (int i = 1; i <= mx + 1; ++i)
          for (int m = 1; m <= meqn; ++m) {
            F(fm, m, i, j, k) = F(fm, m, i, j, k) + fa(W.faddm, m, i);
            F(fp, m, i, j, k) = F(fp, m, i, j, k) + fa(W.faddp, m, i);
          }
      }
    cfl_grid = std::max(cfl_grid, cflx);
    for (int k = 1 - mbc; k <= mz + mbc; ++k)
      for (int j = 1 - mbc; j <= my + mbc; ++j)
        for (int i = 1; i <= mx; ++i)
          for (int m = 1; m <= meqn; ++m) Q(m, i, j, k) = Q(m, i, j, k) - dtdx * (F(fm, m, i + 1, j, k) - F(fp, m, i, j, k));
    // step3y.f
    std::fill(gm, gm + nf, 0.0); std::fill(gp, gp + nf, 0.0);
    double cfly = 0.0;
    for (int k = 1 - mbc; k <= mz + mbc; ++k)
      for (int i = 1; i <= mx; ++i) {
        pencil_in(my, dtdy, [&](int m, int x) { return Q(m, i, x, k); }, [&](int ma, int x) { return A(ma, i, x, k); });
        double cfl1d;
        flux3_dimSplit(2, meqn, mbc, my, W, cfl1d);
        cfly = std::max(cfly, cfl1d);
        for (int j = 1; j <= my + 1; ++j)
          for (int m = 1; m <= meqn; ++m) {
            F(gm, m, i, j, k) = F(gm, m, i, j, k) + fa(W.faddm, m, j);
            F(gp, m, i, j, k) = F(gp, m, i, j, k) + fa(W.faddp, m, j);
          }
      }
    cfl_grid = std::max(cfl_grid, cfly);
    for (int k = 1 - mbc; k <= mz + mbc; ++k)
      for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i)
          for (int m = 1; m <= meqn; ++m) Q(m, i, j, k) = Q(m, i, j, k) - dtdy * (F(gm, m, i, j + 1, k) - F(gp, m, i, j, k));
    // step3z.f
    std::fill(hm, hm + nf, 0.0); std::fill(hp, hp + nf, 0.0);
    double cflz = 0.0;
    for (int j = 1; j <= my; ++j)
      for (int i = 1; i <= mx; ++i) {
        pencil_in(mz, dtdz, [&](int m, int x) { return Q(m, i, j, x); }, [&](int ma, int x) { return A(ma, i, j, x); });
        double cfl1d;
        flux3_dimSplit(3, meqn, mbc, mz, W, cfl1d);
        cflz = std::max(cflz, cfl1d);
        for (int k = 1; k <= mz + 1; ++k)
          for (int m = 1; m <= meqn; ++m) {
            F(hm, m, i, j, k) = F(hm, m, i, j, k) + fa(W.faddm, m, k);
            F(hp, m, i, j, k) = F(hp, m, i, j, k) + fa(W.faddp, m, k);
          }
      }
    cfl_grid = std::max(cfl_grid, cflz);
    for (int k = 1; k <= mz; ++k)
      for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i)
          for (int m = 1; m <= meqn; ++m) Q(m, i, j, k) = Q(m, i, j, k) - dtdz * (F(hm, m, i, j, k + 1) - F(hp, m, i, j, k));
    cflgrid_out = cfl_grid;
    if (cfl_grid > 0.0) dtnew = dt * cfl / cfl_grid;
    else dtnew = RINFINITY3;
  }

  // stepgrid.f:4-236 ; returns dtnew through the argument and the grid's Courant number
  void stepgrid(double* q, double* fm, double* fp, double* gm, double* gp, double* hm, double* hp, int mitot, int mjtot,
                int mktot, double dt, double& dtnew, double dx, double dy, double dz, const double* aux, double& cflgrid) {
    const int mbc = nghost;
    const int mx = mitot - 2 * mbc, my = mjtot - 2 * mbc, mz = mktot - 2 * mbc;
    step3(mx, my, mz, q, aux, dx, dy, dz, dt, cflgrid, fm, fp, gm, gp, hm, hp);
    const double dtdx = dt / dx, dtdy = dt / dy, dtdz = dt / dz;
    FArr3 Q{q, nvar, mitot, mjtot, mktot}, FM{fm, nvar, mitot, mjtot, mktot}, FP{fp, nvar, mitot, mjtot, mktot};
    FArr3 GM{gm, nvar, mitot, mjtot, mktot}, GP{gp, nvar, mitot, mjtot, mktot}, HM{hm, nvar, mitot, mjtot, mktot},
        HP{hp, nvar, mitot, mjtot, mktot};
    for (int k = mbc + 1; k <= mktot - mbc; ++k)
      for (int j = mbc + 1; j <= mjtot - mbc; ++j)
        for (int i = mbc + 1; i <= mitot - mbc; ++i)
          for (int m = 1; m <= nvar; ++m)
            Q(m, i, j, k) = Q(m, i, j, k) - dtdx * (FM(m, i + 1, j, k) - FP(m, i, j, k)) - dtdy * (GM(m, i, j + 1, k) - GP(m, i, j, k)) -
                            dtdz * (HM(m, i, j, k + 1) - HP(m, i, j, k));
    if (cflgrid > 0.0) dtnew = dt * cfl / cflgrid;
    else dtnew = RINFINITY3;
  }

  // ===================================================== ghost cells: bc3amr.f90:70-380
  void bc3amr(double* valp, int nrow, int ncol, int nfil, double hx, double hy, double hz, double xlo_p, double xhi_p,
              double ylo_p, double yhi_p, double zlo_p, double zhi_p) {
    FArr3 val{valp, nvar, nrow, ncol, nfil};
    const double hxmarg = hx * 0.01, hymarg = hy * 0.01, hzmarg = hz * 0.01;
    if (xperdom && yperdom && zperdom) return;
    auto chk = [&](int code) { if (code == 0) throw std::runtime_error("user boundary conditions are not provided"); };
    if (xlo_p < xlower - hxmarg) {
      const int nxl = (int)((xlower + hxmarg - xlo_p) / hx);
      chk(mthbc[1]);
      if (mthbc[1] == 1 || mthbc[1] == 3) {
        for (int k = 1; k <= nfil; ++k) for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nxl; ++i)
          for (int m = 1; m <= nvar; ++m) val(m, i, j, k) = val(m, mthbc[1] == 1 ? nxl + 1 : 2 * nxl + 1 - i, j, k);
        if (mthbc[1] == 3)
          for (int k = 1; k <= nfil; ++k) for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nxl; ++i) val(2, i, j, k) = -val(2, i, j, k);
      }
    }
    if (xhi_p > xupper + hxmarg) {
      const int nxr = (int)((xhi_p - xupper + hxmarg) / hx);
      const int ibeg = std::max(nrow - nxr + 1, 1);
      chk(mthbc[2]);
      if (mthbc[2] == 1 || mthbc[2] == 3) {
        for (int k = 1; k <= nfil; ++k) for (int i = ibeg; i <= nrow; ++i) for (int j = 1; j <= ncol; ++j)
          for (int m = 1; m <= nvar; ++m) val(m, i, j, k) = val(m, mthbc[2] == 1 ? ibeg - 1 : 2 * ibeg - 1 - i, j, k);
        if (mthbc[2] == 3)
          for (int k = 1; k <= nfil; ++k) for (int i = ibeg; i <= nrow; ++i) for (int j = 1; j <= ncol; ++j) val(2, i, j, k) = -val(2, i, j, k);
      }
    }
    if (ylo_p < ylower - hymarg) {
      const int nyl = (int)((ylower + hymarg - ylo_p) / hy);
      chk(mthbc[3]);
      if (mthbc[3] == 1 || mthbc[3] == 3) {
        for (int k = 1; k <= nfil; ++k) for (int j = 1; j <= nyl; ++j) for (int i = 1; i <= nrow; ++i)
          for (int m = 1; m <= nvar; ++m) val(m, i, j, k) = val(m, i, mthbc[3] == 1 ? nyl + 1 : 2 * nyl + 1 - j, k);
        if (mthbc[3] == 3)
          for (int k = 1; k <= nfil; ++k) for (int j = 1; j <= nyl; ++j) for (int i = 1; i <= nrow; ++i) val(3, i, j, k) = -val(3, i, j, k);
      }
    }
    if (yhi_p > yupper + hymarg) {
      const int nyr = (int)((yhi_p - yupper + hymarg) / hy);
      const int jbeg = std::max(ncol - nyr + 1, 1);
      chk(mthbc[4]);
      if (mthbc[4] == 1 || mthbc[4] == 3) {
        for (int k = 1; k <= nfil; ++k) for (int j = jbeg; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i)
          for (int m = 1; m <= nvar; ++m) val(m, i, j, k) = val(m, i, mthbc[4] == 1 ? jbeg - 1 : 2 * jbeg - 1 - j, k);
        if (mthbc[4] == 3)
          for (int k = 1; k <= nfil; ++k) for (int j = jbeg; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i) val(3, i, j, k) = -val(3, i, j, k);
      }
    }
    if (zlo_p < zlower - hzmarg) {
      const int nzl = (int)((zlower + hzmarg - zlo_p) / hz);
      chk(mthbc[5]);
      if (mthbc[5] == 1 || mthbc[5] == 3) {
        for (int k = 1; k <= nzl; ++k) for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i)
          for (int m = 1; m <= nvar; ++m) val(m, i, j, k) = val(m, i, j, mthbc[5] == 1 ? nzl + 1 : 2 * nzl + 1 - k);
        if (mthbc[5] == 3)
          for (int k = 1; k <= nzl; ++k) for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i) val(4, i, j, k) = -val(4, i, j, k);
      }
    }
    if (zhi_p > zupper + hzmarg) {
      const int nzr = (int)((zhi_p - zupper + hzmarg) / hz);
      const int kbeg = std::max(nfil - nzr + 1, 1);
      chk(mthbc[6]);
      if (mthbc[6] == 1 || mthbc[6] == 3) {
        for (int k = kbeg; k <= nfil; ++k) for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i)
          for (int m = 1; m <= nvar; ++m) val(m, i, j, k) = val(m, i, j, mthbc[6] == 1 ? kbeg - 1 : 2 * kbeg - 1 - k);
        if (mthbc[6] == 3)
          for (int k = kbeg; k <= nfil; ++k) for (int j = 1; j <= ncol; ++j) for (int i = 1; i <= nrow; ++i) val(4, i, j, k) = -val(4, i, j, k);
      }
    }
  }

  // ===================================================== ghost cells: intfil.f:4-263
  // flaguse is (ilo:ihi, jlo:jhi, klo:khi)
  void intfil(double* valp, int mi, int mj, int mk, double t, std::vector<signed char>& flaguse, int nrowst, int ncolst,
              int nfilst, int ilo, int ihi, int jlo, int jhi, int klo, int khi, int level, int msrc) {
    FArr3 val{valp, nvar, mi, mj, mk};
    const int nrow = ihi - ilo + 1, ncol = jhi - jlo + 1, nfil = khi - klo + 1;
    auto FU = [&](int i, int j, int k) -> signed char& { return flaguse[(size_t)(i - ilo) + (size_t)nrow * ((j - jlo) + (size_t)ncol * (k - klo))]; };
    const double dt = possk[level];
    const double teps = dt / 10.0;
    flaguse.assign((size_t)nrow * ncol * nfil, 0);
    const std::vector<int>& src = (msrc == -1) ? levelgrids[level] : node[msrc].bnd;
    for (int mptr : src) {
      const Node3& g = node[mptr];
      const int mitot = mitot_of(mptr), mjtot = mjtot_of(mptr);
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi);
      const int jxlo = std::max(g.jlo, jlo), jxhi = std::min(g.jhi, jhi);
      const int kxlo = std::max(g.klo, klo), kxhi = std::min(g.khi, khi);
      if (!((ixlo <= ixhi && jxlo <= jxhi) && (kxlo <= kxhi))) continue;
      const double alphac = (g.time - t) / dt;
      const double alphai = 1.0 - alphac;
      if (alphai < -teps || alphai > 1.0 + teps) throw std::runtime_error("intfil: time not available");
      const double* s1 = nullptr;
      const double* s2 = nullptr;
      bool tint = false;
      if (std::fabs(alphai - 1.0) < teps) s1 = g.q1.data();
      else if (std::fabs(alphai) < teps) {
        if (level == mxnest) throw std::runtime_error("intfil: old time on finest level");
        s1 = g.q2.data();
      } else {
        if (level == mxnest) throw std::runtime_error("intfil: time interpolation on finest level");
        s1 = g.q1.data(); s2 = g.q2.data(); tint = true;
      }
      auto idx = [&](int ivar, int i, int j, int k) { return (size_t)(ivar - 1) + (size_t)nvar * ((size_t)(i - 1) + (size_t)mitot * ((size_t)(j - 1) + (size_t)mjtot * (k - 1))); };
      for (int k = kxlo; k <= kxhi; ++k)
        for (int j = jxlo; j <= jxhi; ++j)
          for (int i = ixlo; i <= ixhi; ++i) {
            for (int ivar = 1; ivar <= nvar; ++ivar) {
              const size_t a = idx(ivar, i - g.ilo + nghost + 1, j - g.jlo + nghost + 1, k - g.klo + nghost + 1);
              if (!tint) val(ivar, i - ilo + nrowst, j - jlo + ncolst, k - klo + nfilst) = s1[a];
              else val(ivar, i - ilo + nrowst, j - jlo + ncolst, k - klo + nfilst) = s1[a] * alphai + s2[a] * alphac;
            }
            FU(i, j, k) = 1;
          }
    }
    if (khi >= kregsz[level])
      for (int k = std::max(kregsz[level], klo); k <= khi; ++k) for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) FU(i, j, k) = 1;
    if (klo < 0) {
      const int nfilend = nfilst + nfil - 1;
      for (int k = klo; k <= std::min(std::min(-1, nfilend), khi); ++k) for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) FU(i, j, k) = 1;
    }
    if (jhi >= jregsz[level])
      for (int k = klo; k <= khi; ++k) for (int j = std::max(jregsz[level], jlo); j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) FU(i, j, k) = 1;
    if (jlo < 0) {
      const int ncolend = ncolst + ncol - 1;
      for (int k = klo; k <= khi; ++k) for (int j = jlo; j <= std::min(std::min(-1, ncolend), jhi); ++j) for (int i = ilo; i <= ihi; ++i) FU(i, j, k) = 1;
    }
    if (ilo < 0) {
      const int nrowend = nrowst + nrow - 1;
      for (int k = klo; k <= khi; ++k) for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= std::min(std::min(-1, nrowend), ihi); ++i) FU(i, j, k) = 1;
    }
    if (ihi >= iregsz[level])
      for (int k = klo; k <= khi; ++k) for (int j = jlo; j <= jhi; ++j) for (int i = std::max(iregsz[level], ilo); i <= ihi; ++i) FU(i, j, k) = 1;
  }

  // trimbd.f:4-99: bounding box (absolute indices) of the cells not yet set
  void trimbd(const std::vector<signed char>& used, bool& set, int& il, int& ir, int& jl, int& jr, int& kl, int& kr,
              int ilo, int ihi, int jlo, int jhi, int klo, int khi) {
    const int nrow = ihi - ilo + 1, ncol = jhi - jlo + 1;
    auto U = [&](int i, int j, int k) { return (int)used[(size_t)(i - ilo) + (size_t)nrow * ((j - jlo) + (size_t)ncol * (k - klo))]; };
    long utot = 0;
    for (int k = klo; k <= khi; ++k) for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) utot += U(i, j, k);
    if (utot >= (long)nrow * ncol * (khi - klo + 1)) { set = true; return; }
    set = false;
    int u = 1;
    for (int i = ilo; i <= ihi; ++i) { for (int k = klo; k <= khi; ++k) for (int j = jlo; j <= jhi; ++j) u = std::min(u, U(i, j, k)); il = i; if (u == 0) break; }
    u = 1;
    for (int i = ihi; i >= ilo; --i) { for (int k = klo; k <= khi; ++k) for (int j = jlo; j <= jhi; ++j) u = std::min(u, U(i, j, k)); ir = i; if (u == 0) break; }
    u = 1;
    for (int j = jlo; j <= jhi; ++j) { for (int k = klo; k <= khi; ++k) for (int i = ilo; i <= ihi; ++i) u = std::min(u, U(i, j, k)); jl = j; if (u == 0) break; }
    u = 1;
    for (int j = jhi; j >= jlo; --j) { for (int k = klo; k <= khi; ++k) for (int i = ilo; i <= ihi; ++i) u = std::min(u, U(i, j, k)); jr = j; if (u == 0) break; }
    u = 1;
    for (int k = klo; k <= khi; ++k) { for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) u = std::min(u, U(i, j, k)); kl = k; if (u == 0) break; }
    u = 1;
    for (int k = khi; k >= klo; --k) { for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i) u = std::min(u, U(i, j, k)); kr = k; if (u == 0) break; }
  }

  // filpatch.f:4-282 (filrecur)
  void filrecur(int level, double* valbig, int mitot, int mjtot, int mktot, double t, int nrowst, int ncolst, int nfilst,
                int ilo, int ihi, int jlo, int jhi, int klo, int khi, bool patchOnly, int msrc) {
    const double hxf = hxposs[level], hyf = hyposs[level], hzf = hzposs[level];
    const double xlp = xlower + (double)ilo * hxf, xrp = xlower + (double)(ihi + 1) * hxf;
    const double ybp = ylower + (double)jlo * hyf, ytp = ylower + (double)(jhi + 1) * hyf;
    const double zfp = zlower + (double)klo * hzf, zrp = zlower + (double)(khi + 1) * hzf;
    const int nrowp = ihi - ilo + 1, ncolp = jhi - jlo + 1, nfilp = khi - klo + 1;
    std::vector<signed char> flaguse;
    intfil(valbig, mitot, mjtot, mktot, t, flaguse, nrowst, ncolst, nfilst, ilo, ihi, jlo, jhi, klo, khi, level, msrc);
    bool set;
    int il = 0, ir = 0, jl = 0, jr = 0, kl = 0, kr = 0;
    trimbd(flaguse, set, il, ir, jl, jr, kl, kr, ilo, ihi, jlo, jhi, klo, khi);
    if (!set) {
      if (level == 1) throw std::runtime_error("filrecur: level 1 cells not covered");
      const int levc = level - 1;
      const double hxc = hxposs[levc], hyc = hyposs[levc], hzc = hzposs[levc];
      const int rx = intratx[levc], ry = intraty[levc], rz = intratz[levc];
      const int iplo = (il - rx + nghost * rx) / rx - nghost, jplo = (jl - ry + nghost * ry) / ry - nghost, kplo = (kl - rz + nghost * rz) / rz - nghost;
      const int iphi = (ir + rx) / rx, jphi = (jr + ry) / ry, kphi = (kr + rz) / rz;
      const double xlc = xlower + iplo * hxc, ybc = ylower + jplo * hyc, zfc = zlower + kplo * hzc;
      const int nrowc = iphi - iplo + 1, ncolc = jphi - jplo + 1, nfilc = kphi - kplo + 1;
      if (nrowc > ihi - ilo + 3 || ncolc > jhi - jlo + 3 || nfilc > khi - klo + 3) throw std::runtime_error("filrecur: coarse box too large");
      std::vector<double> valcrse((size_t)nrowc * ncolc * nfilc * nvar, 0.0);
      // filpatch.f:168-179: a coarse box that leaves a periodic domain is filled by prefilrecur
      const bool sticks = iplo < 0 || jplo < 0 || kplo < 0 || iphi >= iregsz[levc] || jphi >= jregsz[levc] || kphi >= kregsz[levc];
      if ((xperdom || yperdom || zperdom) && sticks)
        prefilrecur(levc, valcrse.data(), nrowc, ncolc, nfilc, t, 1, 1, 1, iplo, iphi, jplo, jphi, kplo, kphi, iplo, jplo, kplo);
      else
        filrecur(levc, valcrse.data(), nrowc, ncolc, nfilc, t, 1, 1, 1, iplo, iphi, jplo, jphi, kplo, kphi, true, -1);
      FArr3 VC{valcrse.data(), nvar, nrowc, ncolc, nfilc};
      FArr3 VB{valbig, nvar, mitot, mjtot, mktot};
      const double ratiox = (double)(float)rx, ratioy = (double)(float)ry, ratioz = (double)(float)rz;
      const int nr0 = ihi - ilo + 1, nc0 = jhi - jlo + 1;
      for (int iff = 1; iff <= nrowp; ++iff) {
        const int ic = (int)std::floor((iff + ilo - 1) / ratiox) - iplo + 1;
        const double xcent_coarse = xlc + (ic - 0.5) * hxc;
        const double xcent_fine = xlower + (iff - 1 + ilo + 0.5) * hxf;
        const double eta1 = (xcent_fine - xcent_coarse) / hxc;
        for (int jf = 1; jf <= ncolp; ++jf) {
          const int jc = (int)std::floor((jf + jlo - 1) / ratioy) - jplo + 1;
          const double ycent_coarse = ybc + (jc - 0.5) * hyc;
          const double ycent_fine = ylower + (jf - 1 + jlo + 0.5) * hyf;
          const double eta2 = (ycent_fine - ycent_coarse) / hyc;
          for (int kf = 1; kf <= nfilp; ++kf) {
            const int kc = (int)std::floor((kf + klo - 1) / ratioz) - kplo + 1;
            const double zcent_coarse = zfc + (kc - 0.5) * hzc;
            const double zcent_fine = zlower + (kf - 1 + klo + 0.5) * hzf;
            const double eta3 = (zcent_fine - zcent_coarse) / hzc;
            if (flaguse[(size_t)(iff - 1) + (size_t)nr0 * ((jf - 1) + (size_t)nc0 * (kf - 1))] != 0) continue;
            for (int ivar = 1; ivar <= nvar; ++ivar) {
              const double valp100 = VC(ivar, ic + 1, jc, kc), valm100 = VC(ivar, ic - 1, jc, kc), valc = VC(ivar, ic, jc, kc);
              const double valp010 = VC(ivar, ic, jc + 1, kc), valm010 = VC(ivar, ic, jc - 1, kc);
              const double valp001 = VC(ivar, ic, jc, kc + 1), valm001 = VC(ivar, ic, jc, kc - 1);
              const double dupc = valp100 - valc, dumc = valc - valm100, ducc = valp100 - valm100;
              double du = std::min(std::fabs(dupc), std::fabs(dumc));
              du = std::min(2.0 * du, 0.5 * std::fabs(ducc));
              const double fu = std::max(0.0, dsign(1.0, dupc * dumc));
              const double uslope = du * dsign(1.0, ducc) * fu;
              const double dvpc = valp010 - valc, dvmc = valc - valm010, dvcc = valp010 - valm010;
              double dv = std::min(std::fabs(dvpc), std::fabs(dvmc));
              dv = std::min(2.0 * dv, 0.5 * std::fabs(dvcc));
              const double fv = std::max(0.0, dsign(1.0, dvpc * dvmc));
              const double vslope = dv * dsign(1.0, dvcc) * fv;
              const double dwpc = valp001 - valc, dwmc = valc - valm001, dwcc = valp001 - valm001;
              double dw = std::min(std::fabs(dwpc), std::fabs(dwmc));
              dw = std::min(2.0 * dw, 0.5 * std::fabs(dwcc));
              const double fw = std::max(0.0, dsign(1.0, dwpc * dwmc));
              const double wslope = dw * dsign(1.0, dwcc) * fw;
              VB(ivar, iff + nrowst - 1, jf + ncolst - 1, kf + nfilst - 1) = valc + eta1 * uslope + eta2 * vslope + eta3 * wslope;
            }
          }
        }
      }
    }
    if (patchOnly) bc3amr(valbig, mitot, mjtot, mktot, hxf, hyf, hzf, xlp, xrp, ybp, ytp, zfp, zrp);
  }

  // prefilp.f / preicall.f / preintcopy.f: the three index ranges of one direction (below
  // the domain, inside, above) and the shift that maps each into the domain when periodic
  void per_ranges(bool per, int lo, int hi, int n, int st[3], int en[3], int sh[3]) const {
    if (per) {
      st[0] = lo; st[1] = 0; st[2] = n; en[0] = -1; en[1] = n - 1; en[2] = hi; sh[0] = n; sh[1] = 0; sh[2] = -n;
    } else {
      st[0] = n; st[1] = lo; st[2] = n; en[0] = -1; en[1] = hi; en[2] = -1; sh[0] = sh[1] = sh[2] = 0;
    }
  }

  // prefilp.f:1-141 (prefilrecur): the patch [ilo,ihi]x[jlo,jhi]x[klo,khi] of level, split
  // into the 27 regions; each non-empty region is filled by filrecur on a scratch patch of
  // its own size at its periodically shifted place, then copied to valbig, whose array
  // starts at index (iglo, jglo, kglo) (patchCopyOut)
  void prefilrecur(int level, double* valbig, int mitot, int mjtot, int mktot, double t, int nrowst, int ncolst, int nfilst,
                   int ilo, int ihi, int jlo, int jhi, int klo, int khi, int iglo, int jglo, int kglo) {
    (void)nrowst; (void)ncolst; (void)nfilst;
    int ist[3], iend[3], ishift[3], jst[3], jend[3], jshift[3], kst[3], kend[3], kshift[3];
    per_ranges(xperdom, ilo, ihi, iregsz[level], ist, iend, ishift);
    per_ranges(yperdom, jlo, jhi, jregsz[level], jst, jend, jshift);
    per_ranges(zperdom, klo, khi, kregsz[level], kst, kend, kshift);
    FArr3 VB{valbig, nvar, mitot, mjtot, mktot};
    for (int i = 0; i < 3; ++i) {
      const int i1 = std::max(ilo, ist[i]), i2 = std::min(ihi, iend[i]);
      if (i1 > i2) continue;
      for (int j = 0; j < 3; ++j) {
        const int j1 = std::max(jlo, jst[j]), j2 = std::min(jhi, jend[j]);
        if (j1 > j2) continue;
        for (int k = 0; k < 3; ++k) {
          const int k1 = std::max(klo, kst[k]), k2 = std::min(khi, kend[k]);
          if (k1 > k2) continue;
          const int mi = i2 - i1 + 1, mj = j2 - j1 + 1, mk = k2 - k1 + 1;
          std::vector<double> vp((size_t)nvar * mi * mj * mk, 0.0);
          filrecur(level, vp.data(), mi, mj, mk, t, 1, 1, 1, i1 + ishift[i], i2 + ishift[i], j1 + jshift[j], j2 + jshift[j],
                   k1 + kshift[k], k2 + kshift[k], true, -1);
          FArr3 VP{vp.data(), nvar, mi, mj, mk};
          const int is = i1 - iglo, js = j1 - jglo, ks = k1 - kglo;
          for (int kk = 1; kk <= mk; ++kk)
            for (int jj = 1; jj <= mj; ++jj)
              for (int ii = 1; ii <= mi; ++ii)
                for (int m = 1; m <= nvar; ++m) VB(m, is + ii, js + jj, ks + kk) = VP(m, ii, jj, kk);
        }
      }
    }
  }

  // preicall.f:1-141 / preintcopy.f: icall over the 27 regions with periodic shifts, each
  // put at its place in val (iputst = i1 - ilo + 1)
  void preicall(double* val, double* aux, int nrow, int ncol, int nfil, int ilo, int ihi, int jlo, int jhi, int klo, int khi,
                int level) {
    int ist[3], iend[3], ishift[3], jst[3], jend[3], jshift[3], kst[3], kend[3], kshift[3];
    per_ranges(xperdom, ilo, ihi, iregsz[level], ist, iend, ishift);
    per_ranges(yperdom, jlo, jhi, jregsz[level], jst, jend, jshift);
    per_ranges(zperdom, klo, khi, kregsz[level], kst, kend, kshift);
    for (int i = 0; i < 3; ++i) {
      const int i1 = std::max(ilo, ist[i]), i2 = std::min(ihi, iend[i]);
      if (i1 > i2) continue;
      for (int j = 0; j < 3; ++j) {
        const int j1 = std::max(jlo, jst[j]), j2 = std::min(jhi, jend[j]);
        if (j1 > j2) continue;
        for (int k = 0; k < 3; ++k) {
          const int k1 = std::max(klo, kst[k]), k2 = std::min(khi, kend[k]);
          if (k1 > k2) continue;
          icall(val, aux, nrow, ncol, nfil, i1 + ishift[i], i2 + ishift[i], j1 + jshift[j], j2 + jshift[j], k1 + kshift[k],
                k2 + kshift[k], level, i1 - ilo + 1, j1 - jlo + 1, k1 - klo + 1);
        }
      }
    }
  }

  // bound.f:4-211: the six ghost slabs, each by prefilrecur where it leaves a periodic
  // domain (the tests of bound.f:60-199), else by filrecur; then bc3amr on the whole array
  void bound(double t, double* valbig, int mitot, int mjtot, int mktot, int mptr, int ng = -1) {
    const Node3& g = node[mptr];
    if (ng < 0) ng = nghost;
    const int lev = g.level;
    const double hx = hxposs[lev], hy = hyposs[lev], hz = hzposs[lev];
    const int iglo = g.ilo - ng, jglo = g.jlo - ng, kglo = g.klo - ng;
    auto slab = [&](bool per, int nrs, int ncs, int nfs, int i0, int i1, int j0, int j1, int k0, int k1) {
      if (per) prefilrecur(lev, valbig, mitot, mjtot, mktot, t, nrs, ncs, nfs, i0, i1, j0, j1, k0, k1, iglo, jglo, kglo);
      else filrecur(lev, valbig, mitot, mjtot, mktot, t, nrs, ncs, nfs, i0, i1, j0, j1, k0, k1, false, mptr);
    };
    const bool ystick = (g.ylo - ng * hy < ylower) || (g.yhi + ng * hy > yupper);
    const bool xstick = (g.xlo - ng * hx < xlower) || (g.xhi + ng * hx > xupper);
    // left, right (x), front, rear (y), bottom, top (z)
    slab((xperdom && g.xlo - ng * hx < xlower) || (yperdom && ystick), 1, 1, ng + 1, g.ilo - ng, g.ilo - 1, g.jlo - ng, g.jhi + ng,
         g.klo, g.khi);
    slab((xperdom && g.xhi + ng * hx > xupper) || (yperdom && ystick), mitot - ng + 1, 1, ng + 1, g.ihi + 1, g.ihi + ng, g.jlo - ng,
         g.jhi + ng, g.klo, g.khi);
    slab(yperdom && g.ylo - ng * hy < ylower, ng + 1, 1, ng + 1, g.ilo, g.ihi, g.jlo - ng, g.jlo - 1, g.klo, g.khi);
    slab(yperdom && g.yhi + ng * hy > yupper, ng + 1, mjtot - ng + 1, ng + 1, g.ilo, g.ihi, g.jhi + 1, g.jhi + ng, g.klo, g.khi);
    slab((zperdom && g.zlo - ng * hz < zlower) || (xperdom && xstick) || (yperdom && ystick), 1, 1, 1, g.ilo - ng, g.ihi + ng,
         g.jlo - ng, g.jhi + ng, g.klo - ng, g.klo - 1);
    slab((zperdom && g.zhi + ng * hz > zupper) || (xperdom && xstick) || (yperdom && ystick), 1, 1, mktot - ng + 1, g.ilo - ng,
         g.ihi + ng, g.jlo - ng, g.jhi + ng, g.khi + 1, g.khi + ng);
    bc3amr(valbig, mitot, mjtot, mktot, hx, hy, hz, g.xlo - ng * hx, g.xhi + ng * hx, g.ylo - ng * hy, g.yhi + ng * hy,
           g.zlo - ng * hz, g.zhi + ng * hz);
  }

  // icall.f:4-98 (with aux) and intcopy.f:4-72 (q only): store1 of every grid at level
  void icall(double* val, double* aux, int nrow, int ncol, int nfil, int ilo, int ihi, int jlo, int jhi, int klo, int khi,
             int level, int iputst, int jputst, int kputst) {
    FArr3 V{val, nvar, nrow, ncol, nfil};
    for (int mptr = lstart[level]; mptr != 0; mptr = node[mptr].levelptr) {
      const Node3& g = node[mptr];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi);
      const int jxlo = std::max(g.jlo, jlo), jxhi = std::min(g.jhi, jhi);
      const int kxlo = std::max(g.klo, klo), kxhi = std::min(g.khi, khi);
      if (!((ixlo <= ixhi && jxlo <= jxhi) && kxlo <= kxhi)) continue;
      const int mitot = mitot_of(mptr), mjtot = mjtot_of(mptr), mktot = mktot_of(mptr);
      FArr3 S{const_cast<double*>(g.q1.data()), nvar, mitot, mjtot, mktot};
      for (int k = kxlo; k <= kxhi; ++k)
        for (int j = jxlo; j <= jxhi; ++j)
          for (int i = ixlo; i <= ixhi; ++i) {
            for (int ivar = 1; ivar <= nvar; ++ivar)
              V(ivar, i - ilo + iputst, j - jlo + jputst, k - klo + kputst) = S(ivar, i - g.ilo + nghost + 1, j - g.jlo + nghost + 1, k - g.klo + nghost + 1);
            if (aux && naux > 0) {
              FArr3 SA{const_cast<double*>(g.aux.data()), naux, mitot, mjtot, mktot};
              FArr3 VA{aux, naux, nrow, ncol, nfil};
              for (int ia = 1; ia <= naux; ++ia)
                VA(ia, i - ilo + iputst, j - jlo + jputst, k - klo + kputst) = SA(ia, i - g.ilo + nghost + 1, j - g.jlo + nghost + 1, k - g.klo + nghost + 1);
            }
          }
    }
  }

  // ===================================================== conservation: saveqc.f:3-111 + cstore.f:4-96
  void saveqc(int level) {
    const int levc = level - 1;
    const double hxc = hxposs[levc], hyc = hyposs[levc], hzc = hzposs[levc];
    for (int mkid = lstart[level]; mkid != 0; mkid = node[mkid].levelptr) {
      Node3& K = node[mkid];
      const int nx = K.ihi - K.ilo + 1, ny = K.jhi - K.jlo + 1, nz = K.khi - K.klo + 1;
      const int ikeep = nx / intratx[levc], jkeep = ny / intraty[levc], kkeep = nz / intratz[levc];
      const int lenbc = 2 * (ikeep * jkeep + jkeep * kkeep + kkeep * ikeep);
      const int iclo = K.ilo / intratx[levc] - 1, jclo = K.jlo / intraty[levc] - 1, kclo = K.klo / intratz[levc] - 1;
      const int ichi = (K.ihi + 1) / intratx[levc], jchi = (K.jhi + 1) / intraty[levc], kchi = (K.khi + 1) / intratz[levc];
      const int nrow = ichi - iclo + 1, ncol = jchi - jclo + 1, nfil = kchi - kclo + 1;
      const double xl = K.xlo - hxc, yf = K.ylo - hyc, zb = K.zlo - hzc;
      const double xr = K.xhi + hxc, yr = K.yhi + hyc, zt = K.zhi + hzc;
      std::vector<double> tq((size_t)nrow * ncol * nfil * nvar, 0.0), ta((size_t)nrow * ncol * nfil * std::max(naux, 1), 0.0);
      const bool sticksout = (iclo < 0 || ichi == iregsz[levc] || jclo < 0 || jchi == jregsz[levc] || kclo < 0 || kchi == kregsz[levc]);
      // saveqc.f:78-91 takes the periodic copy only when all three directions are periodic;
      // with fewer it leaves the ring's cells beyond a periodic face unset (uninitialised
      // memory there, zero density here, and qad's Roe solve breaks). The copy is taken
      // whenever a direction is periodic: the same as the reference with all three
      // periodic or none, and defined with one or two. The aux keeps the reference's rule.
      const bool perdom3 = xperdom && yperdom && zperdom;
      if (sticksout && (xperdom || yperdom || zperdom))
        preicall(tq.data(), ta.data(), nrow, ncol, nfil, iclo, ichi, jclo, jchi, kclo, kchi, levc);
      else icall(tq.data(), ta.data(), nrow, ncol, nfil, iclo, ichi, jclo, jchi, kclo, kchi, levc, 1, 1, 1);
      if (naux > 0 && sticksout && !perdom3) setaux(0, nrow, ncol, nfil, xl, yf, zb, hxc, hyc, hzc, ta.data());
      bc3amr(tq.data(), nrow, ncol, nfil, hxc, hyc, hzc, xl, xr, yf, yr, zb, zt);
      // cstore: sides 1 (x left), 2 (y top), 3 (x right), 4 (y bottom), 5 (z bottom), 6 (z top)
      FArr3 QC{tq.data(), nvar, nrow, ncol, nfil};
      FArr3 AC{ta.data(), std::max(naux, 1), nrow, ncol, nfil};
      double* qc1d = K.ffl.data() + (size_t)nvar * lenbc;
      double* auxc1d = K.ffl.data() + (size_t)2 * nvar * lenbc;
      int index = 0;
      auto put = [&](int i, int j, int k) {
        for (int m = 1; m <= nvar; ++m) qc1d[(m - 1) + (size_t)nvar * index] = QC(m, i, j, k);
        for (int m = 1; m <= naux; ++m) auxc1d[(m - 1) + (size_t)naux * index] = AC(m, i, j, k);
        ++index;
      };
      for (int k = 2; k <= nfil - 1; ++k) for (int j = 2; j <= ncol - 1; ++j) put(1, j, k);
      for (int k = 2; k <= nfil - 1; ++k) for (int i = 2; i <= nrow - 1; ++i) put(i, ncol, k);
      for (int k = 2; k <= nfil - 1; ++k) for (int j = 2; j <= ncol - 1; ++j) put(nrow, j, k);
      for (int k = 2; k <= nfil - 1; ++k) for (int i = 2; i <= nrow - 1; ++i) put(i, 1, k);
      for (int j = 2; j <= ncol - 1; ++j) for (int i = 2; i <= nrow - 1; ++i) put(i, j, 1);
      for (int j = 2; j <= ncol - 1; ++j) for (int i = 2; i <= nrow - 1; ++i) put(i, j, nfil);
    }
  }

  // qad.f:4-534: Riemann problems between the fine ghost cells and the saved coarse values
  void qad(double* valbigp, const double* auxp, int mitot, int mjtot, int mktot, double* svdflx, const double* qc1d,
           const double* auxc1d, int lratiox, int lratioy, int lratioz, double hx, double hy, double hz, double delt) {
    FArr3 vb{valbigp, nvar, mitot, mjtot, mktot};
    const int maux = naux, ng = nghost;
    FArr3 ax{const_cast<double*>(auxp), std::max(maux, 1), mitot, mjtot, mktot};
    const int nf = mktot - 2 * ng, nc = mjtot - 2 * ng, nr = mitot - 2 * ng;
    (void)nf;
    const int ncrsek = nf / lratioz, ncrsej = nc / lratioy, ncrsei = nr / lratiox;
    (void)ncrsek;
    const int maxl = std::max(nr, std::max(nc, nf)) + 2;  // 1-based arrays up to max1d+1
    const int mbc = ng, base = 1 - mbc, L = maxl + 2 * mbc;
    std::vector<double> QLv((size_t)nvar * L, 0), QRv((size_t)nvar * L, 0), WV((size_t)nvar * mwaves * L, 0), SV((size_t)mwaves * L, 0),
        AMv((size_t)nvar * L, 0), APv((size_t)nvar * L, 0), ALv((size_t)std::max(maux, 1) * L, 0), ARv((size_t)std::max(maux, 1) * L, 0);
    // qad's arrays are 1-based (1..max1d+1); the solvers index them from 1-mbc: shift by mbc
    auto ql = [&](int m, int i) -> double& { return QLv[(m - 1) + (size_t)nvar * (i - 1)]; };
    auto qr = [&](int m, int i) -> double& { return QRv[(m - 1) + (size_t)nvar * (i - 1)]; };
    auto al = [&](int m, int i) -> double& { return ALv[(m - 1) + (size_t)std::max(maux, 1) * (i - 1)]; };
    auto ar = [&](int m, int i) -> double& { return ARv[(m - 1) + (size_t)std::max(maux, 1) * (i - 1)]; };
    Slice QL{QLv.data(), nvar, base}, QR{QRv.data(), nvar, base}, AL{ALv.data(), std::max(maux, 1), base}, AR{ARv.data(), std::max(maux, 1), base};
    Waves W{WV.data(), nvar, mwaves, base};
    Slice S{SV.data(), mwaves, base}, AM{AMv.data(), nvar, base}, AP{APv.data(), nvar, base};
    auto amdq = [&](int m, int i) { return AMv[(m - 1) + (size_t)nvar * (i - 1)]; };
    auto apdq = [&](int m, int i) { return APv[(m - 1) + (size_t)nvar * (i - 1)]; };
    auto qc = [&](int m, int idx) { return qc1d[(m - 1) + (size_t)nvar * (idx - 1)]; };
    auto acd = [&](int m, int idx) { return auxc1d[(m - 1) + (size_t)maux * (idx - 1)]; };
    auto sv = [&](int m, int idx) -> double& { return svdflx[(m - 1) + (size_t)nvar * (idx - 1)]; };
    auto is_type = [&](int ma, const char* t) { return auxtype[ma - 1] == t; };
    int index0 = 0, influx0 = 0;
    // side 1 (x left)
    for (int k = ng + 1; k <= mktot - ng; ++k) {
      const int kc = 1 + (k - (ng + 1)) / lratioz, kcnext = 1 + (k + 1 - (ng + 1)) / lratioz;
      int indaux = 1;
      for (int j = ng + 1; j <= mjtot - ng; ++j) {
        indaux = indaux + 1;
        for (int ma = 1; ma <= maux; ++ma) al(ma, indaux) = is_type(ma, "xleft") ? ax(ma, ng + 1, j, k) : ax(ma, ng, j, k);
        for (int m = 1; m <= nvar; ++m) ql(m, indaux) = vb(m, ng, j, k);
      }
      int lind = 0, index = index0;
      for (int jc = 1; jc <= ncrsej; ++jc) {
        index = index + 1;
        for (int l = 1; l <= lratioy; ++l) {
          lind = lind + 1;
          for (int ma = 1; ma <= maux; ++ma) ar(ma, lind) = acd(ma, index);
          for (int m = 1; m <= nvar; ++m) qr(m, lind) = qc(m, index);
        }
      }
      if (kcnext != kc) index0 = index;
      rpn3(prob, 1, nvar, mwaves, mbc, nc + 1 - 2 * ng, QL, QR, AL, AR, W, S, AM, AP);
      int influx = influx0;
      for (int j = 1; j <= nc / lratioy; ++j) {
        influx = influx + 1;
        const int indexa = (j - 1) * lratioy + 1;
        for (int m = 1; m <= nvar; ++m)
          for (int l = 1; l <= lratioy; ++l)
            sv(m, influx) = sv(m, influx) + amdq(m, indexa + l) * hy * hz * delt + apdq(m, indexa + l) * hy * hz * delt;
      }
      if (kcnext != kc) influx0 = influx;
    }
    // side 2 (y top)
    for (int k = ng + 1; k <= mktot - ng; ++k) {
      const int kc = 1 + (k - (ng + 1)) / lratioz, kcnext = 1 + (k + 1 - (ng + 1)) / lratioz;
      int indaux = 0;
      for (int i = ng + 1; i <= mitot - ng; ++i) {
        indaux = indaux + 1;
        for (int ma = 1; ma <= maux; ++ma) ar(ma, indaux) = ax(ma, i, mjtot - ng + 1, k);
        for (int m = 1; m <= nvar; ++m) qr(m, indaux) = vb(m, i, mjtot - ng + 1, k);
      }
      int lind = 0, index = index0;
      for (int ic = 1; ic <= ncrsei; ++ic) {
        index = index + 1;
        for (int l = 1; l <= lratiox; ++l) {
          lind = lind + 1;
          for (int ma = 1; ma <= maux; ++ma) {
            if (is_type(ma, "yleft")) {
              const int kfine = (kc - 1) * lratioz + ng + l, ifine = (ic - 1) * lratiox + ng + l;
              al(ma, lind + 1) = ax(ma, ifine, mjtot - ng + 1, kfine);
            } else al(ma, lind + 1) = acd(ma, index);
          }
          for (int m = 1; m <= nvar; ++m) ql(m, lind + 1) = qc(m, index);
        }
      }
      if (kcnext != kc) index0 = index;
      rpn3(prob, 2, nvar, mwaves, mbc, nr + 1 - 2 * ng, QL, QR, AL, AR, W, S, AM, AP);
      int influx = influx0;
      for (int i = 1; i <= nr / lratiox; ++i) {
        influx = influx + 1;
        const int indexa = (i - 1) * lratiox + 1;
        for (int m = 1; m <= nvar; ++m)
          for (int l = 1; l <= lratiox; ++l)
            sv(m, influx) = sv(m, influx) - amdq(m, indexa + l) * hx * hz * delt - apdq(m, indexa + l) * hx * hz * delt;
      }
      if (kcnext != kc) influx0 = influx;
    }
    // side 3 (x right)
    for (int k = ng + 1; k <= mktot - ng; ++k) {
      const int kc = 1 + (k - (ng + 1)) / lratioz, kcnext = 1 + (k + 1 - (ng + 1)) / lratioz;
      int indaux = 0;
      for (int j = ng + 1; j <= mjtot - ng; ++j) {
        indaux = indaux + 1;
        for (int ma = 1; ma <= maux; ++ma) ar(ma, indaux) = ax(ma, mitot - ng + 1, j, k);
        for (int m = 1; m <= nvar; ++m) qr(m, indaux) = vb(m, mitot - ng + 1, j, k);
      }
      int lind = 0, index = index0;
      for (int jc = 1; jc <= ncrsej; ++jc) {
        index = index + 1;
        for (int l = 1; l <= lratioy; ++l) {
          lind = lind + 1;
          for (int ma = 1; ma <= maux; ++ma) {
            if (is_type(ma, "xleft")) {
              const int kfine = (kc - 1) * lratioz + ng + l, jfine = (jc - 1) * lratioy + ng + l;
              al(ma, lind + 1) = ax(ma, mitot - ng + 1, jfine, kfine);
            } else al(ma, lind + 1) = acd(ma, index);
          }
          for (int m = 1; m <= nvar; ++m) ql(m, lind + 1) = qc(m, index);
        }
      }
      if (kcnext != kc) index0 = index;
      rpn3(prob, 1, nvar, mwaves, mbc, nc + 1 - 2 * ng, QL, QR, AL, AR, W, S, AM, AP);
      int influx = influx0;
      for (int j = 1; j <= nc / lratioy; ++j) {
        influx = influx + 1;
        const int indexa = (j - 1) * lratioy + 1;
        for (int m = 1; m <= nvar; ++m)
          for (int l = 1; l <= lratioy; ++l)
            sv(m, influx) = sv(m, influx) - amdq(m, indexa + l) * hy * hz * delt - apdq(m, indexa + l) * hy * hz * delt;
      }
      if (kcnext != kc) influx0 = influx;
    }
    // side 4 (y bottom)
    for (int k = ng + 1; k <= mktot - ng; ++k) {
      const int kc = 1 + (k - (ng + 1)) / lratioz, kcnext = 1 + (k + 1 - (ng + 1)) / lratioz;
      int indaux = 1;
      for (int i = ng + 1; i <= mitot - ng; ++i) {
        indaux = indaux + 1;
        for (int ma = 1; ma <= maux; ++ma) al(ma, indaux) = is_type(ma, "yleft") ? ax(ma, i, ng + 1, k) : ax(ma, i, ng, k);
        for (int m = 1; m <= nvar; ++m) ql(m, indaux) = vb(m, i, ng, k);
      }
      int lind = 0, index = index0;
      for (int ic = 1; ic <= ncrsei; ++ic) {
        index = index + 1;
        for (int l = 1; l <= lratiox; ++l) {
          lind = lind + 1;
          for (int ma = 1; ma <= maux; ++ma) ar(ma, lind) = acd(ma, index);
          for (int m = 1; m <= nvar; ++m) qr(m, lind) = qc(m, index);
        }
      }
      if (kcnext != kc) index0 = index;
      rpn3(prob, 2, nvar, mwaves, mbc, nr + 1 - 2 * ng, QL, QR, AL, AR, W, S, AM, AP);
      int influx = influx0;
      for (int i = 1; i <= nr / lratiox; ++i) {
        influx = influx + 1;
        const int indexa = (i - 1) * lratiox + 1;
        for (int m = 1; m <= nvar; ++m)
          for (int l = 1; l <= lratiox; ++l)
            sv(m, influx) = sv(m, influx) + amdq(m, indexa + l) * hx * hz * delt + apdq(m, indexa + l) * hx * hz * delt;
      }
      if (kcnext != kc) influx0 = influx;
    }
    // side 5 (z bottom)
    for (int j = ng + 1; j <= mjtot - ng; ++j) {
      const int jc = 1 + (j - (ng + 1)) / lratioy, jcnext = 1 + (j + 1 - (ng + 1)) / lratioy;
      int indaux = 1;
      for (int i = ng + 1; i <= mitot - ng; ++i) {
        indaux = indaux + 1;
        for (int ma = 1; ma <= maux; ++ma) al(ma, indaux) = is_type(ma, "zleft") ? ax(ma, i, j, ng + 1) : ax(ma, i, j, ng);
        for (int m = 1; m <= nvar; ++m) ql(m, indaux) = vb(m, i, j, ng);
      }
      int lind = 0, index = index0;
      for (int ic = 1; ic <= ncrsei; ++ic) {
        index = index + 1;
        for (int l = 1; l <= lratiox; ++l) {
          lind = lind + 1;
          for (int ma = 1; ma <= maux; ++ma) ar(ma, lind) = acd(ma, index);
          for (int m = 1; m <= nvar; ++m) qr(m, lind) = qc(m, index);
        }
      }
      if (jcnext != jc) index0 = index;
      rpn3(prob, 3, nvar, mwaves, mbc, nr + 1 - 2 * ng, QL, QR, AL, AR, W, S, AM, AP);
      int influx = influx0;
      for (int i = 1; i <= nr / lratiox; ++i) {
        influx = influx + 1;
        const int indexa = (i - 1) * lratiox + 1;
        for (int m = 1; m <= nvar; ++m)
          for (int l = 1; l <= lratiox; ++l)
            sv(m, influx) = sv(m, influx) + amdq(m, indexa + l) * hx * hy * delt + apdq(m, indexa + l) * hx * hy * delt;
      }
      if (jcnext != jc) influx0 = influx;
    }
    // side 6 (z top)
    for (int j = ng + 1; j <= mjtot - ng; ++j) {
      const int jc = 1 + (j - (ng + 1)) / lratioy, jcnext = 1 + (j + 1 - (ng + 1)) / lratioy;
      int indaux = 0;
      for (int i = ng + 1; i <= mitot - ng; ++i) {
        indaux = indaux + 1;
        for (int ma = 1; ma <= maux; ++ma) ar(ma, indaux) = ax(ma, i, j, mktot - ng + 1);
        for (int m = 1; m <= nvar; ++m) qr(m, indaux) = vb(m, i, j, mktot - ng + 1);
      }
      int lind = 0, index = index0;
      for (int ic = 1; ic <= ncrsei; ++ic) {
        index = index + 1;
        for (int l = 1; l <= lratiox; ++l) {
          lind = lind + 1;
          for (int ma = 1; ma <= maux; ++ma) {
            if (is_type(ma, "zleft")) {
              const int jfine = (jc - 1) * lratioy + ng + l, ifine = (ic - 1) * lratiox + ng + l;
              al(ma, lind + 1) = ax(ma, ifine, jfine, mktot - ng + 1);
            } else al(ma, lind + 1) = acd(ma, index);
          }
          for (int m = 1; m <= nvar; ++m) ql(m, lind + 1) = qc(m, index);
        }
      }
      if (jcnext != jc) index0 = index;
      rpn3(prob, 3, nvar, mwaves, mbc, nr + 1 - 2 * ng, QL, QR, AL, AR, W, S, AM, AP);
      int influx = influx0;
      for (int i = 1; i <= nr / lratiox; ++i) {
        influx = influx + 1;
        const int indexa = (i - 1) * lratiox + 1;
        for (int m = 1; m <= nvar; ++m)
          for (int l = 1; l <= lratiox; ++l)
            sv(m, influx) = sv(m, influx) - amdq(m, indexa + l) * hx * hy * delt - apdq(m, indexa + l) * hx * hy * delt;
      }
      if (jcnext != jc) influx0 = influx;
    }
  }

  // fluxsv.f:4-94: coarse fluxes next to a kid into the kid's register
  void fluxsv(int mptr, const double* fm, const double* fp, const double* gm, const double* gp, const double* hm,
              const double* hp, int mitot, int mjtot, int mktot, double dtc, double hx, double hy, double hz) {
    const Node3& g = node[mptr];
    FArr3 FM{const_cast<double*>(fm), nvar, mitot, mjtot, mktot}, FP{const_cast<double*>(fp), nvar, mitot, mjtot, mktot};
    FArr3 GM{const_cast<double*>(gm), nvar, mitot, mjtot, mktot}, GP{const_cast<double*>(gp), nvar, mitot, mjtot, mktot};
    FArr3 HM{const_cast<double*>(hm), nvar, mitot, mjtot, mktot}, HP{const_cast<double*>(hp), nvar, mitot, mjtot, mktot};
    const int nsp = (int)g.listbc.size() / 6;
    for (int ispot = 1; ispot <= nsp; ++ispot) {
      const int* e = &g.listbc[6 * (ispot - 1)];
      if (e[0] == 0) break;
      const int i = e[0], j = e[1], k = e[2], side = e[3], mkid = e[4], intopl = e[5];
      double* reg = node[mkid].ffl.data() + (size_t)nvar * (intopl - 1);
      for (int m = 1; m <= nvar; ++m) {
        if (side == 1) reg[m - 1] = -FP(m, i, j, k) * dtc * hy * hz;
        if (side == 2) reg[m - 1] = -GM(m, i, j + 1, k) * dtc * hx * hz;
        if (side == 3) reg[m - 1] = -FM(m, i + 1, j, k) * dtc * hy * hz;
        if (side == 4) reg[m - 1] = -GP(m, i, j, k) * dtc * hx * hz;
        if (side == 5) reg[m - 1] = -HP(m, i, j, k) * dtc * hx * hy;
        if (side == 6) reg[m - 1] = -HM(m, i, j, k + 1) * dtc * hx * hy;
      }
    }
  }

  // fluxad.f:4-155: fine fluxes summed per coarse face into the register
  void fluxad(const double* fm, const double* fp, const double* gm, const double* gp, const double* hm, const double* hp,
              double* svdflx, int mitot, int mjtot, int mktot, int lratiox, int lratioy, int lratioz, double dtf, double dx,
              double dy, double dz) {
    const int ng = nghost;
    FArr3 FM{const_cast<double*>(fm), nvar, mitot, mjtot, mktot}, FP{const_cast<double*>(fp), nvar, mitot, mjtot, mktot};
    FArr3 GM{const_cast<double*>(gm), nvar, mitot, mjtot, mktot}, GP{const_cast<double*>(gp), nvar, mitot, mjtot, mktot};
    FArr3 HM{const_cast<double*>(hm), nvar, mitot, mjtot, mktot}, HP{const_cast<double*>(hp), nvar, mitot, mjtot, mktot};
    const int nxc = (mitot - 2 * ng) / lratiox, nyc = (mjtot - 2 * ng) / lratioy, nzc = (mktot - 2 * ng) / lratioz;
    auto sv = [&](int m, int idx) -> double& { return svdflx[(m - 1) + (size_t)nvar * (idx - 1)]; };
    int lind = 0;
    for (int k = 1; k <= nzc; ++k) {
      const int kf = (k - 1) * lratioz + ng;
      for (int j = 1; j <= nyc; ++j) {
        const int jf = (j - 1) * lratioy + ng;
        ++lind;
        for (int m = 1; m <= nvar; ++m)
          for (int kl = 1; kl <= lratioz; ++kl) for (int jl = 1; jl <= lratioy; ++jl)
            sv(m, lind) = sv(m, lind) + FM(m, ng + 1, jf + jl, kf + kl) * dtf * dy * dz;
      }
    }
    for (int k = 1; k <= nzc; ++k) {
      const int kf = (k - 1) * lratioz + ng;
      for (int i = 1; i <= nxc; ++i) {
        const int iff = (i - 1) * lratiox + ng;
        ++lind;
        for (int m = 1; m <= nvar; ++m)
          for (int kl = 1; kl <= lratioz; ++kl) for (int il = 1; il <= lratiox; ++il)
            sv(m, lind) = sv(m, lind) + GP(m, iff + il, mjtot - ng + 1, kf + kl) * dtf * dx * dz;
      }
    }
    for (int k = 1; k <= nzc; ++k) {
      const int kf = (k - 1) * lratioz + ng;
      for (int j = 1; j <= nyc; ++j) {
        const int jf = (j - 1) * lratioy + ng;
        ++lind;
        for (int m = 1; m <= nvar; ++m)
          for (int kl = 1; kl <= lratioz; ++kl) for (int jl = 1; jl <= lratioy; ++jl)
            sv(m, lind) = sv(m, lind) + FP(m, mitot - ng + 1, jf + jl, kf + kl) * dtf * dy * dz;
      }
    }
    for (int k = 1; k <= nzc; ++k) {
      const int kf = (k - 1) * lratioz + ng;
      for (int i = 1; i <= nxc; ++i) {
        const int iff = (i - 1) * lratiox + ng;
        ++lind;
        for (int m = 1; m <= nvar; ++m)
          for (int kl = 1; kl <= lratioz; ++kl) for (int il = 1; il <= lratiox; ++il)
            sv(m, lind) = sv(m, lind) + GM(m, iff + il, ng + 1, kf + kl) * dtf * dx * dz;
      }
    }
    for (int j = 1; j <= nyc; ++j) {
      const int jf = (j - 1) * lratioy + ng;
      for (int i = 1; i <= nxc; ++i) {
        const int iff = (i - 1) * lratiox + ng;
        ++lind;
        for (int m = 1; m <= nvar; ++m)
          for (int jl = 1; jl <= lratioy; ++jl) for (int il = 1; il <= lratiox; ++il)
            sv(m, lind) = sv(m, lind) + HM(m, iff + il, jf + jl, ng + 1) * dtf * dx * dy;
      }
    }
    for (int j = 1; j <= nyc; ++j) {
      const int jf = (j - 1) * lratioy + ng;
      for (int i = 1; i <= nxc; ++i) {
        const int iff = (i - 1) * lratiox + ng;
        ++lind;
        for (int m = 1; m <= nvar; ++m)
          for (int jl = 1; jl <= lratioy; ++jl) for (int il = 1; il <= lratiox; ++il)
            sv(m, lind) = sv(m, lind) + HP(m, iff + il, jf + jl, mktot - ng + 1) * dtf * dx * dy;
      }
    }
  }

  // gauges_module.f90:302-460 (update_gauges)
  void update_gauges(const double* q, double xlow, double ylow, double zlow, int mitot, int mjtot, int mktot, int mptr) {
    const Node3& g = node[mptr];
    const int lev = g.level;
    const double hx = hxposs[lev], hy = hyposs[lev], hz = hzposs[lev];
    const double tgrid = g.time;
    FArr3 Q{const_cast<double*>(q), nvar, mitot, mjtot, mktot};
    for (size_t i = 0; i < gauges.size(); ++i) {
      if (mbestsrc[i] != mptr) continue;
      Gauge3& G = gauges[i];
      if (tgrid < G.t_start || tgrid > G.t_end) continue;
      if (tgrid - G.last_time < G.min_inc) continue;
      const int ii = (int)(0.5 + (G.x - xlow) / hx), jj = (int)(0.5 + (G.y - ylow) / hy), kk = (int)(0.5 + (G.z - zlow) / hz);
      const double xcent = xlow + (ii - 0.5) * hx, ycent = ylow + (jj - 0.5) * hy, zcent = zlow + (kk - 0.5) * hz;
      const double xoff = (G.x - xcent) / hx, yoff = (G.y - ycent) / hy, zoff = (G.z - zcent) / hz;
      GaugeSample3 smp;
      smp.level = lev; smp.t = tgrid;
      for (int n = 1; n <= nvar; ++n) {
        double v = (1.0 - xoff) * (1.0 - yoff) * Q(n, ii, jj, kk) + xoff * (1.0 - yoff) * Q(n, ii + 1, jj, kk) +
                   (1.0 - xoff) * yoff * Q(n, ii, jj + 1, kk) + xoff * yoff * Q(n, ii + 1, jj + 1, kk);
        v = v * (1.0 - zoff);
        v = v + zoff * ((1.0 - xoff) * (1.0 - yoff) * Q(n, ii, jj, kk + 1) + xoff * (1.0 - yoff) * Q(n, ii + 1, jj, kk + 1) +
                        (1.0 - xoff) * yoff * Q(n, ii, jj + 1, kk + 1) + xoff * yoff * Q(n, ii + 1, jj + 1, kk + 1));
        smp.v.push_back(v);
      }
      G.data.push_back(smp);
      G.last_time = tgrid;
    }
  }

  // advanc.f:166-303 (par_advanc)
  void par_advanc(int mptr, double& dtnew, double& cflgrid) {
    Node3& g = node[mptr];
    const int level = g.level;
    const double hx = hxposs[level], hy = hyposs[level], hz = hzposs[level];
    const double delt = possk[level];
    const int mitot = mitot_of(mptr), mjtot = mjtot_of(mptr), mktot = mktot_of(mptr);
    const int nx = g.ihi - g.ilo + 1, ny = g.jhi - g.jlo + 1, nz = g.khi - g.klo + 1;
    if (level < mxnest) g.q2 = g.q1;
    const double xlow = g.xlo - nghost * hx, ylow = g.ylo - nghost * hy, zlow = g.zlo - nghost * hz;
    if (g.has_ffl) {
      const int lenbc = 2 * ((nx / intratx[level - 1]) * (nz / intratz[level - 1]) + (ny / intraty[level - 1]) * (nz / intratz[level - 1]) +
                             (nx / intratx[level - 1]) * (ny / intraty[level - 1]));
      qad(g.q1.data(), g.aux.data(), mitot, mjtot, mktot, g.ffl.data(), g.ffl.data() + (size_t)nvar * lenbc,
          g.ffl.data() + (size_t)2 * nvar * lenbc, intratx[level - 1], intraty[level - 1], intratz[level - 1], hx, hy, hz, delt);
    }
    if (!gauges.empty() && record_gauges) update_gauges(g.q1.data(), xlow, ylow, zlow, mitot, mjtot, mktot, mptr);
    const size_t n = qsize(mptr);
    std::vector<double> fm(n), fp(n), gm(n), gp(n), hm(n), hp(n);
    if (naux > 0) b4step3(nx, ny, nz, g.xlo, g.ylo, g.zlo, hx, hy, hz, g.time, g.aux.data());
    // src/3d/advanc.f:261-280: unsplit or Godunov-split step
    if (dimensional_split == 0)
      stepgrid(g.q1.data(), fm.data(), fp.data(), gm.data(), gp.data(), hm.data(), hp.data(), mitot, mjtot, mktot, delt, dtnew, hx,
               hy, hz, g.aux.data(), cflgrid);
    else
      stepgrid_dimSplit(g.q1.data(), fm.data(), fp.data(), gm.data(), gp.data(), hm.data(), hp.data(), mitot, mjtot, mktot, delt,
                        dtnew, hx, hy, hz, g.aux.data(), cflgrid);
    if (g.has_cfl) fluxsv(mptr, fm.data(), fp.data(), gm.data(), gp.data(), hm.data(), hp.data(), mitot, mjtot, mktot, delt, hx, hy, hz);
    if (g.has_ffl)
      fluxad(fm.data(), fp.data(), gm.data(), gp.data(), hm.data(), hp.data(), g.ffl.data(), mitot, mjtot, mktot, intratx[level - 1],
             intraty[level - 1], intratz[level - 1], delt, hx, hy, hz);
    g.time = g.time + delt;
  }

  // advanc.f:4-139
  void advanc(int level, double& dtlevnew) {
    const std::vector<int>& G = levelgrids[level];
    for (int mptr : G) {
      Node3& g = node[mptr];
      bound(g.time, g.q1.data(), mitot_of(mptr), mjtot_of(mptr), mktot_of(mptr), mptr);
    }
    if (level + 1 <= mxnest && lstart[level + 1] != 0) saveqc(level + 1);
    dtlevnew = RINFINITY3;
    cfl_level = 0.0;
    std::vector<double> dtn(G.size()), cg(G.size());
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (long j = 0; j < (long)G.size(); ++j) par_advanc(G[j], dtn[j], cg[j]);
    for (size_t j = 0; j < G.size(); ++j) {
      const Node3& g = node[G[j]];
      const double cells = (double)(g.ihi - g.ilo + 1) * (g.jhi - g.jlo + 1) * (g.khi - g.klo + 1);
      rvol += cells; rvoll[level] += cells;
      dtlevnew = std::min(dtlevnew, dtn[j]);
      cfl_level = std::max(cfl_level, cg[j]);
    }
    cflmax = std::max(cflmax, cfl_level);
  }

  // upbnd.f:4-94
  void upbnd(int mptr) {
    Node3& g = node[mptr];
    const int mitot = mitot_of(mptr), mjtot = mjtot_of(mptr), mktot = mktot_of(mptr);
    FArr3 val{g.q1.data(), nvar, mitot, mjtot, mktot};
    std::vector<int> iused((size_t)mitot * mjtot * mktot, 0);
    const double chsign[7] = {0, 1., -1., -1., 1., 1., -1.};
    const int levc = g.level;
    const double volume = hxposs[levc] * hyposs[levc] * hzposs[levc];
    const int nsp = (int)g.listbc.size() / 6;
    for (int ispot = 1; ispot <= nsp; ++ispot) {
      const int* e = &g.listbc[6 * (ispot - 1)];
      const int icrse = e[0];
      if (icrse == 0) break;
      const int jcrse = e[1], kcrse = e[2], iside = e[3];
      const int norm = 1 << (iside - 1);
      int& used = iused[(size_t)(icrse - 1) + (size_t)mitot * ((jcrse - 1) + (size_t)mjtot * (kcrse - 1))];
      if ((used / norm) % 2 == 1) continue;
      const int mkid = e[4], lkid = e[5];
      const double sgnm = chsign[iside];
      const double* reg = node[mkid].ffl.data() + (size_t)nvar * (lkid - 1);
      for (int m = 1; m <= nvar; ++m) val(m, icrse, jcrse, kcrse) = val(m, icrse, jcrse, kcrse) + sgnm * reg[m - 1] / volume;
      used = used + norm;
    }
  }

  // update.f:4-192
  void update(int level) {
    const int lget = level;
    for (int mptr : levelgrids[lget]) {
      Node3& g = node[mptr];
      const int mitot = mitot_of(mptr), mjtot = mjtot_of(mptr), mktot = mktot_of(mptr);
      if (g.has_cfl) upbnd(mptr);
      FArr3 Q{g.q1.data(), nvar, mitot, mjtot, mktot};
      for (int mkid = lstart[lget + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        const Node3& f = node[mkid];
        const int rx = intratx[lget], ry = intraty[lget], rz = intratz[lget];
        const int iclo = f.ilo / rx, jclo = f.jlo / ry, kclo = f.klo / rz, ichi = f.ihi / rx, jchi = f.jhi / ry, kchi = f.khi / rz;
        const int mi = mitot_of(mkid), mj = mjtot_of(mkid), mk = mktot_of(mkid);
        FArr3 QF{const_cast<double*>(f.q1.data()), nvar, mi, mj, mk};
        const int iplo = std::max(g.ilo, iclo), jplo = std::max(g.jlo, jclo), kplo = std::max(g.klo, kclo);
        const int iphi = std::min(g.ihi, ichi), jphi = std::min(g.jhi, jchi), kphi = std::min(g.khi, kchi);
        if (iplo > iphi || jplo > jphi || kplo > kphi) continue;
        const int totrat = rx * ry * rz;
        int iff = iplo * rx - f.ilo + nghost + 1;
        for (int i = iplo - g.ilo + nghost + 1; i <= iphi - g.ilo + nghost + 1; ++i) {
          int jff = jplo * ry - f.jlo + nghost + 1;
          for (int j = jplo - g.jlo + nghost + 1; j <= jphi - g.jlo + nghost + 1; ++j) {
            int kff = kplo * rz - f.klo + nghost + 1;
            for (int k = kplo - g.klo + nghost + 1; k <= kphi - g.klo + nghost + 1; ++k) {
              for (int m = 1; m <= nvar; ++m) Q(m, i, j, k) = 0.0;
              for (int kco = 1; kco <= rz; ++kco)
                for (int jco = 1; jco <= ry; ++jco)
                  for (int ico = 1; ico <= rx; ++ico)
                    for (int m = 1; m <= nvar; ++m) Q(m, i, j, k) = Q(m, i, j, k) + QF(m, iff + ico - 1, jff + jco - 1, kff + kco - 1);
              for (int m = 1; m <= nvar; ++m) Q(m, i, j, k) = Q(m, i, j, k) / totrat;
              kff = kff + rz;
            }
            jff = jff + ry;
          }
          iff = iff + rx;
        }
      }
    }
  }

  // ===================================================== registers: prepf.f, setuse.f, prepc.f, putsp.f
  void prepf(int level) {
    for (int mkid = lstart[level]; mkid != 0; mkid = node[mkid].levelptr) {
      Node3& k = node[mkid];
      const int ikeep = (k.ihi - k.ilo + 1) / intratx[level - 1], jkeep = (k.jhi - k.jlo + 1) / intraty[level - 1];
      const int kkeep = (k.khi - k.klo + 1) / intratz[level - 1];
      const int lenbc = 2 * (ikeep * jkeep + jkeep * kkeep + kkeep * ikeep);
      k.ffl.assign((size_t)2 * nvar * lenbc + (size_t)naux * lenbc, 0.0);
      k.has_ffl = true;
    }
  }
  void setuse(std::vector<int>& lb, int& ispot, int mkid, int ilo, int ihi, int jlo, int jhi, int klo, int khi, int iclo,
              int ichi, int jclo, int jchi, int kclo, int kchi) {
    auto put = [&](int i, int j, int k, int side, int lkid) { ++ispot; lb.insert(lb.end(), {i, j, k, side, mkid, lkid}); };
    const int ng = nghost;
    const int ist = iclo - 1, iend = ichi + 1, jst = jclo - 1, jend = jchi + 1, kst = kclo - 1, kend = kchi + 1;
    const int ni = ichi - iclo + 1, nj = jchi - jclo + 1, nk = kchi - kclo + 1;
    if (!(ist < ilo))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = (k - kclo) * nj + std::max(jlo, jclo) - jclo + 1;
        for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) put(ist - ilo + ng + 1, j - jlo + ng + 1, k - klo + ng + 1, 3, lkid++);
      }
    if (!(jend > jhi))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = nk * nj + (k - kclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + ng + 1, jend - jlo + ng + 1, k - klo + ng + 1, 4, lkid++);
      }
    if (!(iend > ihi))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = nk * nj + nk * ni + (k - kclo) * nj + std::max(jlo, jclo) - jclo + 1;
        for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) put(iend - ilo + ng + 1, j - jlo + ng + 1, k - klo + ng + 1, 1, lkid++);
      }
    if (!(jst < jlo))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = nk * nj + nk * ni + nk * nj + (k - kclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + ng + 1, jst - jlo + ng + 1, k - klo + ng + 1, 2, lkid++);
      }
    if (!(kst < klo))
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) {
        int lkid = nk * nj + nk * ni + nk * nj + nk * ni + (j - jclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + ng + 1, j - jlo + ng + 1, kst - klo + ng + 1, 6, lkid++);
      }
    if (!(kend > khi))
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) {
        int lkid = nk * nj + nk * ni + nk * nj + nk * ni + nj * ni + (j - jclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + ng + 1, j - jlo + ng + 1, kend - klo + ng + 1, 5, lkid++);
      }
  }
  void prepc(int level) {
    int maxsp = 0;
    for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
      const Node3& k = node[mkid];
      const int ik = (k.ihi - k.ilo + 1) / intratx[level], jk = (k.jhi - k.jlo + 1) / intraty[level], kk = (k.khi - k.klo + 1) / intratz[level];
      maxsp += 2 * (ik * jk + jk * kk + kk * ik);
    }
    listsp[level] = maxsp;
    if (maxsp == 0) return;
    for (int mpar = lstart[level]; mpar != 0; mpar = node[mpar].levelptr) {
      int ispot = 0;
      Node3& p = node[mpar];
      p.listbc.clear();
      p.has_cfl = true;
      for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        const Node3& k = node[mkid];
        const int iclo = k.ilo / intratx[level], jclo = k.jlo / intraty[level], kclo = k.klo / intratz[level];
        const int ichi = k.ihi / intratx[level], jchi = k.jhi / intraty[level], kchi = k.khi / intratz[level];
        const int iplo = std::max(p.ilo, iclo), jplo = std::max(p.jlo, jclo), kplo = std::max(p.klo, kclo);
        const int iphi = std::min(p.ihi, ichi), jphi = std::min(p.jhi, jchi), kphi = std::min(p.khi, kchi);
        if ((iplo <= iphi + 1 && jplo <= jphi + 1) && kplo <= kphi + 1)
          setuse(p.listbc, ispot, mkid, p.ilo, p.ihi, p.jlo, p.jhi, p.klo, p.khi, iclo, ichi, jclo, jchi, kclo, kchi);
        // prepc.f:84-122: fine grids touching a periodic boundary, through their images
        const int imax = iregsz[level] - 1, jmax = jregsz[level] - 1, kmax = kregsz[level] - 1;
        const int ni = iregsz[level], nj = jregsz[level], nk = kregsz[level];
        auto use = [&](int a0, int a1, int b0, int b1, int c0, int c1) {
          setuse(p.listbc, ispot, mkid, p.ilo, p.ihi, p.jlo, p.jhi, p.klo, p.khi, a0, a1, b0, b1, c0, c1);
        };
        if (xperdom && p.ilo == 0 && ichi == imax) use(iclo - ni, ichi - ni, jclo, jchi, kclo, kchi);
        if (xperdom && iclo == 0 && p.ihi == imax) use(iclo + ni, ichi + ni, jclo, jchi, kclo, kchi);
        if (yperdom && p.jlo == 0 && jchi == jmax) use(iclo, ichi, jclo - nj, jchi - nj, kclo, kchi);
        if (yperdom && jclo == 0 && p.jhi == jmax) use(iclo, ichi, jclo + nj, jchi + nj, kclo, kchi);
        if (zperdom && p.klo == 0 && kchi == kmax) use(iclo, ichi, jclo, jchi, kclo - nk, kchi - nk);
        if (zperdom && kclo == 0 && p.khi == kmax) use(iclo, ichi, jclo, jchi, kclo + nk, kchi + nk);
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
    }
  }
  // init_bndryList.f:50-107 (neighbours by their i,j extents only, as in the reference)
  void makeBndryList(int level) {
    const std::vector<int>& G = levelgrids[level];
    for (size_t n = 0; n < G.size(); ++n) {
      Node3& g = node[G[n]];
      g.bnd.clear();
      const int imin = g.ilo - nghost, imax = g.ihi + nghost, jmin = g.jlo - nghost, jmax = g.jhi + nghost;
      std::vector<int> found;
      for (size_t k = 0; k < G.size(); ++k) {
        if (k == n) continue;
        const Node3& s = node[G[k]];
        if (std::max(s.ilo, imin) <= std::min(s.ihi, imax) && std::max(s.jlo, jmin) <= std::min(s.jhi, jmax)) found.push_back(G[k]);
      }
      for (auto it = found.rbegin(); it != found.rend(); ++it) g.bnd.push_back(*it);
    }
  }

  // quick_sort1.f (qsorti): non-stable index sort, replicated step by step (1-based views)
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

  // regrid.f:122-159 (arrangeGrids): most expensive first, cost = nx*ny
  void arrangeGrids(int level, int numg) {
    std::vector<int> listgrids(numg + 1), index(numg + 1);
    std::vector<long long> cost(numg + 1);
    int mptr = lstart[level];
    for (int i = 1; i <= numg; ++i) {
      listgrids[i] = mptr;
      cost[i] = (long long)(node[mptr].ihi - node[mptr].ilo + 1) * (node[mptr].jhi - node[mptr].jlo + 1);
      mptr = node[mptr].levelptr;
    }
    qsorti(index, numg, cost);
    lstart[level] = listgrids[index[numg]];
    int prev = listgrids[index[numg]];
    for (int i = 1; i <= numg - 1; ++i) { node[prev].levelptr = listgrids[index[numg - i]]; prev = listgrids[index[numg - i]]; }
    node[prev].levelptr = 0;
  }

  // birect.f:4-172
  void birect(int mptr1) {
    int mptr = mptr1;
    const int level = node[mptr].level;
    const double hx = hxposs[level], hy = hyposs[level], hz = hzposs[level];
    while (true) {
      Node3& a = node[mptr];
      const int nxg = a.ihi - a.ilo + 1, nyg = a.jhi - a.jlo + 1, nzg = a.khi - a.klo + 1;
      if (nxg + 2 * nghost > max1d) {
        int nxl = nxg / 2;
        const int lratio = level > 1 ? intratx[level - 1] : 2;
        nxl = (nxl / lratio) * lratio;
        const double cxmid = a.xlo + nxl * hx;
        const int mn = nodget();
        Node3& p = node[mptr];
        Node3& b = node[mn];
        b.levelptr = p.levelptr; p.levelptr = mn;
        b.ihi = p.ihi; p.ihi = p.ilo + nxl - 1; b.ilo = p.ihi + 1;
        b.jhi = p.jhi; b.jlo = p.jlo; b.khi = p.khi; b.klo = p.klo;
        b.xlo = cxmid; b.ylo = p.ylo; b.zlo = p.zlo; b.xhi = p.xhi; b.yhi = p.yhi; b.zhi = p.zhi;
        p.xhi = cxmid;
        b.time = p.time; b.level = p.level;
      } else if (nyg + 2 * nghost > max1d) {
        int nyl = nyg / 2;
        const int lratio = level > 1 ? intraty[level - 1] : 2;
        nyl = (nyl / lratio) * lratio;
        const double cymid = a.ylo + nyl * hy;
        const int mn = nodget();
        Node3& p = node[mptr];
        Node3& b = node[mn];
        b.levelptr = p.levelptr; p.levelptr = mn;
        b.jhi = p.jhi; p.jhi = p.jlo + nyl - 1; b.jlo = p.jhi + 1;
        b.khi = p.khi; b.klo = p.klo; b.ihi = p.ihi; b.ilo = p.ilo;
        b.xlo = p.xlo; b.ylo = cymid; b.zlo = p.zlo; b.xhi = p.xhi; b.yhi = p.yhi; b.zhi = p.zhi;
        p.yhi = cymid;
        b.level = p.level; b.time = p.time;
      } else if (nzg + 2 * nghost > max1d) {
        int nzl = nzg / 2;
        const int lratio = level > 1 ? intratz[level - 1] : 2;
        nzl = (nzl / lratio) * lratio;
        const double czmid = a.zlo + nzl * hz;
        const int mn = nodget();
        Node3& p = node[mptr];
        Node3& b = node[mn];
        b.levelptr = p.levelptr; p.levelptr = mn;
        b.khi = p.khi; p.khi = p.klo + nzl - 1; b.klo = p.khi + 1;
        b.ihi = p.ihi; b.ilo = p.ilo; b.jhi = p.jhi; b.jlo = p.jlo;
        b.xlo = p.xlo; b.ylo = p.ylo; b.zlo = czmid; b.xhi = p.xhi; b.yhi = p.yhi; b.zhi = p.zhi;
        p.zhi = czmid;
        b.level = p.level; b.time = p.time;
      } else {
        mptr = node[mptr].levelptr;
        if (mptr == 0) break;
      }
    }
  }

  // ================================================================ regrid: domain flags
  // The border ring of domprep/domshrink/domup/domcopy, direction by direction (x, y, z):
  // a periodic direction copies the far interior layer over the whole ring of the other two
  // indices (0..n+1); otherwise the interior edge is extended over the interior (skipped in
  // domshrink's periodic directions, which keep their ring: skip_periodic).
  void extend_borders(I1& f, int is, int js, int ks, bool skip_periodic = false) {
    if (xperdom) {
      if (!skip_periodic)
        for (int k = 0; k <= ks + 1; ++k) for (int j = 0; j <= js + 1; ++j) { f(0, j, k) = f(is, j, k); f(is + 1, j, k) = f(1, j, k); }
    } else {
      for (int k = 1; k <= ks; ++k) for (int j = 1; j <= js; ++j) {
        if (f(1, j, k) == 1) f(0, j, k) = 1;
        if (f(is, j, k) == 1) f(is + 1, j, k) = 1;
      }
    }
    if (yperdom) {
      if (!skip_periodic)
        for (int k = 0; k <= ks + 1; ++k) for (int i = 0; i <= is + 1; ++i) { f(i, 0, k) = f(i, js, k); f(i, js + 1, k) = f(i, 1, k); }
    } else {
      for (int k = 1; k <= ks; ++k) for (int i = 1; i <= is; ++i) {
        if (f(i, 1, k) == 1) f(i, 0, k) = 1;
        if (f(i, js, k) == 1) f(i, js + 1, k) = 1;
      }
    }
    if (zperdom) {
      if (!skip_periodic)
        for (int j = 0; j <= js + 1; ++j) for (int i = 0; i <= is + 1; ++i) { f(i, j, 0) = f(i, j, ks); f(i, j, ks + 1) = f(i, j, 1); }
    } else {
      for (int j = 1; j <= js; ++j) for (int i = 1; i <= is; ++i) {
        if (f(i, j, 1) == 1) f(i, j, 0) = 1;
        if (f(i, j, ks) == 1) f(i, j, ks + 1) = 1;
      }
    }
  }
  // domprep.f:82-154 / domup.f:96-169: edge and corner cells of the border ring
  void fill_edges_corners(I1& f, int is, int js, int ks) {
    for (int k = 1; k <= ks; ++k) {
      if (f(0, 1, k) + f(1, 0, k) == 2) f(0, 0, k) = 1;
      if (f(0, js, k) + f(1, js + 1, k) == 2) f(0, js + 1, k) = 1;
      if (f(is, 0, k) + f(is + 1, 1, k) == 2) f(is + 1, 0, k) = 1;
      if (f(is, js + 1, k) + f(is + 1, js, k) == 2) f(is + 1, js + 1, k) = 1;
    }
    for (int i = 1; i <= is; ++i) {
      if (f(i, 0, 1) + f(i, 1, 0) == 2) f(i, 0, 0) = 1;
      if (f(i, js, 0) + f(i, js + 1, 1) == 2) f(i, js + 1, 0) = 1;
      if (f(i, 0, ks) + f(i, 1, ks + 1) == 2) f(i, 0, ks + 1) = 1;
      if (f(i, js + 1, ks) + f(i, js, ks + 1) == 2) f(i, js + 1, ks + 1) = 1;
    }
    for (int j = 1; j <= js; ++j) {
      if (f(0, j, 1) + f(1, j, 0) == 2) f(0, j, 0) = 1;
      if (f(is, j, 0) + f(is + 1, j, 1) == 2) f(is + 1, j, 0) = 1;
      if (f(0, j, ks) + f(1, j, ks + 1) == 2) f(0, j, ks + 1) = 1;
      if (f(is + 1, j, ks) + f(is, j, ks + 1) == 2) f(is + 1, j, ks + 1) = 1;
    }
    if (f(0, 0, 1) + f(0, 1, 0) + f(1, 0, 0) == 3) f(0, 0, 0) = 1;
    if (f(is + 1, 0, 1) + f(is + 1, 1, 0) + f(is, 0, 0) == 3) f(is + 1, 0, 0) = 1;
    if (f(0, js + 1, 1) + f(0, js, 0) + f(1, js + 1, 0) == 3) f(0, js + 1, 0) = 1;
    if (f(is + 1, js + 1, 1) + f(is + 1, js, 0) + f(is, js + 1, 0) == 3) f(is + 1, js + 1, 0) = 1;
    if (f(0, 0, ks) + f(0, 1, ks + 1) + f(1, 0, ks + 1) == 3) f(0, 0, ks + 1) = 1;
    if (f(is + 1, 0, ks) + f(is + 1, 1, ks + 1) + f(is, 0, ks + 1) == 3) f(is + 1, 0, ks + 1) = 1;
    if (f(0, js + 1, ks) + f(0, js, ks + 1) + f(1, js + 1, ks + 1) == 3) f(0, js + 1, ks + 1) = 1;
    if (f(is + 1, js + 1, ks) + f(is + 1, js, ks + 1) + f(is, js + 1, ks + 1) == 3) f(is + 1, js + 1, ks + 1) = 1;
  }
  // domprep.f:4-169
  void domprep(I1& f, int lbase, int ib, int jb, int kb) {
    f.init(ib, jb, kb);
    for (int m = lstart[lbase]; m != 0; m = node[m].levelptr) {
      const Node3& g = node[m];
      for (int k = g.klo + 1; k <= g.khi + 1; ++k) for (int j = g.jlo + 1; j <= g.jhi + 1; ++j) for (int i = g.ilo + 1; i <= g.ihi + 1; ++i) f(i, j, k) = 1;
    }
    extend_borders(f, ib, jb, kb);
    fill_edges_corners(f, ib, jb, kb);
  }
  // domshrink.f:4-93: keep cells whose 27-cell neighbourhood is all inside; the
  // output keeps its previous border ring, extended where the interior edge is 1
  void domshrink(I1& in, I1& out, int id, int jd, int kd) {
    if (out.is != id || out.js != jd || out.ks != kd) out.init(id, jd, kd);
    for (int k = 1; k <= kd; ++k)
      for (int j = 1; j <= jd; ++j)
        for (int i = 1; i <= id; ++i) {
          bool ok = true;
          for (int c = -1; c <= 1 && ok; ++c) for (int b = -1; b <= 1 && ok; ++b) for (int a = -1; a <= 1; ++a)
            if (in(i + a, j + b, k + c) <= 0) { ok = false; break; }
          out(i, j, k) = ok ? in(i, j, k) : 0;
        }
    extend_borders(out, id, jd, kd, true);
  }
  // domup.f:4-185
  void domup(I1& fine, I1& crse, int ib, int jb, int kb, int is, int js, int ks, int lev) {
    fine.init(is, js, ks);
    const int rx = intratx[lev], ry = intraty[lev], rz = intratz[lev];
    for (int k = 1; k <= kb; ++k)
      for (int j = 1; j <= jb; ++j)
        for (int i = 1; i <= ib; ++i)
          for (int mk = 1; mk <= rz; ++mk) for (int mj = 1; mj <= ry; ++mj) for (int mi = 1; mi <= rx; ++mi)
            fine((i - 1) * rx + mi, (j - 1) * ry + mj, (k - 1) * rz + mk) = crse(i, j, k);
    extend_borders(fine, is, js, ks);
    fill_edges_corners(fine, is, js, ks);
  }
  // domcopy.f:4-82
  void domcopy(I1& dst, I1& src, int is, int js, int ks) {
    dst = src;
    extend_borders(dst, is, js, ks);
  }

  // spest.f:4-101 with flag2refine.f:3-92 and setflags.f:4-33
  void spest(int lcheck, I1& flags) {
    const int isize = iregsz[lcheck], jsize = jregsz[lcheck], ksize = kregsz[lcheck];
    for (int i = 1; i <= isize; ++i) for (int j = 1; j <= jsize; ++j) for (int k = 1; k <= ksize; ++k) flags(i, j, k) = 0;
    const std::vector<int> G(levelgrids[lcheck]);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (long n = 0; n < (long)G.size(); ++n) {
      const int mptr = G[n];
      Node3& g = node[mptr];
      const int mitot = mitot_of(mptr), mjtot = mjtot_of(mptr), mktot = mktot_of(mptr);
      g.tmp = g.q1;
      bound(g.time, g.tmp.data(), mitot, mjtot, mktot, mptr);
    }
    for (int mptr : G) {
      Node3& g = node[mptr];
      if (!flag_gradient) continue;
      const int mitot = mitot_of(mptr), mjtot = mjtot_of(mptr), mktot = mktot_of(mptr);
      const int mx = mitot - 2 * nghost, my = mjtot - 2 * nghost, mz = mktot - 2 * nghost;
      std::vector<double> amr((size_t)mitot * mjtot * mktot, GOODPT);
      FArr3 Q{g.tmp.data(), nvar, mitot, mjtot, mktot};
      auto AF = [&](int i, int j, int k) -> double& { return amr[(size_t)(i + nghost - 1) + (size_t)mitot * ((j + nghost - 1) + (size_t)mjtot * (k + nghost - 1))]; };
      auto q = [&](int m, int i, int j, int k) { return Q(m, i + nghost, j + nghost, k + nghost); };
      for (int k = 1; k <= mz; ++k)
        for (int j = 1; j <= my; ++j)
          for (int i = 1; i <= mx; ++i) {
            AF(i, j, k) = GOODPT;
            double dq = 0.0;
            if (flag_pressure) {
              // euler_3d_radial flag2refine.f pattern: the difference of the pressure
              auto pres = [&](int a, int b, int c) {
                const double rho = q(1, a, b, c), mu = q(2, a, b, c), mv = q(3, a, b, c), mw = q(4, a, b, c);
                return prob.gamma1 * (q(5, a, b, c) - 0.5 * (mu * mu + mv * mv + mw * mw) / rho);
              };
              const double dpi = std::fabs(pres(i + 1, j, k) - pres(i - 1, j, k));
              const double dpj = std::fabs(pres(i, j + 1, k) - pres(i, j - 1, k));
              const double dpk = std::fabs(pres(i, j, k + 1) - pres(i, j, k - 1));
              dq = std::max(std::max(std::max(dq, dpi), dpj), dpk);
            } else {
              for (int m = 1; m <= nvar; ++m) {
                const double dqi = std::fabs(q(m, i + 1, j, k) - q(m, i - 1, j, k));
                const double dqj = std::fabs(q(m, i, j + 1, k) - q(m, i, j - 1, k));
                const double dqk = std::fabs(q(m, i, j, k + 1) - q(m, i, j, k - 1));
                dq = std::max(std::max(std::max(dq, dqi), dqj), dqk);
              }
            }
            if (dq > tolsp) AF(i, j, k) = BADPT;
          }
      // setflags.f: iflags += rctold(1,i,j,k) over the interior (integer*1 truncation of the sum)
      const int ibeg = g.ilo - nghost, jbeg = g.jlo - nghost, kbeg = g.klo - nghost;
      for (int k = nghost + 1; k <= mktot - nghost; ++k)
        for (int j = nghost + 1; j <= mjtot - nghost; ++j)
          for (int i = nghost + 1; i <= mitot - nghost; ++i) {
            signed char& f = flags(ibeg + i, jbeg + j, kbeg + k);
            f = (signed char)(int)((double)f + amr[(size_t)(i - 1) + (size_t)mitot * ((j - 1) + (size_t)mjtot * (k - 1))]);
          }
    }
  }

  // bufnst.f:4-124 with projec.f:4-101 and shiftset.f:4-108; returns numbad
  int bufnst(int lcheck, I1& f) {
    const int isize = iregsz[lcheck], jsize = jregsz[lcheck], ksize = kregsz[lcheck];
    for (int mptr = lstart[lcheck]; mptr != 0; mptr = node[mptr].levelptr) {
      Node3& g = node[mptr];
      // bufnst.f:21-24 (tol > 0): setflags adds component 1 of store2, where errf1.f left
      // goodpt/badpt; errest() above adds those flags itself (a tolerance without
      // flag_richardson is refused at input)
      g.tmp.clear();
      g.tmp.shrink_to_fit();
    }
    if (lcheck + 2 <= mxnest) {
      // projec.f
      const int lrx = intratx[lcheck] * intratx[lcheck + 1], lry = intraty[lcheck] * intraty[lcheck + 1], lrz = intratz[lcheck] * intratz[lcheck + 1];
      for (int mkid = newstl[lcheck + 2]; mkid != 0; mkid = node[mkid].levelptr) {
        const Node3& c = node[mkid];
        int ist = c.ilo / lrx, jst = c.jlo / lry, kst = c.klo / lrz;
        int iend = (c.ihi + lrx - 1) / lrx, jend = (c.jhi + lry - 1) / lry, kend = (c.khi + lrz - 1) / lrz;
        if (ibuff == 0) {
          if (ist * lrx == c.ilo) ist = ist - 1;
          if (jst * lry == c.jlo) jst = jst - 1;
          if (kst * lrz == c.klo) kst = kst - 1;
          if (iend * lrx == c.ihi + 1) iend = iend + 1;
          if (jend * lry == c.jhi + 1) jend = jend + 1;
          if (kend * lrz == c.khi + 1) kend = kend + 1;
        }
        for (int k = kst + 1; k <= kend + 1; ++k) for (int j = jst + 1; j <= jend + 1; ++j) for (int i = ist + 1; i <= iend + 1; ++i)
          if (f(i, j, k) == (signed char)GOODPT) f(i, j, k) = (signed char)BADPRO;
      }
    }
    // shiftset.f: the ring is the periodic image (or zero), then every interior flag is
    // buffered by ibuff into a second array whose interior is added back (the ring of the
    // second array is not: buffering does not wrap)
    for (int k = 0; k <= ksize + 1; ++k) for (int j = 0; j <= jsize + 1; ++j) {
      f(0, j, k) = xperdom ? f(isize, j, k) : 0;
      f(isize + 1, j, k) = xperdom ? f(1, j, k) : 0;
    }
    for (int k = 0; k <= ksize + 1; ++k) for (int i = 0; i <= isize + 1; ++i) {
      f(i, 0, k) = yperdom ? f(i, jsize, k) : 0;
      f(i, jsize + 1, k) = yperdom ? f(i, 1, k) : 0;
    }
    for (int j = 0; j <= jsize + 1; ++j) for (int i = 0; i <= isize + 1; ++i) {
      f(i, j, 0) = zperdom ? f(i, j, ksize) : 0;
      f(i, j, ksize + 1) = zperdom ? f(i, j, 1) : 0;
    }
    I1 f2;
    f2.init(isize, jsize, ksize);
    for (int k = 1; k <= ksize; ++k)
      for (int j = 1; j <= jsize; ++j)
        for (int i = 1; i <= isize; ++i) {
          const signed char v = f(i, j, k);
          if (v > 0) {
            for (int kk = std::max(k - ibuff, 0); kk <= std::min(k + ibuff, ksize + 1); ++kk)
              for (int jj = std::max(j - ibuff, 0); jj <= std::min(j + ibuff, jsize + 1); ++jj)
                for (int ii = std::max(i - ibuff, 0); ii <= std::min(i + ibuff, isize + 1); ++ii) f2(ii, jj, kk) = v;
          }
        }
    for (int k = 1; k <= ksize; ++k) for (int j = 1; j <= jsize; ++j) for (int i = 1; i <= isize; ++i)
      f(i, j, k) = (signed char)(f(i, j, k) + f2(i, j, k));
    int numbad = 0;
    for (int i = 1; i <= isize; ++i) for (int j = 1; j <= jsize; ++j) for (int k = 1; k <= ksize; ++k)
      if (f(i, j, k) != (signed char)GOODPT) ++numbad;
    return numbad;
  }

  // colate.f:4-78: flagged cells inside the nesting domain, as cell centres (i-.5, j-.5, k-.5)
  void colate(std::vector<double>& badpts, int lcheck, I1& f, I1& dom) {
    const int isize = iregsz[lcheck], jsize = jregsz[lcheck], ksize = kregsz[lcheck];
    for (int k = 1; k <= ksize; ++k) for (int j = 1; j <= jsize; ++j) for (int i = 1; i <= isize; ++i)
      f(i, j, k) = std::min(f(i, j, k), dom(i, j, k));
    badpts.clear();
    for (int k = 1; k <= ksize; ++k) for (int j = 1; j <= jsize; ++j) for (int i = 1; i <= isize; ++i)
      if (f(i, j, k) != (signed char)GOODPT) { badpts.push_back((double)i - .5); badpts.push_back((double)j - .5); badpts.push_back((double)k - .5); }
  }

  // flglvl.f:4-85: returns the flagged points and the nesting domain (i1flags) of level lcheck
  // errest.f:4-141 for the grids of level lcheck: per grid, the old interior (copysol.f) in
  // an array with twice the ghost width, filled by bound at t-dt and coarsened by 2
  // (coarsen.f), stepped by 2*dt at 2*h; the spest copy (tmp) stepped by dt; errf1.f:1-120
  // flags the 2x2x2 blocks whose estimate of component 1 reaches tol (allowflag.f: true),
  // and bufnst.f:21-24 (setflags.f) adds them to the level flags when tol > 0
  void errest(int lcheck, I1& flags) {
    const std::vector<int> G(levelgrids[lcheck]);
    const double hx = hxposs[lcheck], hy = hyposs[lcheck], hz = hzposs[lcheck];
    const double hx2 = 2.0 * hx, hy2 = 2.0 * hy, hz2 = 2.0 * hz;
    const double dt = possk[lcheck], dt2 = 2.0 * dt;  // `2. * dt`: the REAL literal 2. is exact
    const int ng2 = 2 * nghost;
    std::vector<std::vector<double>> bgc(G.size());
    // first loop of errest.f: every grid's coarsened big-step input before any step
    for (size_t n = 0; n < G.size(); ++n) {
      const int mptr = G[n];
      const Node3& g = node[mptr];
      const int nx = g.ihi - g.ilo + 1, ny = g.jhi - g.jlo + 1, nz = g.khi - g.klo + 1;
      const int mitot = nx + 2 * nghost, mjtot = ny + 2 * nghost, mktot = nz + 2 * nghost;
      const int mi2 = nx / 2 + 2 * nghost, mj2 = ny / 2 + 2 * nghost, mk2 = nz / 2 + 2 * nghost;
      const int midub = nx + 4 * nghost, mjdub = ny + 4 * nghost, mkdub = nz + 4 * nghost;
      const double tpre = g.time - dt;
      std::vector<double> dub((size_t)nvar * midub * mjdub * mkdub, 0.0);
      FArr3 V{dub.data(), nvar, midub, mjdub, mkdub};
      const FArr3 Q2{const_cast<double*>(g.q2.data()), nvar, mitot, mjtot, mktot};
      for (int k = nghost + 1; k <= mktot - nghost; ++k)
        for (int j = nghost + 1; j <= mjtot - nghost; ++j)
          for (int i = nghost + 1; i <= mitot - nghost; ++i)
            for (int m = 1; m <= nvar; ++m) V(m, i - nghost + ng2, j - nghost + ng2, k - nghost + ng2) = Q2(m, i, j, k);
      bound(tpre, dub.data(), midub, mjdub, mkdub, mptr, ng2);
      bgc[n].assign((size_t)nvar * mi2 * mj2 * mk2, 0.0);
      FArr3 C{bgc[n].data(), nvar, mi2, mj2, mk2};
      for (int m = 1; m <= nvar; ++m)
        for (int k = 1; k <= mk2; ++k) {
          const int kf = 2 * (k - 1) + 1;
          for (int j = 1; j <= mj2; ++j) {
            const int jf = 2 * (j - 1) + 1;
            for (int i = 1; i <= mi2; ++i) {
              const int iff = 2 * (i - 1) + 1;
              C(m, i, j, k) = (((((((V(m, iff, jf, kf) + V(m, iff + 1, jf, kf)) + V(m, iff, jf + 1, kf)) + V(m, iff + 1, jf + 1, kf)) +
                                  V(m, iff, jf, kf + 1)) + V(m, iff + 1, jf, kf + 1)) + V(m, iff, jf + 1, kf + 1)) + V(m, iff + 1, jf + 1, kf + 1)) / 8.0;
            }
          }
        }
    }
    const double order = (double)((1 << (method[2] + 1)) - 2);
    for (size_t n = 0; n < G.size(); ++n) {
      const int mptr = G[n];
      Node3& g = node[mptr];
      const int nx = g.ihi - g.ilo + 1, ny = g.jhi - g.jlo + 1, nz = g.khi - g.klo + 1;
      const int mitot = nx + 2 * nghost, mjtot = ny + 2 * nghost, mktot = nz + 2 * nghost;
      const int mi2 = nx / 2 + 2 * nghost, mj2 = ny / 2 + 2 * nghost, mk2 = nz / 2 + 2 * nghost;
      double dtnew, cflg;
      {
        const size_t nf = (size_t)nvar * mi2 * mj2 * mk2;
        std::vector<double> fm(nf), fp(nf), gm(nf), gp(nf), hm(nf), hp(nf);
        stepgrid(bgc[n].data(), fm.data(), fp.data(), gm.data(), gp.data(), hm.data(), hp.data(), mi2, mj2, mk2, dt2, dtnew, hx2, hy2, hz2,
                 nullptr, cflg);
      }
      std::vector<double> big = g.tmp;
      {
        const size_t nf = (size_t)nvar * mitot * mjtot * mktot;
        std::vector<double> fm(nf), fp(nf), gm(nf), gp(nf), hm(nf), hp(nf);
        stepgrid(big.data(), fm.data(), fp.data(), gm.data(), gp.data(), hm.data(), hp.data(), mitot, mjtot, mktot, dt, dtnew, hx, hy, hz,
                 nullptr, cflg);
      }
      if (!(tol > 0)) continue;
      const FArr3 F{big.data(), nvar, mitot, mjtot, mktot};
      const FArr3 C{bgc[n].data(), nvar, mi2, mj2, mk2};
      for (int k = nghost + 1, kf = nghost + 1; k <= mk2 - nghost; ++k, kf += 2)
        for (int j = nghost + 1, jf = nghost + 1; j <= mj2 - nghost; ++j, jf += 2)
          for (int i = nghost + 1, iff = nghost + 1; i <= mi2 - nghost; ++i, iff += 2) {
            const double aval = (((((((F(1, iff, jf, kf) + F(1, iff + 1, jf, kf)) + F(1, iff + 1, jf + 1, kf)) + F(1, iff, jf + 1, kf)) +
                                    F(1, iff, jf, kf + 1)) + F(1, iff + 1, jf, kf + 1)) + F(1, iff + 1, jf + 1, kf + 1)) + F(1, iff, jf + 1, kf + 1)) / 8.0;
            const double est = std::fabs((aval - C(1, i, j, k)) / order);
            if (!(est >= tol)) continue;
            // setflags.f: iflags(ibeg+i, ...) with ibeg = ilo - nghost
            for (int dk = 0; dk <= 1; ++dk)
              for (int dj = 0; dj <= 1; ++dj)
                for (int di = 0; di <= 1; ++di) {
                  signed char& f = flags(g.ilo - nghost + iff + di, g.jlo - nghost + jf + dj, g.klo - nghost + kf + dk);
                  f = (signed char)(f + (signed char)BADPT);
                }
          }
    }
  }

  void flglvl(int lcheck, int lbase, std::vector<double>& badpts, I1& i1flags) {
    int idim = iregsz[lbase], jdim = jregsz[lbase], kdim = kregsz[lbase];
    I1 dom1;
    domprep(i1flags, lbase, idim, jdim, kdim);
    domshrink(i1flags, dom1, idim, jdim, kdim);
    for (int lev = lbase + 1; lev <= lcheck; ++lev) {
      domup(i1flags, dom1, idim, jdim, kdim, intratx[lev - 1] * idim, intraty[lev - 1] * jdim, intratz[lev - 1] * kdim, lev - 1);
      idim = intratx[lev - 1] * idim; jdim = intraty[lev - 1] * jdim; kdim = intratz[lev - 1] * kdim;
      domshrink(i1flags, dom1, idim, jdim, kdim);
    }
    domcopy(i1flags, dom1, iregsz[lcheck], jregsz[lcheck], kregsz[lcheck]);
    spest(lcheck, dom1);
    if (flag_richardson) errest(lcheck, dom1);
    const int numbad = bufnst(lcheck, dom1);
    badpts.clear();
    if (numbad > 0) colate(badpts, lcheck, dom1, i1flags);
  }

  // ================================================================ regrid: clustering
  // moment.f:4-70
  void moment(int rect[6], const double* bp, int npt, double& usage) {
    double emx1 = bp[0], emn1 = emx1, emx2 = bp[1], emn2 = emx2, emx3 = bp[2], emn3 = emx3;
    for (int p = 0; p < npt; ++p) {
      const double* q = bp + 3 * p;
      if (q[0] > emx1) emx1 = q[0];
      if (q[0] < emn1) emn1 = q[0];
      if (q[1] > emx2) emx2 = q[1];
      if (q[1] < emn2) emn2 = q[1];
      if (q[2] > emx3) emx3 = q[2];
      if (q[2] < emn3) emn3 = q[2];
    }
    rect[0] = (int)std::lround(emn1 - .5); rect[1] = (int)std::lround(emx1 - .5);
    rect[2] = (int)std::lround(emn2 - .5); rect[3] = (int)std::lround(emx2 - .5);
    rect[4] = (int)std::lround(emn3 - .5); rect[5] = (int)std::lround(emx3 - .5);
    const int s1 = rect[1] - rect[0] + 1, s2 = rect[3] - rect[2] + 1, s3 = rect[5] - rect[4] + 1;
    const int gpall = s1 * s2 * s3;
    usage = (double)npt / gpall;
  }
  // signs.f:4-86 + findcut.f:4-198 ; returns index (0: none) and iside
  void findcut(const double* bp, int ist, int iend, int idim, int jdim, int kdim, int& index, int& iside) {
    std::vector<int> iscr(idim + 2, 0), jscr(jdim + 2, 0), kscr(kdim + 2, 0);
    int ilo = 1, ihi = idim, jlo = 1, jhi = jdim, klo = 1, khi = kdim;
    for (int p = ist; p <= iend; ++p) {
      const double* q = bp + 3 * (p - 1);
      iscr[(int)(q[0] + 1.1)] += 1; jscr[(int)(q[1] + 1.1)] += 1; kscr[(int)(q[2] + 1.1)] += 1;
    }
    for (int t = 1; t <= idim; ++t) if (iscr[t] != 0) { ilo = t; break; }
    for (int t = 1; t <= idim; ++t) if (iscr[idim + 1 - t] != 0) { ihi = idim + 1 - t; break; }
    for (int t = 1; t <= jdim; ++t) if (jscr[t] != 0) { jlo = t; break; }
    for (int t = 1; t <= jdim; ++t) if (jscr[jdim + 1 - t] != 0) { jhi = jdim + 1 - t; break; }
    for (int t = 1; t <= kdim; ++t) if (kscr[t] != 0) { klo = t; break; }
    for (int t = 1; t <= kdim; ++t) if (kscr[kdim + 1 - t] != 0) { khi = kdim + 1 - t; break; }
    for (int i = ilo; i <= ihi; ++i) if (iscr[i] == 0) { index = i; iside = IPLANE; return; }
    for (int j = jlo; j <= jhi; ++j) if (jscr[j] == 0) { index = j; iside = JPLANE; return; }
    for (int k = klo; k <= khi; ++k) if (kscr[k] == 0) { index = k; iside = KPLANE; return; }
    const int minoff = 2, ithres = 2;
    auto lap = [&](std::vector<int>& s, int lo, int hi, int& locmax, int& idx, int& mid) {
      int pre = s[lo];
      for (int i = lo + 1; i <= hi - 1; ++i) { const int cur = s[i]; s[i] = s[i + 1] - 2 * cur + pre; pre = cur; }
      locmax = 0; idx = 0; mid = (lo + hi) / 2;
      for (int i = lo + minoff; i <= hi - minoff + 1; ++i) {
        const int t1 = s[i - 1], t2 = s[i], d = std::abs(t1 - t2);
        if (t1 * t2 < 0) {
          if (d > locmax) { locmax = d; idx = i; }
          else if (d == locmax && std::abs(i - mid) < std::abs(idx - mid)) idx = i;
        }
      }
    };
    int lv[3][4];  // locval(1..4, 1..3): locmax, plane, index, mid
    lap(iscr, ilo, ihi, lv[0][0], lv[0][2], lv[0][3]); lv[0][1] = IPLANE;
    lap(jscr, jlo, jhi, lv[1][0], lv[1][2], lv[1][3]); lv[1][1] = JPLANE;
    lap(kscr, klo, khi, lv[2][0], lv[2][2], lv[2][3]); lv[2][1] = KPLANE;
    for (int a = 0; a < 2; ++a)
      for (int b = a + 1; b < 3; ++b)
        if (lv[a][0] < lv[b][0]) for (int t = 0; t < 4; ++t) std::swap(lv[a][t], lv[b][t]);
    int icount;
    if (lv[0][0] > lv[1][0]) icount = 1;
    else if (lv[1][0] > lv[2][0]) icount = 2;
    else icount = 3;
    if (icount != 1)
      for (int a = 0; a < icount - 1; ++a)
        for (int b = a + 1; b < icount; ++b)
          if (std::abs(lv[a][2] - lv[a][3]) > std::abs(lv[b][2] - lv[b][3])) for (int t = 0; t < 4; ++t) std::swap(lv[a][t], lv[b][t]);
    index = lv[0][2];
    iside = lv[0][1];
    if (lv[0][0] < ithres) index = 0;
  }
  // smartbis.f:4-157 ; numptc is 1-based
  void smartbis(std::vector<double>& bp, int npts, double cutoff, std::vector<int>& numptc, int& nclust, int idim, int jdim, int kdim) {
    nclust = 1;
    numptc.assign(2, 0);
    numptc[1] = npts;
    int icl = 1, ist = 1, iend = numptc[icl];
    while (true) {
      int rect[6]; double usenew;
      moment(rect, bp.data() + 3 * (ist - 1), numptc[icl], usenew);
      bool advance = (usenew >= cutoff);
      int index = 0, iside = 0;
      if (!advance) {
        findcut(bp.data(), ist, iend, idim, jdim, kdim, index, iside);
        if (index == 0) advance = true;
      }
      if (advance) {
        icl = icl + 1;
        if (icl > nclust) break;
        ist = iend + 1;
        iend = ist + numptc[icl] - 1;
        continue;
      }
      const double fmid = index - .5;
      const int idir = (iside == KPLANE) ? 3 : (iside == JPLANE) ? 2 : 1;
      auto c = [&](int p) { return bp[3 * (p - 1) + idir - 1]; };
      auto swp = [&](int a, int b) { for (int d = 0; d < 3; ++d) std::swap(bp[3 * (a - 1) + d], bp[3 * (b - 1) + d]); };
      int itop = ist - 1, ibot = iend + 1, i = ist;
      while (true) {
        if (c(i) < fmid) {
          bool done = false;
          while (true) {
            ibot = ibot - 1;
            if (c(ibot) < fmid) {
              if (ibot == i) { done = true; break; }
              continue;
            }
            swp(ibot, i);
            break;
          }
          if (done) break;
          if (itop + 1 < ibot) continue;
          break;
        } else {
          itop = itop + 1;
          if (itop + 1 >= ibot) break;
          i = i + 1;
        }
      }
      numptc[icl] = itop - ist + 1;
      numptc.insert(numptc.begin() + icl + 1, iend - ibot + 1);
      nclust = nclust + 1;
      iend = itop;
    }
  }
  // nestck.f:4-131: true when the new grid lies in the nesting domain, else splits the cluster
  bool nestck(int mnew, int lbase, std::vector<double>& bp, int ibase, int npts, std::vector<int>& numptc, int icl, int& nclust, I1& dom) {
    if (lbase == 1) return true;
    const Node3& n = node[mnew];
    const int levnew = n.level;
    const int rx = intratx[levnew - 1], ry = intraty[levnew - 1], rz = intratz[levnew - 1];
    bool nested = true;
    for (int k = n.klo / rz + 1; k <= n.khi / rz + 1 && nested; ++k)
      for (int j = n.jlo / ry + 1; j <= n.jhi / ry + 1 && nested; ++j)
        for (int i = n.ilo / rx + 1; i <= n.ihi / rx + 1; ++i)
          if (dom(i, j, k) == 0) { nested = false; break; }
    if (nested) return true;
    if (npts <= 1) throw std::runtime_error("nestck: a single point cannot be properly nested");
    double sidemx = std::max(n.xhi - n.xlo, n.yhi - n.ylo);
    sidemx = std::max(sidemx, n.zhi - n.zlo);
    double rmid; int idir;
    if (n.xhi - n.xlo >= sidemx) { rmid = (double)(float)((n.ihi + n.ilo + 1) / 2.f); rmid = rmid / rx; idir = 1; }
    else if (n.yhi - n.ylo >= sidemx) { rmid = (double)(float)((n.jhi + n.jlo + 1) / 2.f); rmid = rmid / ry; idir = 2; }
    else { rmid = (double)(float)((n.khi + n.klo + 1) / 2.f); rmid = rmid / rz; idir = 3; }
    auto c = [&](int p) { return bp[3 * (ibase + p - 1) + idir - 1]; };
    int ipt = 1, ntop = npts;
    while (true) {
      if (c(ipt) < rmid) { ipt = ipt + 1; if (ipt <= ntop) continue; break; }
      for (int d = 0; d < 3; ++d) std::swap(bp[3 * (ibase + ipt - 1) + d], bp[3 * (ibase + ntop - 1) + d]);
      ntop = ntop - 1;
      if (ipt <= ntop) continue;
      break;
    }
    numptc[icl] = ntop;
    numptc.insert(numptc.begin() + icl + 1, npts - ntop);
    nclust = nclust + 1;
    return false;
  }

  // grdfit.f:4-138
  void grdfit(int lbase, int lcheck, double t) {
    std::vector<double> badpts;
    I1 i1flags;
    flglvl(lcheck, lbase, badpts, i1flags);
    const int npts = (int)badpts.size() / 3;
    if (npts == 0) return;
    const int levnew = lcheck + 1;
    const double hxf = hxposs[levnew], hyf = hyposs[levnew], hzf = hzposs[levnew];
    std::vector<int> numptc;
    int nclust = 0;
    smartbis(badpts, npts, cut, numptc, nclust, iregsz[lcheck], jregsz[lcheck], kregsz[lcheck]);
    int ibase = 0, icl = 1, prv = 0;
    while (icl <= nclust) {
      const int mnew = nodget();
      while (true) {
        int rect[6]; double usage;
        moment(rect, badpts.data() + 3 * ibase, numptc[icl], usage);
        Node3& n = node[mnew];
        n.ilo = rect[0] * intratx[lcheck]; n.jlo = rect[2] * intraty[lcheck]; n.klo = rect[4] * intratz[lcheck];
        n.ihi = (rect[1] + 1) * intratx[lcheck] - 1; n.jhi = (rect[3] + 1) * intraty[lcheck] - 1; n.khi = (rect[5] + 1) * intratz[lcheck] - 1;
        n.xlo = n.ilo * hxf + xlower; n.ylo = n.jlo * hyf + ylower; n.zlo = n.klo * hzf + zlower;
        n.xhi = (n.ihi + 1) * hxf + xlower; n.yhi = (n.jhi + 1) * hyf + ylower; n.zhi = (n.khi + 1) * hzf + zlower;
        n.level = levnew; n.time = t;
        if (nestck(mnew, lbase, badpts, ibase, numptc[icl], numptc, icl, nclust, i1flags)) break;
      }
      if (newstl[levnew] == 0) newstl[levnew] = mnew;
      else node[prv].levelptr = mnew;
      prv = mnew;
      ibase = ibase + numptc[icl];
      icl = icl + 1;
    }
    birect(newstl[levnew]);
  }

  // filval.f:4-153: new patch from the coarse level (minmod-limited), then copies from the old grids
  void filval(int m, int lev) {
    Node3& g = node[m];
    const int mitot = mitot_of(m), mjtot = mjtot_of(m), mktot = mktot_of(m);
    const int levc = lev - 1;
    const int rx = intratx[levc], ry = intraty[levc], rz = intratz[levc];
    const double hxc = hxposs[lev] * rx, hyc = hyposs[lev] * ry, hzc = hzposs[lev] * rz;
    const double xl = g.xlo - hxc, xr = g.xhi + hxc, yf = g.ylo - hyc, yr = g.yhi + hyc, zb = g.zlo - hzc, zt = g.zhi + hzc;
    const int nxg = g.ihi - g.ilo + 1, nyg = g.jhi - g.jlo + 1, nzg = g.khi - g.klo + 1;
    const int mic = nxg / rx + 2, mjc = nyg / ry + 2, mkc = nzg / rz + 2;
    const int iclo = g.ilo / rx - 1, jclo = g.jlo / ry - 1, kclo = g.klo / rz - 1;
    const int ichi = (g.ihi + 1) / rx - 1 + 1, jchi = (g.jhi + 1) / ry - 1 + 1, kchi = (g.khi + 1) / rz - 1 + 1;
    std::vector<double> valc((size_t)nvar * mic * mjc * mkc, 0.0);
    // filval.f:52-58: preintcopy with any periodic direction (the fine copy below is intcopy)
    if (xperdom || yperdom || zperdom) preicall(valc.data(), nullptr, mic, mjc, mkc, iclo, ichi, jclo, jchi, kclo, kchi, levc);
    else icall(valc.data(), nullptr, mic, mjc, mkc, iclo, ichi, jclo, jchi, kclo, kchi, levc, 1, 1, 1);
    bc3amr(valc.data(), mic, mjc, mkc, hxc, hyc, hzc, xl, xr, yf, yr, zb, zt);
    FArr3 V{g.q1.data(), nvar, mitot, mjtot, mktot}, VC{valc.data(), nvar, mic, mjc, mkc};
    std::vector<double> dudx(mic + 1), dudy(mic + 1), dudz(mic + 1);
    for (int k = 2; k <= mkc - 1; ++k)
      for (int j = 2; j <= mjc - 1; ++j)
        for (int iv = 1; iv <= nvar; ++iv) {
          for (int i = 2; i <= mic - 1; ++i) {
            double slp = VC(iv, i + 1, j, k) - VC(iv, i, j, k), slm = VC(iv, i, j, k) - VC(iv, i - 1, j, k);
            double s = std::min(std::fabs(slp), std::fabs(slm)) * dsign(1.0, VC(iv, i + 1, j, k) - VC(iv, i - 1, j, k));
            dudx[i] = (slm * slp > 0.0) ? s : 0.0;
            slp = VC(iv, i, j + 1, k) - VC(iv, i, j, k); slm = VC(iv, i, j, k) - VC(iv, i, j - 1, k);
            s = std::min(std::fabs(slp), std::fabs(slm)) * dsign(1.0, VC(iv, i, j + 1, k) - VC(iv, i, j - 1, k));
            dudy[i] = (slm * slp > 0.0) ? s : 0.0;
            slp = VC(iv, i, j, k + 1) - VC(iv, i, j, k); slm = VC(iv, i, j, k) - VC(iv, i, j, k - 1);
            s = std::min(std::fabs(slp), std::fabs(slm)) * dsign(1.0, VC(iv, i, j, k + 1) - VC(iv, i, j, k - 1));
            dudz[i] = (slm * slp > 0.0) ? s : 0.0;
          }
          for (int kco = 1; kco <= rz; ++kco) {
            const int kfine = (k - 2) * rz + nghost + kco;
            const double zoff = ((double)kco - .5) / rz - .5;
            for (int jco = 1; jco <= ry; ++jco) {
              const int jfine = (j - 2) * ry + nghost + jco;
              const double yoff = ((double)jco - .5) / ry - .5;
              for (int ico = 1; ico <= rx; ++ico) {
                const double xoff = ((double)ico - .5) / rx - .5;
                for (int i = 2; i <= mic - 1; ++i) {
                  const int ifine = (i - 2) * rx + nghost + ico;
                  V(iv, ifine, jfine, kfine) = VC(iv, i, j, k) + xoff * dudx[i] + yoff * dudy[i] + zoff * dudz[i];
                }
              }
            }
          }
        }
    icall(g.q1.data(), nullptr, mitot, mjtot, mktot, g.ilo - nghost, g.ihi + nghost, g.jlo - nghost, g.jhi + nghost, g.klo - nghost,
          g.khi + nghost, lev, 1, 1, 1);
  }

  // gfixup.f:4-180
  void gfixup(int lbase, int lfnew) {
    putsp(lbase, lbase);
    for (int level = lbase + 1; level <= lfine; ++level) {
      putsp(lbase, level);
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].q2.clear(); node[m].has_q2 = false; }
    }
    for (int lcheck = lbase + 1; lcheck <= mxnest; ++lcheck) {
      const double hx = hxposs[lcheck], hy = hyposs[lcheck], hz = hzposs[lcheck];
      std::vector<int> lnew;
      for (int m = newstl[lcheck]; m != 0; m = node[m].levelptr) lnew.push_back(m);
      for (int m : lnew) {
        Node3& g = node[m];
        g.q1.assign(qsize(m), 0.0);
        if (naux > 0) {
          g.aux.assign(asize(m), 0.0);
          setaux(nghost, g.ihi - g.ilo + 1, g.jhi - g.jlo + 1, g.khi - g.klo + 1, g.xlo, g.ylo, g.zlo, hx, hy, hz, g.aux.data());
        }
      }
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
      for (long k = 0; k < (long)lnew.size(); ++k) filval(lnew[k], lcheck);
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
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].q2.assign(qsize(m), 0.0); node[m].has_q2 = true; }
  }

  // regrid.f:4-118
  void regrid(int lbase) {
    int lcheck = std::min(lfine, mxnest - 1);
    int lfnew = lbase;
    for (int i = 1; i <= mxnest; ++i) newstl[i] = 0;
    const double t = node[lstart[lbase]].time;
    while (lcheck >= lbase) {
      grdfit(lbase, lcheck, t);
      if (newstl[lcheck + 1] != 0) lfnew = std::max(lcheck + 1, lfnew);
      lcheck = lcheck - 1;
    }
    gfixup(lbase, lfnew);
    for (int level = lbase; level <= lfine - 1; ++level) { prepf(level + 1); prepc(level); }
    for (int levnew = lbase + 1; levnew <= mxnest; ++levnew) {
      int cnt = 0;
      for (int m = lstart[levnew]; m != 0; m = node[m].levelptr) ++cnt;
      if (cnt > 1) arrangeGrids(levnew, cnt);
    }
    makeGridList();
    for (int levnew = lbase + 1; levnew <= lfine; ++levnew) makeBndryList(levnew);
  }

  // ================================================================ init: ginit.f, domain.f, setgrd.f
  void ginit(int msave, bool first, double start_time) {
    if (msave == 0) return;
    const int level = node[msave].level;
    const double hx = hxposs[level], hy = hyposs[level], hz = hzposs[level];
    for (int mptr = msave; mptr != 0; mptr = node[mptr].levelptr) {
      Node3& g = node[mptr];
      const int mx = g.ihi - g.ilo + 1, my = g.jhi - g.jlo + 1, mz = g.khi - g.klo + 1;
      double* loc;
      if (first) {
        g.q1.assign(qsize(mptr), 0.0);
        if (naux > 0) { g.aux.assign(asize(mptr), 0.0); setaux(nghost, mx, my, mz, g.xlo, g.ylo, g.zlo, hx, hy, hz, g.aux.data()); }
        if (level < mxnest) { g.q2.assign(qsize(mptr), 0.0); g.has_q2 = true; }
        g.time = start_time;
        loc = g.q1.data();
      } else {
        loc = g.q2.data();
      }
      qinit(nghost, mx, my, mz, g.xlo, g.ylo, g.zlo, hx, hy, hz, loc);
    }
  }
  void domain(double start_time) {
    const int ms = nodget();
    Node3& g = node[ms];
    g.xlo = xlower; g.ylo = ylower; g.zlo = zlower; g.xhi = xupper; g.yhi = yupper; g.zhi = zupper;
    g.level = 1; g.levelptr = 0;
    lstart[1] = ms;
    if ((nx / 2) * 2 != nx || (ny / 2) * 2 != ny || (nz / 2) * 2 != nz) throw std::runtime_error("domain: cell counts must be even");
    g.ilo = 0; g.jlo = 0; g.klo = 0; g.ihi = nx - 1; g.jhi = ny - 1; g.khi = nz - 1;
    lfine = 1;
    birect(ms);
    ginit(ms, true, start_time);
    int cnt = 0;
    for (int m = lstart[1]; m != 0; m = node[m].levelptr) ++cnt;
    if (cnt > 1) arrangeGrids(1, cnt);
    makeGridList();
    makeBndryList(1);
    iregsz[1] = nx; jregsz[1] = ny; kregsz[1] = nz;
    for (int level = 2; level <= mxnest; ++level) {
      iregsz[level] = iregsz[level - 1] * intratx[level - 1];
      jregsz[level] = jregsz[level - 1] * intraty[level - 1];
      kregsz[level] = kregsz[level - 1] * intratz[level - 1];
      possk[level] = possk[level - 1] / (double)kratio[level - 1];
    }
  }
  void setgrd(double start_time) {
    if (mxnest == 1) return;
    int levnew = 2;
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
      grdfit(lbase, levold, start_time);
      if (newstl[levnew] != 0) lfnew = levnew;
      ginit(newstl[levnew], true, start_time);
      lstart[levnew] = newstl[levnew];
      lfine = lfnew;
      ginit(lstart[levold], false, start_time);
      int cnt = 0;
      for (int m = lstart[levnew]; m != 0; m = node[m].levelptr) ++cnt;
      if (cnt > 1) arrangeGrids(levnew, cnt);
      makeGridList();
      makeBndryList(levnew);
      levnew = levnew + 1;
    }
    for (int lev = 1; !(lev == mxnest || lev > lfine); ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) { std::swap(node[m].q1, node[m].q2); node[m].time = start_time; }
    for (int level = 1; level <= lfine - 1; ++level) update(lfine - level);
    for (int level = 1; level <= lfine - 1; ++level) { prepf(level + 1); prepc(level); }
  }

  void setbestsrc() {
    mbestsrc.assign(gauges.size(), 0);
    for (size_t i = 0; i < gauges.size(); ++i)
      for (int lev = lfine; lev >= 1 && mbestsrc[i] == 0; --lev)
        for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
          const Node3& g = node[m];
          const Gauge3& G = gauges[i];
          if (G.x >= g.xlo && G.x <= g.xhi && G.y >= g.ylo && G.y <= g.yhi && G.z >= g.zlo && G.z <= g.zhi) { mbestsrc[i] = m; break; }
        }
  }

  // conck.f:4-87 (level 1 mass)
  double conck(int level) {
    const double hx = hxposs[level], hy = hyposs[level], hz = hzposs[level];
    double totmass = 0.0;
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
      const Node3& g = node[m];
      const int mitot = mitot_of(m), mjtot = mjtot_of(m), mktot = mktot_of(m);
      for (int k = nghost + 1; k <= mktot - nghost; ++k)
        for (int j = nghost + 1; j <= mjtot - nghost; ++j)
          for (int i = nghost + 1; i <= mitot - nghost; ++i)
            totmass = totmass + g.q1[(size_t)nvar * ((size_t)(i - 1) + (size_t)mitot * ((j - 1) + (size_t)mjtot * (k - 1)))];
    }
    return totmass * hx * hy * hz;
  }

  // valout.f90 (3D ascii form); valout.f90:140-147 first zeroes |q| < 1e-90 of the interior cells in place
  // src/3d/valout.f90:190-260: fort.aNNNN, the aux arrays in fort.q's layout (headers, then
  // naux values per interior cell), after zeroing |aux| < 1e-90 of the interior cells in place
  void zero_tiny_aux(int lbeg, int lend) {
    for (int level = lbeg; level <= lend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        const int mitot = mitot_of(m), mjtot = mjtot_of(m), mktot = mktot_of(m);
        for (int k = nghost + 1; k <= mktot - nghost; ++k)
          for (int j = nghost + 1; j <= mjtot - nghost; ++j)
            for (int i = nghost + 1; i <= mitot - nghost; ++i)
              for (int ia = 1; ia <= naux; ++ia) {
                double& v = node[m].aux[(size_t)(ia - 1) + (size_t)naux * ((size_t)(i - 1) + (size_t)mitot * ((j - 1) + (size_t)mjtot * (k - 1)))];
                if (std::fabs(v) < 1e-90) v = 0.0;
              }
      }
  }
  void write_aux(int lbeg, int lend) {
    char fn[64];
    std::snprintf(fn, sizeof(fn), "/fort.a%04d", matlabu);
    FILE* f = std::fopen((outdir + fn).c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + outdir + fn);
    for (int level = lbeg; level <= lend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        Node3& g = node[m];
        const int mitot = mitot_of(m), mjtot = mjtot_of(m), mktot = mktot_of(m);
        std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n%6d                 mx\n%6d                 my\n%6d                 mz\n",
                     m, level, g.ihi - g.ilo + 1, g.jhi - g.jlo + 1, g.khi - g.klo + 1);
        std::fprintf(f, "%s    xlow\n%s    ylow\n%s    zlow\n%s    dx\n%s    dy\n%s    dz\n\n", fmtE(g.xlo, 26, 16).c_str(),
                     fmtE(g.ylo, 26, 16).c_str(), fmtE(g.zlo, 26, 16).c_str(), fmtE(hxposs[level], 26, 16).c_str(),
                     fmtE(hyposs[level], 26, 16).c_str(), fmtE(hzposs[level], 26, 16).c_str());
        for (int k = nghost + 1; k <= mktot - nghost; ++k) {
          for (int j = nghost + 1; j <= mjtot - nghost; ++j) {
            for (int i = nghost + 1; i <= mitot - nghost; ++i) {
              for (int ia = 1; ia <= naux; ++ia)
                std::fputs(fmtE(g.aux[(size_t)(ia - 1) + (size_t)naux * ((size_t)(i - 1) + (size_t)mitot * ((j - 1) + (size_t)mjtot * (k - 1)))], 26, 16).c_str(), f);
              std::fputc('\n', f);
            }
            std::fputs("  \n", f);
          }
          std::fputs("  \n", f);
        }
        std::fputs("  \n", f);
      }
    std::fclose(f);
  }

  // Binary form (output_format 3, src/3d/valout.f90:161-172): fort.q holds the grid headers
  // only, fort.b every grid's whole array (ghost cells included, q(m,i,j,k) with m fastest)
  // as raw doubles and, when aux output is due, fort.a the aux arrays likewise; nothing is
  // zeroed.
  void valout_binary(int lbeg, int lend, double t, bool out_aux) {
    char fn[64], fb[64], fa[64];
    std::snprintf(fn, sizeof(fn), "/fort.q%04d", matlabu);
    std::snprintf(fb, sizeof(fb), "/fort.b%04d", matlabu);
    std::snprintf(fa, sizeof(fa), "/fort.a%04d", matlabu);
    FILE* f = std::fopen((outdir + fn).c_str(), "w");
    FILE* b = std::fopen((outdir + fb).c_str(), "wb");
    FILE* a = out_aux ? std::fopen((outdir + fa).c_str(), "wb") : nullptr;
    if (!f || !b || (out_aux && !a)) throw std::runtime_error("cannot write output files in " + outdir);
    int ngrids = 0;
    for (int level = lbeg; level <= lend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        ++ngrids;
        Node3& g = node[m];
        std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n%6d                 mx\n%6d                 my\n%6d                 mz\n",
                     m, level, g.ihi - g.ilo + 1, g.jhi - g.jlo + 1, g.khi - g.klo + 1);
        std::fprintf(f, "%s    xlow\n%s    ylow\n%s    zlow\n%s    dx\n%s    dy\n%s    dz\n\n", fmtE(g.xlo, 26, 16).c_str(),
                     fmtE(g.ylo, 26, 16).c_str(), fmtE(g.zlo, 26, 16).c_str(), fmtE(hxposs[level], 26, 16).c_str(),
                     fmtE(hyposs[level], 26, 16).c_str(), fmtE(hzposs[level], 26, 16).c_str());
        std::fwrite(g.q1.data(), sizeof(double), g.q1.size(), b);
        if (a) std::fwrite(g.aux.data(), sizeof(double), g.aux.size(), a);
      }
    std::fclose(f);
    std::fclose(b);
    if (a) std::fclose(a);
    std::snprintf(fn, sizeof(fn), "/fort.t%04d", matlabu);
    f = std::fopen((outdir + fn).c_str(), "w");
    std::fprintf(f, "%s    time\n%6d                 meqn\n%6d                 ngrids\n%6d                 naux\n%6d                 ndim\n%6d                 nghost\n\n",
                 fmtE(t, 18, 8).c_str(), nvar, ngrids, naux, 3, nghost);
    std::fclose(f);
  }

  void valout(int lbeg, int lend, double t) {
    // valout.f90: aux output when any component is requested, every frame or only at t0
    int naux_out = 0;
    for (int x : output_aux_components) naux_out += x;
    const bool out_aux = naux_out > 0 && (!output_aux_onlyonce || std::fabs(t - t0) < 1e-90);
    if (output_format == 3) {
      if (write_output) valout_binary(lbeg, lend, t, out_aux);
      matlabu = matlabu + 1;
      return;
    }
    if (out_aux) zero_tiny_aux(lbeg, lend);
    for (int level = lbeg; level <= lend; ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        const int mitot = mitot_of(m), mjtot = mjtot_of(m), mktot = mktot_of(m);
        for (int k = nghost + 1; k <= mktot - nghost; ++k)
          for (int j = nghost + 1; j <= mjtot - nghost; ++j)
            for (int i = nghost + 1; i <= mitot - nghost; ++i)
              for (int iv = 1; iv <= nvar; ++iv) {
                double& v = node[m].q1[(size_t)(iv - 1) + (size_t)nvar * ((size_t)(i - 1) + (size_t)mitot * ((j - 1) + (size_t)mjtot * (k - 1)))];
                if (std::fabs(v) < 1e-90) v = 0.0;
              }
      }
    if (write_output) {
      char fn[64];
      std::snprintf(fn, sizeof(fn), "/fort.q%04d", matlabu);
      FILE* f = std::fopen((outdir + fn).c_str(), "w");
      int ngrids = 0;
      for (int level = lbeg; level <= lend; ++level)
        for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
          ++ngrids;
          Node3& g = node[m];
          const int mitot = mitot_of(m), mjtot = mjtot_of(m), mktot = mktot_of(m);
          std::fprintf(f, "%6d                 grid_number\n%6d                 AMR_level\n%6d                 mx\n%6d                 my\n%6d                 mz\n",
                       m, level, g.ihi - g.ilo + 1, g.jhi - g.jlo + 1, g.khi - g.klo + 1);
          std::fprintf(f, "%s    xlow\n%s    ylow\n%s    zlow\n%s    dx\n%s    dy\n%s    dz\n\n", fmtE(g.xlo, 26, 16).c_str(),
                       fmtE(g.ylo, 26, 16).c_str(), fmtE(g.zlo, 26, 16).c_str(), fmtE(hxposs[level], 26, 16).c_str(),
                       fmtE(hyposs[level], 26, 16).c_str(), fmtE(hzposs[level], 26, 16).c_str());
          FArr3 Q{g.q1.data(), nvar, mitot, mjtot, mktot};
          for (int k = nghost + 1; k <= mktot - nghost; ++k) {
            for (int j = nghost + 1; j <= mjtot - nghost; ++j) {
              for (int i = nghost + 1; i <= mitot - nghost; ++i) {
                for (int iv = 1; iv <= nvar; ++iv) std::fputs(fmtE(Q(iv, i, j, k), 26, 16).c_str(), f);
                std::fputc('\n', f);
              }
              std::fputs("  \n", f);
            }
            std::fputs("  \n", f);
          }
          std::fputs("  \n", f);  // src/3d/valout.f90:159
        }
      std::fclose(f);
      if (out_aux) write_aux(lbeg, lend);
      std::snprintf(fn, sizeof(fn), "/fort.t%04d", matlabu);
      f = std::fopen((outdir + fn).c_str(), "w");
      std::fprintf(f, "%s    time\n%6d                 meqn\n%6d                 ngrids\n%6d                 naux\n%6d                 ndim\n%6d                 nghost\n\n",
                   fmtE(t, 18, 8).c_str(), nvar, ngrids, naux, 3, nghost);
      std::fclose(f);
    }
    matlabu = matlabu + 1;
  }

  // ================================================================ tick.f (the 2D cycle, src/2d/tick.f:4-391)
  int max_cycles = 0;
  static double wtime() {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
  }
  void tick() {
    double dtnew[12];
    double* tlevel = tk_tlevel;  // kept across calls: a run split by max_cycles equals one tick.f call
    int ntogo[12];
    int cycles = 0;
    setbestsrc();
    int nextout = 0;
    if (iout == 0) { iout = IINFINITY3; nextout = 0; if (nout > 0) nextout = 1; }
    if (tick_started) nextout = tk_nextout;
    if (!tick_started) {
      tlevel[1] = time;
      for (int i = 2; i <= mxnest; ++i) tlevel[i] = tlevel[1];
    }
    tick_started = true;
    while (!(ncycle >= nstop || time >= tfinal)) {
      double outtime;
      if (nout > 0) outtime = (nextout <= nout) ? tout[nextout - 1] : RINFINITY3;
      else outtime = tfinal;
      bool dumpout = false;
      if (time < outtime && time + (double)1.001f * possk[1] >= outtime) {
        possk[1] = outtime - time;
        for (int i = 2; i <= mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
        if (nout > 0) { nextout = nextout + 1; dumpout = true; }
      }
      int level = 1;
      ntogo[level] = 1;
      for (int i = 1; i <= 10; ++i) dtnew[i] = RINFINITY3;
      while (true) {
        int lbase = -1;
        if (icheck[level] >= kcheck) lbase = level;
        else if (level + 1 >= mxnest) lbase = -1;
        else if (icheck[level + 1] >= kcheck) lbase = level + 1;
        else if (level + 2 >= mxnest) lbase = -1;
        else if (icheck[level + 2] >= kcheck) lbase = level + 2;
        if (lbase > 0) {
          if (!(lbase == mxnest || lbase > lfine)) {
            const double t0c = wtime();
            regrid(lbase);
            regrid_seconds += wtime() - t0c;
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
          } else {
            level = level - 1;
            update(level);
          }
        }
        if (done) break;
      }
      time = time + possk[1];
      ncycle = ncycle + 1;
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
  bool tick_started = false;
  int tk_nextout = 0;
  double tk_tlevel[12] = {0};
  double regrid_seconds = 0;

  // ================================================================ amr3.f90 driver
  void init(const std::string& dir) {
    read_input(dir);
    hxposs[1] = (xupper - xlower) / nx;
    hyposs[1] = (yupper - ylower) / ny;
    hzposs[1] = (zupper - zlower) / nz;
    matlabu = output_t0 ? 0 : 1;
    possk[1] = dt_initial;
    node.assign(10001, Node3());
    for (int k = 1; k <= 10000; ++k) node[k].nextfree = k + 1;
    node[10000].nextfree = 0;
    ndfree = 1;
    lfine = 1;
    for (int i = 0; i < 12; ++i) { lstart[i] = 0; icheck[i] = 0; }
    for (int level = 2; level <= mxnest; ++level) {
      hxposs[level] = hxposs[level - 1] / (double)intratx[level - 1];
      hyposs[level] = hyposs[level - 1] / (double)intraty[level - 1];
      hzposs[level] = hzposs[level - 1] / (double)intratz[level - 1];
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

}  // namespace orc3

// ============================================================== C entry points (tests only)
using orc3::Amr3;
extern "C" {

void* oracle3d_create(const char* dir, const char* outdir, int write_output, int nthreads) {
  try {
    Amr3* a = new Amr3();
    a->outdir = outdir ? outdir : "";
    a->write_output = write_output != 0;
    a->nthreads = nthreads > 0 ? nthreads : 1;
    a->init(dir);
    return a;
  } catch (std::exception& e) {
    std::fprintf(stderr, "oracle3d_create: %s\n", e.what());
    return nullptr;
  }
}
void oracle3d_destroy(void* h) { delete (Amr3*)h; }

// Advance until tfinal; max_cycles > 0 stops after that many coarse steps (a later call continues).
int oracle3d_run(void* h, int max_cycles, double* seconds_out) {
  Amr3* a = (Amr3*)h;
  try {
    a->max_cycles = max_cycles;
    const double t0 = Amr3::wtime();
    a->tick();
    if (seconds_out) *seconds_out = Amr3::wtime() - t0;
    return 0;
  } catch (std::exception& e) {
    std::fprintf(stderr, "oracle3d_run: %s\n", e.what());
    return 1;
  }
}
double oracle3d_time(void* h) { return ((Amr3*)h)->time; }
double oracle3d_cell_updates(void* h) { return ((Amr3*)h)->rvol; }
double oracle3d_mass(void* h) { return ((Amr3*)h)->conck(1); }
double oracle3d_mass0(void* h) { return ((Amr3*)h)->tmass0; }
int oracle3d_lfine(void* h) { return ((Amr3*)h)->lfine; }
int oracle3d_ncycle(void* h) { return ((Amr3*)h)->ncycle; }

// Rows (grid_number, level, ilo, ihi, jlo, jhi, klo, khi) in output order.
int oracle3d_grids(void* h, int* out, int cap) {
  Amr3* a = (Amr3*)h;
  int n = 0;
  for (int level = 1; level <= a->lfine; ++level)
    for (int m = a->lstart[level]; m != 0; m = a->node[m].levelptr) {
      if (out && n < cap) {
        const auto& g = a->node[m];
        int* r = out + 8 * n;
        r[0] = m; r[1] = level; r[2] = g.ilo; r[3] = g.ihi; r[4] = g.jlo; r[5] = g.jhi; r[6] = g.klo; r[7] = g.khi;
      }
      ++n;
    }
  return n;
}
// Interior values in oracle3d_grids order, layout [m][k][j][i] per grid.
long oracle3d_values(void* h, double* out, long cap) {
  Amr3* a = (Amr3*)h;
  long n = 0;
  for (int level = 1; level <= a->lfine; ++level)
    for (int m = a->lstart[level]; m != 0; m = a->node[m].levelptr) {
      const auto& g = a->node[m];
      const int mitot = a->mitot_of(m), mjtot = a->mjtot_of(m), mktot = a->mktot_of(m), ng = a->nghost;
      for (int iv = 1; iv <= a->nvar; ++iv)
        for (int k = ng + 1; k <= mktot - ng; ++k)
          for (int j = ng + 1; j <= mjtot - ng; ++j)
            for (int i = ng + 1; i <= mitot - ng; ++i) {
              if (out && n < cap) out[n] = g.q1[(iv - 1) + (size_t)a->nvar * ((size_t)(i - 1) + (size_t)mitot * ((j - 1) + (size_t)mjtot * (k - 1)))];
              ++n;
            }
    }
  return n;
}
// Gauge samples: rows (gauge_num, level, t, q1..qnvar)
int oracle3d_gauges(void* h, double* out, int cap_rows) {
  Amr3* a = (Amr3*)h;
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
