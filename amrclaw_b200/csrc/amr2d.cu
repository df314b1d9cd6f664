// Host orchestrator of the 2D B200 patch-advance path.
//
// The hierarchy lives on the device: every patch owns two solution buffers
// (ping-pong store1/store2) in one device pool, and flux registers in a second
// pool (the reference's alloc/node store, src/2d/amr_module.f90:30-236,
// igetsp.f, reclam.f, nodget.f). The host keeps only metadata (boxes, level
// lists, grid numbers) and compiles, once per regrid, the device programs that a
// level substep runs:
//   * ghost-fill programs (bound.f90 / filpatch.f90 / prefilp.f90 / intfil.f90 /
//     bc2amr.f90) as staged lists of copy / interpolate / boundary ops,
//   * saveqc programs (saveqc.f, icall.f, cstore.f),
//   * the step work list with the flux-register epilogue entries (fluxsv.f, fluxad.f),
//   * qad jobs (qad.f) and the level-sync plan (update.f, upbnd.f).
// The scheduler (tick.f:4-391) and the regrid decisions stay on the host; the
// flag stencil runs on the device and the clustering on the host
// (regrid.f, grdfit2.f, flagger.f, bufnst2.f, colate2.f, smartbis.f, gfixup.f, filval.f90).
#include "kernels2d.cuh"
#include "params.hpp"
#include "cluster2d.hpp"
#include "flags3d.cuh"
#include "gridindex.hpp"
#include "workpool.hpp"
#include "noalloc2d.cuh"
#include "stepbatch.hpp"
#include "hostutil.hpp"
#include "valout.hpp"
#include "solver.hpp"
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

namespace amrb {

// the "not set" marker of aux values (amr_module.f90:170, a default-real literal)
static const double NEEDS_TO_BE_SET = (double)10.e33f;

// ------------------------------------------------------------------ host patch metadata
struct HPatch {
  int ilo = 0, ihi = 0, jlo = 0, jhi = 0, level = 0, levelptr = 0, nextfree = 0;
  double xlo = 0, xhi = 0, ylo = 0, yhi = 0, time = 0;
  long long q0 = -1, q1 = -1, nq = 0;
  long long aux = -1;                // pool offset of the aux array [m][j][i] (enlarged), -1 without aux
  std::vector<double> haux;          // its host copy (setaux values; icall copies read them)
  long long ffl = -1, nffl = 0;
  int lenbc = 0;
  int cur = 0;
  bool has_cfl = false;
  std::vector<int> listbc;
  std::vector<int> bnd;
  int numflags = 0;
  std::vector<int8_t> flags, dom2;
  int nx() const { return ihi - ilo + 1; }
  int ny() const { return jhi - jlo + 1; }
};

// ------------------------------------------------------------------ device programs
struct FillProg {
  std::vector<ScratchRect> rects;
  std::vector<FillOp> ops;
  std::vector<int> op_stage;
  std::vector<BcOp> bcs;
  std::vector<int> bc_stage;
  int nstages = 0;
  long long scratch_off = -1, scratch_len = 0, scratch_alloc = 0;
  // the scratch starts at zero each run: programs whose rects come from icall copies
  // (saveqc.f, filval.f90) leave uncovered cells at the reference's initial 0
  bool zero_scratch = false;
  std::vector<double> capa;  // coarse kappa of the FIXCAPA ops' source rects (filval.f90's auxc)
  DBuf<ScratchRect> d_rects;
  DBuf<FillOp> d_ops;
  DBuf<FillChunk> d_chunks;
  DBuf<BcOp> d_bcs;
  DBuf<double> d_capa;
  std::vector<int> ch_lo, ch_hi, bc_lo, bc_hi;
  void clear() {
    rects.clear(); ops.clear(); op_stage.clear(); bcs.clear(); bc_stage.clear(); capa.clear();
    nstages = 0; zero_scratch = false;
  }
  int add_rect(int ni, int nj, int nvar) {
    ScratchRect r;
    r.off = scratch_len; r.ni = ni; r.nj = nj;
    scratch_len += Arena::rnd((long long)ni * nj * nvar);
    rects.push_back(r);
    return (int)rects.size() - 1;
  }
  void add_op(const FillOp& o, int st) { ops.push_back(o); op_stage.push_back(st); nstages = std::max(nstages, st + 1); }
  void add_bc(const BcOp& b, int st) { bcs.push_back(b); bc_stage.push_back(st); nstages = std::max(nstages, st + 1); }
};

struct LevelPlan {
  FillProg bound, saveqc;
  std::vector<StepWork> work;
  std::vector<FsvEntry> fsv;
  std::vector<FadEntry> fad;
  std::vector<int> patch_work_lo, patch_work_hi;  // per patch in level order: range in work
  DBuf<StepWork> d_work;
  DBuf<FsvEntry> d_fsv;
  DBuf<FadEntry> d_fad;
  std::vector<QadJob> qad;
  DBuf<QadJob> d_qad;
  std::vector<UpbndCell> upc;
  std::vector<UpbndTerm> upt;
  std::vector<AvgRect> avg;
  DBuf<UpbndCell> d_upc;
  DBuf<UpbndTerm> d_upt;
  DBuf<AvgRect> d_avg;
  std::vector<int> plist;
  DBuf<int> d_plist;
};

struct GaugeRow { int gauge; int level; double t; int slot; };

class Amr2Gpu {
 public:
  RunParams p;
  ProbDev prob{};
  StepParams sp{};
  int nvar = 1, ng = 2;
  bool xperdom = false, yperdom = false;
  double xlower, ylower, xupper, yupper;
  int nxc, nyc;
  // hierarchy
  std::vector<HPatch> node;
  int ndfree = 0;
  int lfine = 1;
  int lstart[12] = {0}, newstl[12] = {0}, listsp[12] = {0}, icheck[12] = {0};
  std::vector<int> lgrids[12];
  GridIndex gidx[12];
  bool gidx_ok[12] = {false};
  double hxposs[12] = {0}, hyposs[12] = {0}, possk[12] = {0};
  int iregsz[12] = {0}, jregsz[12] = {0};
  int intratx[12] = {0}, intraty[12] = {0}, kratio[12] = {0};
  // device
  Arena pool, regs;
  Staging stg;
  WorkPool pool_host;
  HostProf hprof;
  void sync_stream() { AMR_CUDA(cudaStreamSynchronize(st)); stg.reset(); }
  DBuf<PatchDev> d_patches;
  std::vector<PatchDev> h_patches;
  int id_hwm = 1;  // 1 + largest patch id that ever held storage (descriptor table size)
  LevelPlan plan[12];
  FillProg newfill;  // gfixup/filval program of the level being regridded
  // Richardson estimation (errest.f) of the level being flagged: the ghost fill of the
  // big step, the virtual patches of both steps, one byte per 2x2 block
  FillProg rich_prog;
  DBuf<PatchDev> rich_vp;
  DBuf<StepWork> rich_work;
  DBuf<int> rich_rect;
  DBuf<long long> rich_off;
  DBuf<int8_t> rich_out;
  DBuf<unsigned long long> rich_cfl;
  long long rich_buf = -1, rich_len = 0;
  unsigned long long* d_cfl = nullptr;
  double* d_mass = nullptr;
  DBuf<double> d_gauge_out;
  DBuf<int8_t> fl_out;
  DBuf<long long> fl_off;
  DBuf<int> fl_pl;
  cudaStream_t st = nullptr;
  LevelConst lc{};
  // run state
  double time = 0, start_time = 0;
  int ncycle = 0;
#ifdef AMRB_DEBUG_HOOKS
  struct DebugStop {};
  int dbg_stop = 0, dbg_count = 0;
#endif
  double rvol = 0, rvoll[12] = {0};
  double cfl_level = 0, cflmax_run = 0;
  double tmass0 = 0;
  bool batched = true;
  bool record_gauges = true;
  int max_cycles = 0;
  std::vector<int> mbestsrc;
  std::vector<double> glast;
  std::vector<GaugeRow> grows;
  std::vector<GaugeJob> gjobs_pending;
  int gslots = 0;
  double t_regrid = 0, t_step = 0;
  double tr_flags = 0, tr_host = 0, tr_cluster = 0, tr_fill = 0, tr_prep = 0, tr_compile = 0;
  // profiling: CUDA events around every step launch and around each run call
  bool profile = false;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_run0 = nullptr, ev_run1 = nullptr;
  double step_kernel_ms = 0, step_kernel_cells = 0, last_run_ms = 0, run_cells = 0, h2d_bytes = 0;
  // scheduler state kept between run calls (tick.f locals)
  bool tick_started = false;
  int tk_nextout = 0, tk_iout = 0;
  double tk_tlevel[12] = {0};
  long long nsteps_launched = 0, nkernels = 0;
  int frame = 0;
  std::string outdir;
  bool write_output = false;
  int status = 0;

  ~Amr2Gpu() {
    if (st) cudaStreamSynchronize(st);
    if (batch_window_us > 0) StepBatcher::get().leave(batch_member);
    for (auto& G : lgraph) G.reset();
    if (d_sub) cudaFree(d_sub);
    if (h_sub) cudaFreeHost(h_sub);
    if (h_cfl) cudaFreeHost(h_cfl);
    for (int l = 0; l < 12; ++l) free_plan(l);
    newfill.d_rects.free(); newfill.d_ops.free(); newfill.d_chunks.free(); newfill.d_bcs.free();
    rich_prog.d_rects.free(); rich_prog.d_ops.free(); rich_prog.d_chunks.free(); rich_prog.d_bcs.free();
    rich_vp.free(); rich_work.free(); rich_rect.free(); rich_off.free(); rich_out.free(); rich_cfl.free();
    pool.destroy(); regs.destroy();
    if (st) cudaStreamSynchronize(st);
    stg.destroy();
    d_patches.free(); d_gauge_out.free(); fl_out.free(); fl_off.free(); fl_pl.free();
    if (d_cfl) cudaFree(d_cfl);
    if (d_mass) cudaFree(d_mass);
    for (cudaEvent_t e : {ev_a, ev_b, ev_run0, ev_run1}) if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  // ================================================================ setup
  void setup_problem() {
    const std::string& pr = p.problem;
    prob = ProbDev{};
    prob.efix = 1;
    if (pr == "advection_square") {
      prob.solver = SOLVER_ADVECTION; prob.ubar = p.pn("u", 0.5); prob.vbar = p.pn("v", 1.0);
    } else if (pr == "acoustics_cosine" || pr == "acoustics_gauss") {
      prob.solver = SOLVER_ACOUSTICS; prob.rho = p.pn("rho", 1.0); prob.bulk = p.pn("bulk", 4.0);
      prob.cc = std::sqrt(prob.bulk / prob.rho); prob.zz = prob.rho * prob.cc;
    } else if (pr == "euler_quadrants") {
      prob.solver = SOLVER_EULER; prob.gamma = p.pn("gamma", 1.4); prob.gamma1 = prob.gamma - 1.0;
      prob.efix = (int)p.pn("efix", 1.0);
    } else if (pr == "advection_annulus") {
      // tests/advection_2d_annulus: vc advection on the mapped annulus (setprob.f: the two
      // Gaussians of qinit.f)
      prob.solver = SOLVER_VC_ADVECTION;
      const char* names[8] = {"A1", "beta1", "x1", "y1", "A2", "beta2", "x2", "y2"};
      for (int k = 0; k < 8; ++k) ann[k] = p.pn(names[k], 0.0);
    } else throw std::runtime_error("unknown problem '" + pr + "'");
    const bool adv = prob.solver == SOLVER_ADVECTION || prob.solver == SOLVER_VC_ADVECTION;
    const int me = adv ? 1 : prob.solver == SOLVER_ACOUSTICS ? 3 : 4;
    const int mw = adv ? 1 : prob.solver == SOLVER_ACOUSTICS ? 2 : 4;
    if (p.nvar != me || p.mwaves != mw) throw std::runtime_error("num_eqn/num_waves do not match the Riemann solver");
    // aux arrays: amr2.f90:398-425 (one capacity component, typed "capacity"; the types
    // qad.f reads); only problems with a setaux carry them
    prob.naux = p.naux;
    int mc = 0;
    for (int k = 0; k < p.naux; ++k) {
      std::string t = k < (int)p.auxtype.size() ? p.auxtype[k] : "";
      if (t == "leftface") t = "xleft";
      if (t == "bottomface") t = "yleft";
      int code;
      if (t == "xleft") code = AUX_XLEFT;
      else if (t == "yleft") code = AUX_YLEFT;
      else if (t == "capacity") code = AUX_CAPACITY;
      else if (t == "center") code = AUX_CENTER;
      else throw std::runtime_error("unknown type for auxiliary variables: " + t);
      if (code == AUX_CAPACITY) {
        if (mc != 0) throw std::runtime_error("only 1 capacity allowed");
        mc = k + 1;
      }
      if (k < MAXAUX2) prob.auxtype[k] = code;
    }
    if (mc != p.mcapa) throw std::runtime_error("capa_index does not agree with aux_type");
    if (p.naux > 0 && pr != "advection_annulus")
      throw std::runtime_error("problem '" + pr + "' has no aux arrays (setaux)");
    if (p.naux > MAXAUX2) throw std::runtime_error("at most " + std::to_string(MAXAUX2) + " aux components in 2D");
    if (prob.solver == SOLVER_VC_ADVECTION && p.naux < VcAdvection2::NAUX)
      throw std::runtime_error("vc_advection reads aux(1) and aux(2): num_aux must be at least 2");
    sp.prob = prob;
    for (int k = 0; k < MAXVAR; ++k) sp.mthlim[k] = k < (int)p.mthlim.size() ? p.mthlim[k] : 0;
    sp.order = p.order; sp.trans = p.trans; sp.use_fwaves = p.use_fwaves ? 1 : 0; sp.mcapa = p.mcapa;
    sp.split = p.dimsplit;
  }

  // amrgpu_set_solver: rpn2/rpt2 plugin by name with its /cparam/ constants.
  //   advection       [u, v]         (examples/advection_2d_square/setprob.f:4, /cparam/ ubar,vbar)
  //   acoustics       [rho, bulk]    (/cparam/ rho,bulk,cc,zz of the acoustics solvers)
  //   euler_roe_efix  [gamma] or [gamma, efix]  (examples/euler_2d_quadrants/setprob.f:7)
  //   vc_advection    []             (velocities are aux(1), aux(2); tests/advection_2d_annulus)
  // No constants keep the current ones. The equations and waves of the run must match.
  void set_solver(const std::string& name, const std::vector<double>& v) {
    ProbDev q = prob;
    auto need = [&](int me, int mw, size_t n0, size_t n1) {
      if (p.nvar != me || p.mwaves != mw)
        throw std::invalid_argument("Riemann solver '" + name + "' needs num_eqn = " + std::to_string(me) +
                                    " and num_waves = " + std::to_string(mw));
      if (!v.empty() && v.size() != n0 && v.size() != n1)
        throw std::invalid_argument("Riemann solver '" + name + "': wrong number of constants");
    };
    if (name == "advection") {
      need(1, 1, 2, 2);
      q.solver = SOLVER_ADVECTION;
      if (!v.empty()) { q.ubar = v[0]; q.vbar = v[1]; }
    } else if (name == "acoustics") {
      need(3, 2, 2, 2);
      q.solver = SOLVER_ACOUSTICS;
      if (!v.empty()) {
        if (!(v[0] > 0.0) || !(v[1] > 0.0)) throw std::invalid_argument("acoustics: rho and bulk must be positive");
        q.rho = v[0]; q.bulk = v[1];
        q.cc = std::sqrt(q.bulk / q.rho); q.zz = q.rho * q.cc;
      }
    } else if (name == "euler_roe_efix") {
      need(4, 4, 1, 2);
      q.solver = SOLVER_EULER;
      if (!v.empty()) {
        if (!(v[0] > 1.0)) throw std::invalid_argument("euler_roe_efix: gamma must exceed 1");
        q.gamma = v[0]; q.gamma1 = q.gamma - 1.0;
        if (v.size() == 2) q.efix = v[1] != 0.0 ? 1 : 0;
      }
    } else if (name == "vc_advection") {
      need(1, 1, 0, 0);
      if (p.naux < VcAdvection2::NAUX) throw std::invalid_argument("vc_advection reads aux(1) and aux(2): the run has no aux arrays");
      q.solver = SOLVER_VC_ADVECTION;
    } else {
      throw std::invalid_argument("unknown 2D Riemann solver '" + name + "' (advection, acoustics, euler_roe_efix, vc_advection)");
    }
    if (q.solver != prob.solver)
      throw std::invalid_argument("Riemann solver '" + name + "' does not solve this run's equations");
    prob = q;
    sp.prob = q;
    for (auto& G : lgraph) G.reset();  // captured launches hold the old constants
  }

  // qinit of the supported problems (per-application qinit.f of the reference)
  void qinit(int mx, int my, double xl, double yl, double dx, double dy, std::vector<double>& q) {
    const int mitot = mx + 2 * ng, mjtot = my + 2 * ng;
    q.assign((size_t)nvar * mitot * mjtot, 0.0);
    auto Q = [&](int m, int i, int j) -> double& { return q[(size_t)m * mitot * mjtot + (size_t)(j + ng - 1) * mitot + (i + ng - 1)]; };
    const std::string& pr = p.problem;
    if (pr == "advection_square") {
      const double x0 = p.pn("x0", 0.1), x1 = p.pn("x1", 0.6), y0 = p.pn("y0", 0.1), y1 = p.pn("y1", 0.6);
      for (int j = 1; j <= my; ++j) {
        const double yj = yl + (j - 0.5) * dy;
        for (int i = 1; i <= mx; ++i) {
          const double xi = xl + (i - 0.5) * dx;
          Q(0, i, j) = (xi > x0 && xi < x1 && yj > y0 && yj < y1) ? 1.0 : 0.1;
        }
      }
    } else if (pr == "acoustics_cosine" || pr == "acoustics_gauss") {
      const bool cosine = pr == "acoustics_cosine";
      const double r0 = p.pn("r0", cosine ? 0.5 : 0.3), w = p.pn("width", cosine ? 0.2 : 0.05);
      const double pi = 4.0 * std::atan(1.0);
      for (int i = 1; i <= mx; ++i) {
        const double xc = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j) {
          const double yc = yl + (j - 0.5) * dy;
          const double r = std::sqrt(xc * xc + yc * yc);
          double pv;
          if (cosine) pv = (std::fabs(r - r0) <= w) ? 1.0 + std::cos(pi * (r - r0) / w) : 0.0;
          else { const double z = (r - r0) / w; pv = std::exp(-(z * z)); }
          Q(0, i, j) = pv; Q(1, i, j) = 0.0; Q(2, i, j) = 0.0;
        }
      }
    } else if (pr == "advection_annulus") {
      // tests/advection_2d_annulus/qinit.f: two Gaussians at the mapped cell centre
      for (int i = 1; i <= mx; ++i) {
        const double xc = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j) {
          const double yc = yl + (j - 0.5) * dy;
          double xp, yp;
          mapc2p_annulus(xc, yc, xp, yp);
          Q(0, i, j) = ann[0] * std::exp(-ann[1] * ((xp - ann[2]) * (xp - ann[2]) + (yp - ann[3]) * (yp - ann[3]))) +
                       ann[4] * std::exp(-ann[5] * ((xp - ann[6]) * (xp - ann[6]) + (yp - ann[7]) * (yp - ann[7])));
        }
      }
    } else if (pr == "euler_quadrants") {
      const double rpp[5] = {0, 1.5, 0.3, 0.029032258064516, 0.3};
      const double rpr[5] = {0, 1.5, 0.532258064516129, 0.137992831541219, 0.532258064516129};
      const double rpu[5] = {0, 0.0, 1.206045378311055, 1.206045378311055, 0.0};
      const double rpv[5] = {0, 0.0, 0.0, 1.206045378311055, 1.206045378311055};
      const double g1 = prob.gamma - 1.0, xs = p.pn("xs", 0.8), ys = p.pn("ys", 0.8);
      for (int i = 1; i <= mx; ++i) {
        const double xc = xl + (i - 0.5) * dx;
        for (int j = 1; j <= my; ++j) {
          const double yc = yl + (j - 0.5) * dy;
          int iq = 1;
          if (xc >= xs && yc >= ys) iq = 1;
          if (xc < xs && yc >= ys) iq = 2;
          if (xc < xs && yc < ys) iq = 3;
          if (xc >= xs && yc < ys) iq = 4;
          Q(0, i, j) = rpr[iq]; Q(1, i, j) = rpr[iq] * rpu[iq]; Q(2, i, j) = rpr[iq] * rpv[iq];
          Q(3, i, j) = rpp[iq] / g1 + 0.5 * rpr[iq] * (rpu[iq] * rpu[iq] + rpv[iq] * rpv[iq]);
        }
      }
    }
  }

  // tests/advection_2d_annulus/mapc2p.f and stream.f
  static void mapc2p_annulus(double xc, double yc, double& xp, double& yp) {
    xp = xc * std::cos(yc);
    yp = xc * std::sin(yc);
  }
  static double stream_annulus(double x, double y) { return 3.1415926535897931 * (x * x + y * y); }
  // setaux of the problem for an array of (mx + 2 mbc) x (my + 2 mbc) cells whose interior
  // starts at (xlow, ylow): tests/advection_2d_annulus/setaux.f, the edge velocities by
  // differencing the stream function between mapped corners and kappa = mapped area /
  // (dxc dyc). It sets every cell. Layout [m][j][i].
  void setaux(int mbc, int mx, int my, double xlow, double ylow, double dxc, double dyc, std::vector<double>& aux) const {
    const int mi = mx + 2 * mbc, mj = my + 2 * mbc;
    const size_t plane = (size_t)mi * mj;
    aux.assign((size_t)p.naux * plane, 0.0);
    for (int j = 1 - mbc; j <= my + mbc; ++j)
      for (int i = 1 - mbc; i <= mx + mbc; ++i) {
        double xc[5], yc[5], xp[5], yp[5];
        xc[0] = xlow + (i - 1) * dxc; yc[0] = ylow + (j - 1) * dyc;
        xc[1] = xc[0]; yc[1] = yc[0] + dyc;
        xc[2] = xc[0] + dxc; yc[2] = yc[0] + dyc;
        xc[3] = xc[0] + dxc; yc[3] = yc[0];
        for (int c = 0; c < 4; ++c) mapc2p_annulus(xc[c], yc[c], xp[c], yp[c]);
        const size_t k = (size_t)(j + mbc - 1) * mi + (i + mbc - 1);
        aux[k] = (stream_annulus(xp[1], yp[1]) - stream_annulus(xp[0], yp[0])) / dyc;
        aux[plane + k] = -(stream_annulus(xp[3], yp[3]) - stream_annulus(xp[0], yp[0])) / dxc;
        xp[4] = xp[0]; yp[4] = yp[0];
        double area = 0.0;
        for (int c = 0; c < 4; ++c) area = area + 0.5 * (yp[c] + yp[c + 1]) * (xp[c + 1] - xp[c]);
        if (p.naux > 2) aux[2 * plane + k] = area / (dxc * dyc);
      }
  }
  double ann[8] = {0};  // advection_annulus: A1, beta1, x1, y1, A2, beta2, x2, y2

  // ================================================================ node numbers (nodget.f / putnod.f)
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
    node[m] = HPatch();
    return m;
  }
  void putnod(int m) { node[m].nextfree = ndfree; ndfree = m; }

  int mitot(int m) const { return node[m].nx() + 2 * ng; }
  int mjtot(int m) const { return node[m].ny() + 2 * ng; }

  // Patch pool offsets count elements of the storage type: doubles, or floats in the FP32
  // form (two per pool double; the pool's 32-double rounding keeps them 256-byte aligned).
  bool f32 = false;
  long long palloc(long long n) { return f32 ? pool.alloc((n + 1) / 2) * 2 : pool.alloc(n); }
  void pfree(long long off, long long n) {
    if (off < 0) return;
    if (f32) pool.release(off / 2, (n + 1) / 2); else pool.release(off, n);
  }
  size_t elem() const { return f32 ? sizeof(float) : sizeof(double); }

  // storage of a new patch; with aux arrays its aux is set by setaux on the patch
  // (ginit.f:48-58; filval.f90:112-130, whose copies from the old grids the problem's
  // setaux overwrites) and uploaded
  void alloc_patch(int m) {
    id_hwm = std::max(id_hwm, m + 1);
    HPatch& g = node[m];
    g.nq = (long long)nvar * mitot(m) * mjtot(m);
    g.q0 = palloc(g.nq);
    g.q1 = palloc(g.nq);
    g.cur = 0;
    g.aux = -1;
    g.haux.clear();
    if (p.naux > 0) {
      setaux(ng, g.nx(), g.ny(), g.xlo, g.ylo, hxposs[g.level], hyposs[g.level], g.haux);
      g.aux = palloc((long long)g.haux.size());
      upload_to(reinterpret_cast<char*>(pool.d) + sizeof(double) * g.aux, g.haux.data(), sizeof(double) * g.haux.size());
    }
  }
  void upload_to(void* dst, const void* src, size_t bytes) {
    if (!bytes) return;
    AMR_CUDA(cudaMemcpyAsync(dst, stg.put(src, bytes, st), bytes, cudaMemcpyHostToDevice, st));
    h2d_bytes += (double)bytes;
  }
  void free_patch(int m) {
    HPatch& g = node[m];
    pfree(g.q0, g.nq); pfree(g.q1, g.nq);
    if (g.aux >= 0) pfree(g.aux, (long long)g.haux.size());
    g.aux = -1;
    g.haux.clear();
    g.q0 = g.q1 = -1;
    if (g.ffl >= 0) regs.release(g.ffl, g.nffl);
    g.ffl = -1;
  }
  long long qcur(int m) const { return node[m].cur ? node[m].q1 : node[m].q0; }

  void sync_descriptors() {
    HPROF("sync_descriptors");
    h_patches.assign(id_hwm, PatchDev{});
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) {
        const HPatch& g = node[m];
        PatchDev& d = h_patches[m];
        d.q[0] = g.q0; d.q[1] = g.q1; d.cur = g.cur; d.ffl = g.ffl; d.aux = g.aux;
        d.ilo = g.ilo; d.ihi = g.ihi; d.jlo = g.jlo; d.jhi = g.jhi; d.klo = d.khi = 0;
        d.mitot = mitot(m); d.mjtot = mjtot(m); d.mktot = 1;
        d.level = g.level; d.lenbc = g.lenbc;
      }
    d_patches.upload(h_patches, st, stg);
  }

  // ================================================================ level lists
  void make_lists() {
    for (int lev = 1; lev <= 11; ++lev) {
      lgrids[lev].clear();
      if (lev > p.mxnest) continue;
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) lgrids[lev].push_back(m);
    }
  }
  // Index of the committed patches of a level (the list from lstart), rebuilt after touch(lev).
  void touch(int lev) { gidx_ok[lev] = false; }
  const GridIndex& GI(int lev) {
    if (!gidx_ok[lev]) {
      std::vector<int> l;
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) l.push_back(m);
      gidx[lev].build(l, [&](int m) { const HPatch& g = node[m]; return std::array<int, 6>{g.ilo, g.ihi, g.jlo, g.jhi, 0, 0}; });
      gidx_ok[lev] = true;
    }
    return gidx[lev];
  }
  // init_bndryList.f:50-107: same-level neighbours touching the ghost region, most recent first
  void make_bndry(int lev) {
    HPROF("make_bndry");
    const GridIndex& X = GI(lev);
    std::vector<int> hits;
    for (int m : lgrids[lev]) {
      HPatch& g = node[m];
      g.bnd.clear();
      X.query2(g.ilo - ng, g.ihi + ng, g.jlo - ng, g.jhi + ng, hits);
      for (size_t k = hits.size(); k-- > 0;)
        if (X.id(hits[k]) != m) g.bnd.push_back(X.id(hits[k]));
    }
  }
  // regrid.f:132-169: order grids by cost, most expensive first, with quick_sort1.f tie breaking
  void arrange(int lev) {
    std::vector<int> gl;
    for (int m = lstart[lev]; m != 0; m = node[m].levelptr) gl.push_back(m);
    const int n = (int)gl.size();
    if (n <= 1) return;
    std::vector<long long> cost(n + 1);
    std::vector<int> ord(n + 1);
    for (int i = 1; i <= n; ++i) cost[i] = (long long)(node[gl[i - 1]].ihi - node[gl[i - 1]].ilo + 3) * (node[gl[i - 1]].jhi - node[gl[i - 1]].jlo + 2);
    qsort_index(ord, n, cost);
    lstart[lev] = gl[ord[n] - 1];
    int prev = lstart[lev];
    for (int i = 1; i <= n - 1; ++i) { node[prev].levelptr = gl[ord[n - i] - 1]; prev = node[prev].levelptr; }
    node[prev].levelptr = 0;
    touch(lev);
  }
  // birect.f:10-120: split patches wider than max1d
  void birect(int m1) {
    int m = m1;
    const int lev = node[m].level;
    const double hx = hxposs[lev], hy = hyposs[lev];
    while (true) {
      const int nx = node[m].nx(), ny = node[m].ny();
      if (nx + 2 * ng > p.max1d) {
        int nxl = nx / 2;
        const int r = lev > 1 ? intratx[lev - 1] : 2;
        nxl = (nxl / r) * r;
        const double cxmid = node[m].xlo + nxl * hx;
        const int mn = nodget();
        HPatch& a = node[m]; HPatch& b = node[mn];
        b.levelptr = a.levelptr; a.levelptr = mn;
        b.ihi = a.ihi; a.ihi = a.ilo + nxl - 1; b.ilo = a.ihi + 1; b.jhi = a.jhi; b.jlo = a.jlo;
        b.xlo = cxmid; b.ylo = a.ylo; b.yhi = a.yhi; b.xhi = a.xhi; a.xhi = cxmid;
        b.time = a.time; b.level = a.level;
      } else if (ny + 2 * ng > p.max1d) {
        int nyl = ny / 2;
        const int r = lev > 1 ? intraty[lev - 1] : 2;
        nyl = (nyl / r) * r;
        const double cymid = node[m].ylo + nyl * hy;
        const int mn = nodget();
        HPatch& a = node[m]; HPatch& b = node[mn];
        b.levelptr = a.levelptr; a.levelptr = mn;
        b.jhi = a.jhi; a.jhi = a.jlo + nyl - 1; b.jlo = a.jhi + 1; b.ihi = a.ihi; b.ilo = a.ilo;
        b.xlo = a.xlo; b.ylo = cymid; b.yhi = a.yhi; b.xhi = a.xhi; a.yhi = cymid;
        b.level = a.level; b.time = a.time;
      } else {
        m = node[m].levelptr;
        if (m == 0) break;
      }
    }
  }

  // ================================================================ fill-program compiler
  struct Tgt { int patch, rect, ni, nj; };

  BcOp make_bc(Tgt t, double hx, double hy, double xlo_p, double xhi_p, double ylo_p, double yhi_p, bool& any) {
    BcOp b{};
    b.dst_patch = t.patch; b.dst_rect = t.rect; b.nrow = t.ni; b.ncol = t.nj;
    any = false;
    if (xperdom && yperdom) return b;
    const double hxm = hx * 0.01, hym = hy * 0.01;
    auto chk = [&](int code) { if (code == 0) throw std::runtime_error("user boundary conditions are not provided"); };
    if (xlo_p < xlower - hxm) { b.nxl = (int)((xlower + hxm - xlo_p) / hx); b.bxl = p.mthbc[1]; chk(b.bxl); any = true; }
    if (xhi_p > xupper + hxm) { const int nxr = (int)((xhi_p - xupper + hxm) / hx); b.ibeg = std::max(t.ni - nxr + 1, 1); b.bxr = p.mthbc[2]; chk(b.bxr); any = true; }
    if (ylo_p < ylower - hym) { b.nyb = (int)((ylower + hym - ylo_p) / hy); b.byl = p.mthbc[3]; chk(b.byl); any = true; }
    if (yhi_p > yupper + hym) { const int nyt = (int)((yhi_p - yupper + hym) / hy); b.jbeg = std::max(t.nj - nyt + 1, 1); b.byr = p.mthbc[4]; chk(b.byr); any = true; }
    return b;
  }

  // Runs of cells with mask==0 over an (ni x nj) region, merged into rectangles.
  static void runs(const std::vector<int8_t>& mask, int ni, int nj, std::vector<int>& out /* i0, j0, w, h */) {
    out.clear();
    std::vector<int> prev;  // runs of the previous row as (i0, w, rect index)
    for (int j = 0; j < nj; ++j) {
      std::vector<int> cur;
      int i = 0;
      while (i < ni) {
        if (mask[(size_t)j * ni + i] != 0) { ++i; continue; }
        int k = i;
        while (k < ni && mask[(size_t)j * ni + k] == 0) ++k;
        int ridx = -1;
        for (size_t q = 0; q < prev.size(); q += 3)
          if (prev[q] == i && prev[q + 1] == k - i) { ridx = prev[q + 2]; break; }
        if (ridx >= 0) out[4 * ridx + 3] += 1;
        else { ridx = (int)out.size() / 4; out.push_back(i); out.push_back(j); out.push_back(k - i); out.push_back(1); }
        cur.push_back(i); cur.push_back(k - i); cur.push_back(ridx);
        i = k;
      }
      prev.swap(cur);
    }
  }

  void add_split_ops(FillProg& P, FillOp o, int st) {
    // split tall copies so no op is huge (keeps chunks balanced)
    P.add_op(o, st);
  }

  // filpatch.f90:71-355 as a program; returns the stage at which the region is complete
  int c_filrecur(FillProg& P, int level, Tgt T, int nrowst, int ncolst, int ilo, int ihi, int jlo, int jhi, bool patchOnly, int msrc) {
    const int ni = ihi - ilo + 1, nj = jhi - jlo + 1;
    std::vector<int8_t> used((size_t)ni * nj, 0);
    std::vector<FillOp> copies;
    // intfil.f90:153-260
    std::vector<int> src;
    if (msrc == -1) {
      const GridIndex& X = GI(level);
      std::vector<int> hits;
      X.query2(ilo, ihi, jlo, jhi, hits);
      for (int r : hits) src.push_back(X.id(r));
    } else {
      src = node[msrc].bnd;
    }
    for (int m : src) {
      const HPatch& g = node[m];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi), jxlo = std::max(g.jlo, jlo), jxhi = std::min(g.jhi, jhi);
      if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
      FillOp o{};
      o.kind = FILL_COPY; o.dst_patch = T.patch; o.dst_rect = T.rect;
      o.di0 = nrowst - 1 + (ixlo - ilo); o.dj0 = ncolst - 1 + (jxlo - jlo);
      o.ni = ixhi - ixlo + 1; o.nj = jxhi - jxlo + 1;
      o.src = m; o.si0 = ixlo - g.ilo + ng; o.sj0 = jxlo - g.jlo + ng; o.level = level;
      copies.push_back(o);
      for (int j = jxlo; j <= jxhi; ++j) for (int i = ixlo; i <= ixhi; ++i) used[(size_t)(j - jlo) * ni + (i - ilo)] = 1;
    }
    auto mark = [&](int i0, int i1, int j0, int j1) {
      for (int j = std::max(j0, jlo); j <= std::min(j1, jhi); ++j)
        for (int i = std::max(i0, ilo); i <= std::min(i1, ihi); ++i) used[(size_t)(j - jlo) * ni + (i - ilo)] = 1;
    };
    if (jhi >= jregsz[level]) mark(ilo, ihi, std::max(jregsz[level], jlo), jhi);
    if (jlo < 0) mark(ilo, ihi, jlo, std::min(-1, ncolst + jhi - jlo));
    if (ilo < 0) mark(ilo, std::min(-1, nrowst + ihi - ilo), jlo, jhi);
    if (ihi >= iregsz[level]) mark(std::max(iregsz[level], ilo), ihi, jlo, jhi);
    // trimbd.f90: bounding box of unset cells
    int ui0 = ni, ui1 = -1, uj0 = nj, uj1 = -1;
    for (int j = 0; j < nj; ++j) for (int i = 0; i < ni; ++i)
      if (!used[(size_t)j * ni + i]) { ui0 = std::min(ui0, i); ui1 = std::max(ui1, i); uj0 = std::min(uj0, j); uj1 = std::max(uj1, j); }
    int stage = 0;
    if (ui1 >= 0) {
      if (level == 1) throw std::runtime_error("ghost fill: level 1 cells not covered");
      const int rx = intratx[level - 1], ry = intraty[level - 1];
      const int u0 = ui0 + ilo, u1 = ui1 + ilo, v0 = uj0 + jlo, v1 = uj1 + jlo;
      const int iplo = (u0 - rx + ng * rx) / rx - ng, iphi = (u1 + rx) / rx;
      const int jplo = (v0 - ry + ng * ry) / ry - ng, jphi = (v1 + ry) / ry;
      const int mic = iphi - iplo + 1, mjc = jphi - jplo + 1;
      const int R = P.add_rect(mic, mjc, nvar);
      Tgt C{-1, R, mic, mjc};
      const bool sticks = (iplo < 0 || jplo < 0 || iphi >= iregsz[level - 1] || jphi >= jregsz[level - 1]);
      int cst;
      if ((xperdom || yperdom) && sticks) cst = c_prefil(P, level - 1, C, iplo, iphi, jplo, jphi, iplo, jplo);
      else cst = c_filrecur(P, level - 1, C, 1, 1, iplo, iphi, jplo, jphi, true, -1);
      stage = cst + 1;
      std::vector<int> rr;
      runs(used, ni, nj, rr);
      for (size_t k = 0; k < rr.size(); k += 4) {
        FillOp o{};
        o.kind = FILL_INTERP; o.dst_patch = T.patch; o.dst_rect = T.rect;
        o.di0 = nrowst - 1 + rr[k]; o.dj0 = ncolst - 1 + rr[k + 1]; o.ni = rr[k + 2]; o.nj = rr[k + 3];
        o.src = R; o.si0 = ilo + rr[k]; o.sj0 = jlo + rr[k + 1]; o.level = level; o.cilo = iplo; o.cjlo = jplo;
        P.add_op(o, stage);
      }
    }
    for (auto& o : copies) P.add_op(o, stage);
    if (patchOnly) {
      bool any;
      const double dx = hxposs[level], dy = hyposs[level];
      BcOp b = make_bc(T, dx, dy, xlower + ilo * dx, xlower + (ihi + 1) * dx, ylower + jlo * dy, ylower + (jhi + 1) * dy, any);
      if (any) P.add_bc(b, stage);
    }
    return stage;
  }

  // prefilp.f90:18-214: periodic pieces filled at wrapped indices, then copied into place
  int c_prefil(FillProg& P, int level, Tgt T, int ilo, int ihi, int jlo, int jhi, int iglo, int jglo) {
    int ist[3], iend[3], jst[3], jend[3], ish[3], jsh[3];
    if (xperdom) { ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[level]; iend[0] = -1; iend[1] = iregsz[level] - 1; iend[2] = ihi; ish[0] = iregsz[level]; ish[1] = 0; ish[2] = -iregsz[level]; }
    else { ist[0] = iregsz[level]; ist[1] = ilo; ist[2] = iregsz[level]; iend[0] = -1; iend[1] = ihi; iend[2] = -1; ish[0] = ish[1] = ish[2] = 0; }
    if (yperdom) { jst[0] = jlo; jst[1] = 0; jst[2] = jregsz[level]; jend[0] = -1; jend[1] = jregsz[level] - 1; jend[2] = jhi; jsh[0] = jregsz[level]; jsh[1] = 0; jsh[2] = -jregsz[level]; }
    else { jst[0] = jregsz[level]; jst[1] = jlo; jst[2] = jregsz[level]; jend[0] = -1; jend[1] = jhi; jend[2] = -1; jsh[0] = jsh[1] = jsh[2] = 0; }
    int done = 0;
    for (int a = 0; a < 3; ++a) {
      const int i1 = std::max(ilo, ist[a]), i2 = std::min(ihi, iend[a]);
      if (i1 > i2) continue;
      for (int b = 0; b < 3; ++b) {
        const int j1 = std::max(jlo, jst[b]), j2 = std::min(jhi, jend[b]);
        if (j1 > j2) continue;
        const int mi = i2 - i1 + 1, mj = j2 - j1 + 1;
        const int R = P.add_rect(mi, mj, nvar);
        const int s = c_filrecur(P, level, Tgt{-1, R, mi, mj}, 1, 1, i1 + ish[a], i2 + ish[a], j1 + jsh[b], j2 + jsh[b], true, -1);
        FillOp o{};
        o.kind = FILL_PIECE; o.dst_patch = T.patch; o.dst_rect = T.rect;
        o.di0 = i1 - iglo; o.dj0 = j1 - jglo; o.ni = mi; o.nj = mj; o.src = R; o.si0 = 0; o.sj0 = 0;
        P.add_op(o, s + 1);
        done = std::max(done, s + 1);
      }
    }
    return done;
  }

  // Appends program S after the ops already in D (rect indices and scratch offsets shifted).
  static void merge_prog(FillProg& D, const FillProg& S) {
    const int r0 = (int)D.rects.size();
    const long long s0 = D.scratch_len;
    for (ScratchRect r : S.rects) { r.off += s0; D.rects.push_back(r); }
    D.scratch_len += S.scratch_len;
    const int c0 = (int)D.capa.size();
    D.capa.insert(D.capa.end(), S.capa.begin(), S.capa.end());
    for (size_t k = 0; k < S.ops.size(); ++k) {
      FillOp o = S.ops[k];
      if (o.dst_patch < 0) o.dst_rect += r0;
      if (o.kind != FILL_COPY) o.src += r0;
      if (o.kind == FILL_FIXCAPA) o.capa0 += c0;
      D.add_op(o, S.op_stage[k]);
    }
    for (size_t k = 0; k < S.bcs.size(); ++k) {
      BcOp b = S.bcs[k];
      if (b.dst_patch < 0) b.dst_rect += r0;
      D.add_bc(b, S.bc_stage[k]);
    }
  }

  // bound.f90:51-158 for every patch of the level: compiled per patch on the host
  // threads, then joined in level order.
  void compile_bound(int lev) {
    ++plan_gen[lev];
    HPROF("compile_bound");
    FillProg& P = plan[lev].bound;
    P.clear();
    P.scratch_len = 0;
    for (int l = 1; l <= lev; ++l) GI(l);
    const std::vector<int>& G = lgrids[lev];
    std::vector<FillProg> part(G.size());
    pool_host.run((int)G.size(), [&](int k) { compile_bound_patch(part[k], lev, G[k]); });
    for (auto& q : part) merge_prog(P, q);
    upload_prog(P);
  }
  void compile_bound_patch(FillProg& P, int lev, int m) {
    P.scratch_len = 0;
    bound_strips(P, lev, m, Tgt{m, -1, mitot(m), mjtot(m)}, ng);
  }
  // bound.f90:51-158 with ghost width gw into target T (the enlarged array of patch m, or
  // a scratch rect of the same shape): the four strips, then the physical boundaries
  void bound_strips(FillProg& P, int lev, int m, Tgt T, int gw) {
    const HPatch& g = node[m];
    const double hx = hxposs[lev], hy = hyposs[lev];
    const int mi = T.ni, mj = T.nj;
    int s = 0;
    double xl = g.xlo - gw * hx, xr, yb;
    if (xl < xlower && xperdom) s = std::max(s, c_prefil(P, lev, T, g.ilo - gw, g.ilo - 1, g.jlo, g.jhi, g.ilo - gw, g.jlo - gw));
    else s = std::max(s, c_filrecur(P, lev, T, 1, gw + 1, g.ilo - gw, g.ilo - 1, g.jlo, g.jhi, false, m));
    xr = g.xhi + gw * hx;
    if (xr > xupper && xperdom) s = std::max(s, c_prefil(P, lev, T, g.ihi + 1, g.ihi + gw, g.jlo, g.jhi, g.ilo - gw, g.jlo - gw));
    else s = std::max(s, c_filrecur(P, lev, T, mi - gw + 1, gw + 1, g.ihi + 1, g.ihi + gw, g.jlo, g.jhi, false, m));
    xl = g.xlo - gw * hx; xr = g.xhi + gw * hx; yb = g.ylo - gw * hy;
    if ((yb < ylower && yperdom) || ((xl < xlower || xr > xupper) && xperdom))
      s = std::max(s, c_prefil(P, lev, T, g.ilo - gw, g.ihi + gw, g.jlo - gw, g.jlo - 1, g.ilo - gw, g.jlo - gw));
    else s = std::max(s, c_filrecur(P, lev, T, 1, 1, g.ilo - gw, g.ihi + gw, g.jlo - gw, g.jlo - 1, false, m));
    const double yt = g.yhi + gw * hy;
    if ((yt > yupper && yperdom) || ((xl < xlower || xr > xupper) && xperdom))
      s = std::max(s, c_prefil(P, lev, T, g.ilo - gw, g.ihi + gw, g.jhi + 1, g.jhi + gw, g.ilo - gw, g.jlo - gw));
    else s = std::max(s, c_filrecur(P, lev, T, 1, mj - gw + 1, g.ilo - gw, g.ihi + gw, g.jhi + 1, g.jhi + gw, false, m));
    bool any;
    BcOp b = make_bc(T, hx, hy, g.xlo - gw * hx, g.xhi + gw * hx, g.ylo - gw * hy, g.yhi + gw * hy, any);
    if (any) P.add_bc(b, s);
  }

  // prepbigstep.f:28-58 for patch m: copysol.f puts the old interior in the middle of a
  // scratch rect with twice the ghost width, bound.f90 fills that ring at the previous time
  // (same-level sources from the patch's neighbour list, as intfil does with msrc = m)
  void compile_bigstep_patch(FillProg& P, int lev, int m) {
    P.scratch_len = 0;
    const HPatch& g = node[m];
    const int gw = 2 * ng, ni = g.nx() + 2 * gw, nj = g.ny() + 2 * gw;
    const int R = P.add_rect(ni, nj, nvar);
    FillOp o{};
    o.kind = FILL_COPY; o.dst_patch = -1; o.dst_rect = R;
    o.di0 = gw; o.dj0 = gw; o.ni = g.nx(); o.nj = g.ny();
    o.src = m; o.si0 = ng; o.sj0 = ng; o.level = lev;  // the time mode of level lev picks the old values
    P.add_op(o, 0);
    bound_strips(P, lev, m, Tgt{-1, R, ni, nj}, gw);
  }

  // icall.f / preicall.f: copies of store1 of every grid at `level` into a rect
  void c_icall(FillProg& P, Tgt T, int ilo, int ihi, int jlo, int jhi, int level, int iput, int jput, int st_) {
    const GridIndex& X = GI(level);
    std::vector<int> hits;
    X.query2(ilo, ihi, jlo, jhi, hits);
    for (int r : hits) {
      const int m = X.id(r);
      const HPatch& g = node[m];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi), jxlo = std::max(g.jlo, jlo), jxhi = std::min(g.jhi, jhi);
      if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
      FillOp o{};
      o.kind = FILL_COPY; o.dst_patch = T.patch; o.dst_rect = T.rect;
      o.di0 = ixlo - ilo + iput - 1; o.dj0 = jxlo - jlo + jput - 1; o.ni = ixhi - ixlo + 1; o.nj = jxhi - jxlo + 1;
      o.src = m; o.si0 = ixlo - g.ilo + ng; o.sj0 = jxlo - g.jlo + ng; o.level = -1;
      P.add_op(o, st_);
    }
  }
  void c_preicall(FillProg& P, Tgt T, int ilo, int ihi, int jlo, int jhi, int level, int st_) {
    int ist[3], iend[3], jst[3], jend[3], ish[3], jsh[3];
    if (xperdom) { ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[level]; iend[0] = -1; iend[1] = iregsz[level] - 1; iend[2] = ihi; ish[0] = iregsz[level]; ish[1] = 0; ish[2] = -iregsz[level]; }
    else { ist[0] = iregsz[level]; ist[1] = ilo; ist[2] = iregsz[level]; iend[0] = -1; iend[1] = ihi; iend[2] = -1; ish[0] = ish[1] = ish[2] = 0; }
    if (yperdom) { jst[0] = jlo; jst[1] = 0; jst[2] = jregsz[level]; jend[0] = -1; jend[1] = jregsz[level] - 1; jend[2] = jhi; jsh[0] = jregsz[level]; jsh[1] = 0; jsh[2] = -jregsz[level]; }
    else { jst[0] = jregsz[level]; jst[1] = jlo; jst[2] = jregsz[level]; jend[0] = -1; jend[1] = jhi; jend[2] = -1; jsh[0] = jsh[1] = jsh[2] = 0; }
    for (int a = 0; a < 3; ++a) {
      const int i1 = std::max(ilo, ist[a]), i2 = std::min(ihi, iend[a]);
      if (i1 > i2) continue;
      for (int b = 0; b < 3; ++b) {
        const int j1 = std::max(jlo, jst[b]), j2 = std::min(jhi, jend[b]);
        if (j1 > j2) continue;
        c_icall(P, T, i1 + ish[a], i2 + ish[a], j1 + jsh[b], j2 + jsh[b], level, i1 - ilo + 1, j1 - jlo + 1, st_);
      }
    }
  }

  // saveqc.f:13-109 for the kids at level lev+1
  void compile_saveqc(int lev) {
    ++plan_gen[lev];
    HPROF("compile_saveqc");
    FillProg& P = plan[lev].saveqc;
    P.clear();
    P.zero_scratch = true;
    P.scratch_len = 0;
    if (lev + 1 > p.mxnest || lstart[lev + 1] == 0) { upload_prog(P); return; }
    const double hxc = hxposs[lev], hyc = hyposs[lev];
    for (int k = lstart[lev + 1]; k != 0; k = node[k].levelptr) {
      const HPatch& g = node[k];
      const int rx = intratx[lev], ry = intraty[lev];
      const int iclo = g.ilo / rx - 1, jclo = g.jlo / ry - 1, ichi = (g.ihi + 1) / rx, jchi = (g.jhi + 1) / ry;
      const int nrow = ichi - iclo + 1, ncol = jchi - jclo + 1;
      const int R = P.add_rect(nrow, ncol, nvar);
      Tgt T{-1, R, nrow, ncol};
      const bool sticks = (iclo < 0 || ichi == iregsz[lev] || jclo < 0 || jchi == jregsz[lev]);
      if (sticks && (xperdom || yperdom)) c_preicall(P, T, iclo, ichi, jclo, jchi, lev, 0);
      else c_icall(P, T, iclo, ichi, jclo, jchi, lev, 1, 1, 0);
      bool any;
      BcOp b = make_bc(T, hxc, hyc, g.xlo - hxc, g.xhi + hxc, g.ylo - hyc, g.yhi + hyc, any);
      if (any) P.add_bc(b, 0);
      FillOp o{};
      o.kind = FILL_RING; o.dst_patch = k; o.dst_rect = -1; o.ni = g.lenbc; o.nj = 1; o.src = R;
      P.add_op(o, 1);
      if (p.naux > 0) ring_aux(k, lev, iclo, jclo, nrow, ncol, sticks);
    }
    upload_prog(P);
  }
  // saveqc.f:58-90 and cstore.f for the aux: the coarse ring's aux, copied from the coarse
  // grids' aux (icall), or set by setaux on the whole ring where it leaves the domain (the
  // problem's setaux sets every cell); stored after svdflx and qc1d of kid k, in cstore's
  // order. The aux does not change between regrids, so it is written when saveqc is compiled.
  void ring_aux(int k, int lev, int iclo, int jclo, int nrow, int ncol, bool sticks) {
    const HPatch& g = node[k];
    const int na = p.naux;
    const double hxc = hxposs[lev], hyc = hyposs[lev];
    std::vector<double> tx;
    if (sticks) setaux(0, nrow, ncol, g.xlo - hxc, g.ylo - hyc, hxc, hyc, tx);
    const size_t rpl = (size_t)nrow * ncol;
    const GridIndex& XC = GI(lev);
    std::vector<int> hits;
    std::vector<double> ac((size_t)na * g.lenbc, NEEDS_TO_BE_SET);
    int index = 0;
    auto put = [&](int ii, int jj) {  // 0-based cell of the ring rect
      double* dst = &ac[(size_t)na * index++];
      if (sticks) {
        for (int m = 0; m < na; ++m) dst[m] = tx[m * rpl + (size_t)jj * nrow + ii];
        return;
      }
      const int I = iclo + ii, J = jclo + jj;
      XC.query2(I, I, J, J, hits);
      for (int r : hits) {
        const HPatch& c = node[XC.id(r)];
        if (I < c.ilo || I > c.ihi || J < c.jlo || J > c.jhi) continue;
        const int mi = c.nx() + 2 * ng, mj = c.ny() + 2 * ng;
        const size_t at = (size_t)(J - c.jlo + ng) * mi + (I - c.ilo + ng);
        for (int m = 0; m < na; ++m) dst[m] = c.haux[(size_t)m * mi * mj + at];
      }
    };
    for (int j = 1; j <= ncol - 2; ++j) put(0, j);
    for (int i = 1; i <= nrow - 2; ++i) put(i, ncol - 1);
    for (int j = 1; j <= ncol - 2; ++j) put(nrow - 1, j);
    for (int i = 1; i <= nrow - 2; ++i) put(i, 0);
    upload_to(regs.d + g.ffl + (long long)2 * nvar * g.lenbc, ac.data(), sizeof(double) * ac.size());
  }

  void upload_prog(FillProg& P) {
    HPROF("upload_prog");
    if (P.scratch_off >= 0) pfree(P.scratch_off, P.scratch_alloc);
    P.scratch_alloc = std::max<long long>(P.scratch_len, 1);
    P.scratch_off = palloc(P.scratch_alloc);
    std::vector<ScratchRect> rects = P.rects;
    for (auto& r : rects) r.off += P.scratch_off;
    P.d_rects.upload(rects, st, stg);
    // order ops and bcs by stage; chunks of <= 128 cells
    std::vector<int> oidx(P.ops.size());
    for (size_t i = 0; i < oidx.size(); ++i) oidx[i] = (int)i;
    std::stable_sort(oidx.begin(), oidx.end(), [&](int a, int b) { return P.op_stage[a] < P.op_stage[b]; });
    std::vector<FillOp> ops;
    std::vector<FillChunk> ch;
    P.ch_lo.assign(P.nstages, 0); P.ch_hi.assign(P.nstages, 0);
    int s = -1;
    for (int k : oidx) {
      const int stg = P.op_stage[k];
      while (s < stg) { ++s; P.ch_lo[s] = (int)ch.size(); P.ch_hi[s] = (int)ch.size(); }
      const int id = (int)ops.size();
      ops.push_back(P.ops[k]);
      const int cells = P.ops[k].ni * P.ops[k].nj;
      for (int c0 = 0; c0 < cells; c0 += 128) ch.push_back(FillChunk{id, c0, std::min(128, cells - c0)});
      P.ch_hi[s] = (int)ch.size();
    }
    while (s + 1 < P.nstages) { ++s; P.ch_lo[s] = P.ch_hi[s] = (int)ch.size(); }
    std::vector<int> bidx(P.bcs.size());
    for (size_t i = 0; i < bidx.size(); ++i) bidx[i] = (int)i;
    std::stable_sort(bidx.begin(), bidx.end(), [&](int a, int b) { return P.bc_stage[a] < P.bc_stage[b]; });
    std::vector<BcOp> bcs;
    P.bc_lo.assign(P.nstages, 0); P.bc_hi.assign(P.nstages, 0);
    s = -1;
    for (int k : bidx) {
      const int stg = P.bc_stage[k];
      while (s < stg) { ++s; P.bc_lo[s] = (int)bcs.size(); P.bc_hi[s] = (int)bcs.size(); }
      bcs.push_back(P.bcs[k]);
      P.bc_hi[s] = (int)bcs.size();
    }
    while (s + 1 < P.nstages) { ++s; P.bc_lo[s] = P.bc_hi[s] = (int)bcs.size(); }
    P.d_ops.upload(ops, st, stg);
    P.d_chunks.upload(ch, st, stg);
    P.d_bcs.upload(bcs, st, stg);
    if (!P.capa.empty()) P.d_capa.upload(P.capa, st, stg);
  }

  void run_prog(FillProg& P, const SrcMode& modes, const SrcMode* modes_dev = nullptr) {
    if (P.zero_scratch && P.scratch_len > 0 && P.nstages > 0)
      AMR_CUDA(cudaMemsetAsync(reinterpret_cast<char*>(pool.d) + elem() * P.scratch_off, 0, elem() * P.scratch_len, st));
    for (int s = 0; s < P.nstages; ++s) {
      if (P.ch_hi[s] > P.ch_lo[s]) {
        FillArgs a{};
        a.pool = pool.d; a.regs = regs.d; a.patches = d_patches.d; a.rects = P.d_rects.d; a.ops = P.d_ops.d;
        a.chunks = P.d_chunks.d + P.ch_lo[s]; a.nchunks = P.ch_hi[s] - P.ch_lo[s]; a.nvar = nvar; a.modes = modes;
        a.modes_dev = modes_dev;
        a.lc = lc; a.xlower = xlower; a.ylower = ylower;
        a.mcapa = p.mcapa; a.capa = P.d_capa.d;
        launch_fill(a, st, f32);
        ++nkernels;
      }
      if (P.bc_hi[s] > P.bc_lo[s]) {
        BcArgs b{};
        b.pool = pool.d; b.patches = d_patches.d; b.rects = P.d_rects.d; b.ops = P.d_bcs.d + P.bc_lo[s];
        b.nops = P.bc_hi[s] - P.bc_lo[s]; b.nvar = nvar;
        launch_bc(b, 0, st, f32);
        launch_bc(b, 1, st, f32);
        nkernels += 2;
      }
    }
  }

  // Two independent programs stage by stage (the bound and saveqc programs of a level:
  // saveqc reads the level's interiors and its own scratch, bound writes the ghost cells
  // and its own scratch): stage s of both in one fill launch, then their boundary ops,
  // both phases, in one launch. Q may be null; P's fills read their time-interpolation
  // modes from modes (or modes_dev), Q's from zero modes.
  void run_prog_pair(FillProg& P, const SrcMode& modes, const SrcMode* modes_dev, FillProg* Q) {
    for (FillProg* X : {&P, Q})
      if (X && X->zero_scratch && X->scratch_len > 0 && X->nstages > 0)
        AMR_CUDA(cudaMemsetAsync(reinterpret_cast<char*>(pool.d) + elem() * X->scratch_off, 0, elem() * X->scratch_len, st));
    const int ns = std::max(P.nstages, Q ? Q->nstages : 0);
    for (int s = 0; s < ns; ++s) {
      FillArgs fa[2]{};
      BcArgs ba[2]{};
      FillProg* X2[2] = {&P, Q};
      for (int k = 0; k < 2; ++k) {
        FillArgs& a = fa[k];
        BcArgs& b = ba[k];
        a.pool = pool.d; a.regs = regs.d; a.patches = d_patches.d; a.nvar = nvar; a.lc = lc; a.xlower = xlower; a.ylower = ylower;
        b.pool = pool.d; b.patches = d_patches.d; b.nvar = nvar;
        FillProg* X = X2[k];
        if (!X || s >= X->nstages) continue;
        a.rects = X->d_rects.d; a.ops = X->d_ops.d; a.chunks = X->d_chunks.d + X->ch_lo[s]; a.nchunks = X->ch_hi[s] - X->ch_lo[s];
        if (k == 0) { a.modes = modes; a.modes_dev = modes_dev; }
        b.rects = X->d_rects.d; b.ops = X->d_bcs.d + X->bc_lo[s]; b.nops = X->bc_hi[s] - X->bc_lo[s];
      }
      if (fa[0].nchunks + fa[1].nchunks > 0) { launch_fill_pair(fa[0], fa[1], st, f32); ++nkernels; }
      if (ba[0].nops + ba[1].nops > 0) { launch_bc_pair(ba[0], ba[1], st, f32); ++nkernels; }
    }
  }

  // ================================================================ step work, registers, update plans
  void compile_step(int lev) {
    ++plan_gen[lev];
    HPROF("compile_step");
    LevelPlan& L = plan[lev];
    L.work.clear(); L.fsv.clear(); L.fad.clear(); L.patch_work_lo.clear(); L.patch_work_hi.clear(); L.qad.clear();
    L.plist = lgrids[lev];
    for (int m : lgrids[lev]) {
      const HPatch& g = node[m];
      const int mx = g.nx(), my = g.ny();
      const int ntx = (mx + TILE2 - 1) / TILE2, nty = (my + TILE2 - 1) / TILE2;
      std::vector<std::vector<FsvEntry>> tf(ntx * nty);
      std::vector<std::vector<FadEntry>> ta(ntx * nty);
      if (g.has_cfl) {
        for (int sp_ = 1; sp_ <= (int)g.listbc.size() / 5; ++sp_) {
          const int* e = &g.listbc[5 * (sp_ - 1)];
          if (e[0] == 0) break;
          FsvEntry f{};
          f.ic = e[0] - ng; f.jc = e[1] - ng; f.side = e[2];
          f.dst = node[e[3]].ffl + (long long)nvar * (e[4] - 1);
          tf[((f.jc - 1) / TILE2) * ntx + (f.ic - 1) / TILE2].push_back(f);
        }
      }
      if (lev > 1 && g.ffl >= 0) {
        const int rx = intratx[lev - 1], ry = intraty[lev - 1];
        if (TILE2 % rx != 0 || TILE2 % ry != 0) throw std::runtime_error("refinement ratio must divide the tile size");
        const int nyc_ = my / ry, nxc_ = mx / rx;
        int seg = 0;
        for (int j = 0; j < nyc_; ++j, ++seg) { FadEntry a{1, j * ry + 1, seg, ry}; ta[(j * ry / TILE2) * ntx + 0].push_back(a); }
        for (int i = 0; i < nxc_; ++i, ++seg) { FadEntry a{2, i * rx + 1, seg, rx}; ta[(nty - 1) * ntx + i * rx / TILE2].push_back(a); }
        for (int j = 0; j < nyc_; ++j, ++seg) { FadEntry a{3, j * ry + 1, seg, ry}; ta[(j * ry / TILE2) * ntx + ntx - 1].push_back(a); }
        for (int i = 0; i < nxc_; ++i, ++seg) { FadEntry a{4, i * rx + 1, seg, rx}; ta[0 * ntx + i * rx / TILE2].push_back(a); }
        L.qad.push_back(QadJob{m, 1, 0, nyc_, 0});
        L.qad.push_back(QadJob{m, 2, nyc_, nxc_, 0});
        L.qad.push_back(QadJob{m, 3, nyc_ + nxc_, nyc_, 0});
        L.qad.push_back(QadJob{m, 4, 2 * nyc_ + nxc_, nxc_, 0});
      }
      L.patch_work_lo.push_back((int)L.work.size());
      for (int ty = 0; ty < nty; ++ty)
        for (int tx = 0; tx < ntx; ++tx) {
          StepWork w{};
          w.patch = m; w.ti0 = tx * TILE2 + 1; w.tj0 = ty * TILE2 + 1;
          auto& F = tf[ty * ntx + tx];
          auto& A = ta[ty * ntx + tx];
          w.fsv_start = (int)L.fsv.size(); w.fsv_count = (int)F.size();
          L.fsv.insert(L.fsv.end(), F.begin(), F.end());
          w.fad_start = (int)L.fad.size(); w.fad_count = (int)A.size();
          L.fad.insert(L.fad.end(), A.begin(), A.end());
          L.work.push_back(w);
        }
      L.patch_work_hi.push_back((int)L.work.size());
    }
    L.d_work.upload(L.work, st, stg);
    L.d_fsv.upload(L.fsv, st, stg);
    L.d_fad.upload(L.fad, st, stg);
    L.d_qad.upload(L.qad, st, stg);
    L.d_plist.upload(L.plist, st, stg);
  }

  // update.f:16-189 + upbnd.f:18-127 for coarse level lev
  void compile_update(int lev) {
    ++plan_gen[lev];
    HPROF("compile_update");
    LevelPlan& L = plan[lev];
    L.upc.clear(); L.upt.clear(); L.avg.clear();
    if (lev >= p.mxnest) { L.d_upc.upload(L.upc, st, stg); L.d_upt.upload(L.upt, st, stg); L.d_avg.upload(L.avg, st, stg); return; }
    GI(lev + 1);
    const std::vector<int>& G = lgrids[lev];
    struct Part { std::vector<UpbndCell> upc; std::vector<UpbndTerm> upt; std::vector<AvgRect> avg; };
    std::vector<Part> part(G.size());
    pool_host.run((int)G.size(), [&](int k) { compile_update_patch(lev, G[k], part[k].upc, part[k].upt, part[k].avg); });
    for (auto& q : part) {
      const int base = (int)L.upt.size();
      for (UpbndCell c : q.upc) { c.first += base; L.upc.push_back(c); }
      L.upt.insert(L.upt.end(), q.upt.begin(), q.upt.end());
      L.avg.insert(L.avg.end(), q.avg.begin(), q.avg.end());
    }
    L.d_upc.upload(L.upc, st, stg); L.d_upt.upload(L.upt, st, stg); L.d_avg.upload(L.avg, st, stg);
  }
  // upbnd.f:62-124 cells (one term per side not yet used, in listbc order) and
  // update.f:95-175 overlap rectangles of coarse patch m
  void compile_update_patch(int lev, int m, std::vector<UpbndCell>& upc, std::vector<UpbndTerm>& upt, std::vector<AvgRect>& avg) {
    const GridIndex& XF = gidx[lev + 1];
    std::vector<int> hits;
    const HPatch& g = node[m];
    if (g.has_cfl) {
      const int mi = mitot(m), mj = mjtot(m);
      std::vector<int> used((size_t)mi * mj, 0), slot((size_t)mi * mj, -1), order;
      std::vector<std::vector<UpbndTerm>> terms;
      for (int s = 1; s <= (int)g.listbc.size() / 5; ++s) {
        const int* e = &g.listbc[5 * (s - 1)];
        if (e[0] == 0) break;
        const int side = e[2];
        const int side1 = side < 5 ? side : (side == 5 ? 2 : 4);
        const int norm = 1 << (side1 - 1);
        const size_t key = (size_t)(e[1] - 1) * mi + (e[0] - 1);
        if ((used[key] / norm) % 2 == 1) continue;
        double sgn = (side == 2 || side == 3 || side == 6) ? -1.0 : 1.0;
        // upbnd.f:104-108: with a capacity array the correction is divided by kappa
        if (p.mcapa > 0) sgn = sgn / g.haux[(size_t)(p.mcapa - 1) * mi * mj + key];
        if (slot[key] < 0) { slot[key] = (int)terms.size(); terms.emplace_back(); order.push_back((int)key); }
        terms[slot[key]].push_back(UpbndTerm{node[e[3]].ffl + (long long)nvar * (e[4] - 1), sgn});
        used[key] += norm;
      }
      for (int key : order) {
        UpbndCell c{};
        c.patch = m; c.ie = key % mi; c.je = key / mi;
        const auto& T = terms[slot[key]];
        c.first = (int)upt.size(); c.count = (int)T.size();
        upt.insert(upt.end(), T.begin(), T.end());
        upc.push_back(c);
      }
    }
    const int rx = intratx[lev], ry = intraty[lev];
    XF.query2(g.ilo * rx, g.ihi * rx + rx - 1, g.jlo * ry, g.jhi * ry + ry - 1, hits);
    for (int r : hits) {
      const int k = XF.id(r);
      const HPatch& f = node[k];
      const int iclo = f.ilo / rx, jclo = f.jlo / ry, ichi = f.ihi / rx, jchi = f.jhi / ry;
      const int iplo = std::max(g.ilo, iclo), jplo = std::max(g.jlo, jclo), iphi = std::min(g.ihi, ichi), jphi = std::min(g.jhi, jchi);
      if (iplo > iphi || jplo > jphi) continue;
      AvgRect a{};
      a.cpatch = m; a.kpatch = k;
      a.ci0 = iplo - g.ilo + ng; a.cj0 = jplo - g.jlo + ng; a.ni = iphi - iplo + 1; a.nj = jphi - jplo + 1;
      a.fi0 = iplo * rx - f.ilo + ng; a.fj0 = jplo * ry - f.jlo + ng;
      avg.push_back(a);
    }
  }

  // prepf.f / prepc.f / setuse.f
  void prepf(int lev) {
    HPROF("prepf");
    std::vector<std::pair<long long, long long>> zr;
    for (int k = lstart[lev]; k != 0; k = node[k].levelptr) {
      HPatch& g = node[k];
      g.lenbc = 2 * (g.nx() / intratx[lev - 1] + g.ny() / intraty[lev - 1]);
      if (g.ffl >= 0) regs.release(g.ffl, g.nffl);
      g.nffl = (long long)(2 * nvar + p.naux) * g.lenbc;  // svdflx, qc1d, auxc1d (saveqc.f's ffluxptr)
      g.ffl = regs.alloc(g.nffl);
      zr.emplace_back(g.ffl, Arena::rnd(g.nffl));
    }
    zero_ranges(regs.d, zr);
  }
  // one cudaMemsetAsync per run of adjacent ranges
  void zero_ranges(double* base, std::vector<std::pair<long long, long long>>& zr) {
    std::sort(zr.begin(), zr.end());
    for (size_t a = 0; a < zr.size();) {
      long long lo = zr[a].first, hi = zr[a].first + zr[a].second;
      size_t b = a + 1;
      while (b < zr.size() && zr[b].first <= hi) { hi = std::max(hi, zr[b].first + zr[b].second); ++b; }
      AMR_CUDA(cudaMemsetAsync(base + lo, 0, sizeof(double) * (hi - lo), st));
      a = b;
    }
  }
  static void setuse(std::vector<int>& lb, int& ispot, int mkid, int ilo, int ihi, int jlo, int jhi, int iclo, int ichi,
                     int jclo, int jchi, int ngh) {
    auto put = [&](int i, int j, int side, int lkid) {
      ++ispot;
      lb.insert(lb.end(), {i, j, side, mkid, lkid});
    };
    const int ist = iclo - 1, iend = ichi + 1, jst = jclo - 1, jend = jchi + 1;
    if (!(ist < ilo)) {
      int lkid = std::max(jlo, jclo) - jclo + 1;
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) put(ist - ilo + ngh + 1, j - jlo + ngh + 1, 3, lkid++);
    }
    if (!(jend > jhi)) {
      int lkid = (jchi - jclo + 1) + std::max(ilo, iclo) - iclo + 1;
      for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + ngh + 1, jend - jlo + ngh + 1, 4, lkid++);
    }
    if (!(iend > ihi)) {
      int lkid = (ichi - iclo + 1) + (jchi - jclo + 1) + std::max(jlo, jclo) - jclo + 1;
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) put(iend - ilo + ngh + 1, j - jlo + ngh + 1, 1, lkid++);
    }
    if (!(jst < jlo)) {
      int lkid = 2 * (jchi - jclo + 1) + (ichi - iclo + 1) + std::max(ilo, iclo) - iclo + 1;
      for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + ngh + 1, jst - jlo + ngh + 1, 2, lkid++);
    }
  }
  void prepc(int lev) {
    HPROF("prepc");
    int maxsp = 0;
    for (int k = lstart[lev + 1]; k != 0; k = node[k].levelptr)
      maxsp += 2 * (node[k].nx() / intratx[lev] + node[k].ny() / intraty[lev]);
    listsp[lev] = maxsp;
    if (maxsp == 0) return;
    const int imax = iregsz[lev] - 1, jmax = jregsz[lev] - 1;
    const GridIndex& XF = GI(lev + 1);
    std::vector<int> hits;
    const int rx = intratx[lev], ry = intraty[lev];
    for (int mp = lstart[lev]; mp != 0; mp = node[mp].levelptr) {
      HPatch& g = node[mp];
      int ispot = 0;
      g.listbc.clear();  // only the entries setuse makes (the reference reserves 5*maxsp per patch)
      g.has_cfl = true;
      // kids within one coarse cell of the patch; periodic images can come from anywhere
      const bool wrap = (xperdom && (g.ilo == 0 || g.ihi == imax)) || (yperdom && (g.jlo == 0 || g.jhi == jmax));
      if (wrap) { hits.resize(XF.size()); for (size_t r = 0; r < hits.size(); ++r) hits[r] = (int)r; }
      else XF.query2((g.ilo - 1) * rx, (g.ihi + 2) * rx - 1, (g.jlo - 1) * ry, (g.jhi + 2) * ry - 1, hits);
      for (int r : hits) {
        const int k = XF.id(r);
        const HPatch& f = node[k];
        const int iclo = f.ilo / intratx[lev], jclo = f.jlo / intraty[lev], ichi = f.ihi / intratx[lev], jchi = f.jhi / intraty[lev];
        const int iplo = std::max(g.ilo, iclo), jplo = std::max(g.jlo, jclo), iphi = std::min(g.ihi, ichi), jphi = std::min(g.jhi, jchi);
        if (iplo <= iphi + 1 && jplo <= jphi + 1) setuse(g.listbc, ispot, k, g.ilo, g.ihi, g.jlo, g.jhi, iclo, ichi, jclo, jchi, ng);
        if (xperdom && g.ilo == 0 && ichi == imax) setuse(g.listbc, ispot, k, g.ilo, g.ihi, g.jlo, g.jhi, iclo - iregsz[lev], ichi - iregsz[lev], jclo, jchi, ng);
        if (xperdom && iclo == 0 && g.ihi == imax) setuse(g.listbc, ispot, k, g.ilo, g.ihi, g.jlo, g.jhi, iclo + iregsz[lev], ichi + iregsz[lev], jclo, jchi, ng);
        if (yperdom && g.jlo == 0 && jchi == jmax) setuse(g.listbc, ispot, k, g.ilo, g.ihi, g.jlo, g.jhi, iclo, ichi, jclo - jregsz[lev], jchi - jregsz[lev], ng);
        if (yperdom && jclo == 0 && g.jhi == jmax) setuse(g.listbc, ispot, k, g.ilo, g.ihi, g.jlo, g.jhi, iclo, ichi, jclo + jregsz[lev], jchi + jregsz[lev], ng);
      }
    }
  }

  void free_plan(int lev) {
    LevelPlan& L = plan[lev];
    for (FillProg* P : {&L.bound, &L.saveqc}) {
      P->d_rects.free(); P->d_ops.free(); P->d_chunks.free(); P->d_bcs.free();
    }
    L.d_work.free(); L.d_fsv.free(); L.d_fad.free(); L.d_qad.free(); L.d_upc.free(); L.d_upt.free(); L.d_avg.free(); L.d_plist.free();
  }

  // Programs of levels finer than lbase change with a regrid of lbase+1..; the
  // saveqc, step and update plans of lbase itself change with its kids. A regrid marks
  // them; every consumer ensures its own plan before use, so a plan is never used stale.
  // The marked plans are compiled while the GPU runs the level substeps that follow
  // (compile_while_busy), the rest on first use. Compiling reads only the hierarchy
  // (rectangles, lists, register offsets), which changes only in a regrid.
  enum { NEED_BOUND = 1, NEED_SAVEQC = 2, NEED_STEP = 4, NEED_UPDATE = 8 };
  int dirty[12] = {0};
  void compile_all(int lbase = 0) {
    sync_descriptors();
    for (int lev = 1; lev <= p.mxnest; ++lev) {
      if (lev > lfine) {
        plan[lev].work.clear(); plan[lev].plist.clear();
        dirty[lev] = 0;
        continue;
      }
      if (lev > lbase) dirty[lev] |= NEED_BOUND;
      if (lev >= lbase) dirty[lev] |= NEED_SAVEQC | NEED_STEP | NEED_UPDATE;
    }
  }
  void ensure(int lev, int what) {
    if (lev < 1 || lev > p.mxnest) return;
    const int todo = dirty[lev] & what;
    if (!todo) return;
    dirty[lev] &= ~todo;
    if (todo & NEED_BOUND) compile_bound(lev);
    if (todo & NEED_SAVEQC) compile_saveqc(lev);
    if (todo & NEED_STEP) compile_step(lev);
    if (todo & NEED_UPDATE) compile_update(lev);
  }
  // every marked plan, before control returns to a caller of the C ABI: the fixed-scratch
  // substep (amrgpu_level_advance_noalloc) then finds its level compiled and allocates nothing
  void ensure_all() { for (int lev = 1; lev <= p.mxnest; ++lev) ensure(lev, NEED_BOUND | NEED_SAVEQC | NEED_STEP | NEED_UPDATE); }
  // While the substep of level lev runs on the GPU the host compiles marked plans, in the
  // order the next consumers want them: the finer levels' substeps, then the updates from
  // the finest down, then the rest. It stops once the stream has drained. No plan compiled
  // here is one the substep in flight reads: that substep's own plans were ensured before
  // its launch, and compiling a plan touches only that plan's buffers and scratch (uploads
  // and stream-ordered reallocations queue behind the substep; a pool growth waits for the
  // device first).
  void compile_while_busy(int lev) {
    auto busy = [&]() {
      const cudaError_t e = cudaStreamQuery(st);
      if (e == cudaErrorNotReady) return true;
      AMR_CUDA(e);
      return false;
    };
    for (int l = lev + 1; l <= lfine; ++l)
      for (int what : {NEED_BOUND, NEED_SAVEQC, NEED_STEP}) {
        if (!(dirty[l] & what)) continue;
        if (!busy()) return;
        ensure(l, what);
      }
    for (int l = lfine; l >= 1; --l)
      if (dirty[l] & NEED_UPDATE) {
        if (!busy()) return;
        ensure(l, NEED_UPDATE);
      }
    for (int l = 1; l <= lfine; ++l)
      for (int what : {NEED_BOUND, NEED_SAVEQC, NEED_STEP}) {
        if (!(dirty[l] & what)) continue;
        if (!busy()) return;
        ensure(l, what);
      }
  }

  // ================================================================ time interpolation modes (intfil.f90:183-232)
  SrcMode modes_for(int level, double t) {
    SrcMode M{};
    for (int l = 1; l <= level; ++l) {
      if (lgrids[l].empty()) continue;
      const double gt = node[lgrids[l][0]].time;
      const double dt = possk[l];
      const double ac = (gt - t) / dt, ai = 1.0 - ac;
      const double eps = 1.0e-4;
      if (ai < -eps || ai > 1.0 + eps) { M.mode[l] = -1; continue; }
      M.alphai[l] = ai; M.alphac[l] = ac;
      if (std::fabs(ai - 1.0) < eps) M.mode[l] = 0;
      else if (std::fabs(ai) < eps) M.mode[l] = 1;
      else M.mode[l] = 2;
      if (M.mode[l] != 0 && l == p.mxnest) M.mode[l] = -2;
    }
    return M;
  }

  SrcMode bound_modes(int lev, double t) {
    SrcMode M = modes_for(lev, t);
    for (int l = 1; l <= lev; ++l)
      if (M.mode[l] < 0 && !lgrids[l].empty() && l != lev + 100) {
        // a level whose time cannot serve this fill; only an error if the program reads it
        M.mode[l] = 0;
      }
    return M;
  }
  void bound_level(int lev, double t) {
    ensure(lev, NEED_BOUND);
    run_prog(plan[lev].bound, bound_modes(lev, t));
  }

  // ---- scalars of a level substep that change from substep to substep; a captured graph
  // reads them from device memory, refreshed by one copy before each replay
  struct Substep2 { SrcMode modes; double dt; };
  Substep2* d_sub = nullptr;  // [12] on the device
  Substep2* h_sub = nullptr;  // [12] pinned
  unsigned long long* h_cfl = nullptr;  // pinned: the CFL read-back of a substep
  // a level's substep as two CUDA graphs around the gauge sampling: pre (ghost fill,
  // saveqc, qad) and post (CFL reset, step, store swap, CFL read-back). Valid while the
  // level's plans and the buffers they point into stay the same.
  struct LevelGraph {
    cudaGraphExec_t pre = nullptr, post = nullptr;
    long long gen = -1;
    int batched = -1;
    const void* ptrs[4] = {};
    long long kpre = 0, kpost = 0;
    void reset() {
      if (pre) cudaGraphExecDestroy(pre);
      if (post) cudaGraphExecDestroy(post);
      pre = post = nullptr; gen = -1;
    }
  };
  LevelGraph lgraph[12];
  bool use_graphs = false;
  // cross-request batching of the level step (amrgpu_set_step_batching): membership in the
  // process's step batcher, the window a leader waits for the other members, and counts of
  // the submissions made and of those that shared their launch with another solve
  StepBatcher::Member batch_member;
  int batch_window_us = 0;
  long long batch_submits = 0, batch_shared = 0, batch_members_seen = 0;
  bool stepped = false;  // a level substep has run (store2 then holds the last step's input)
  long long plan_gen[12] = {0};
  long long graph_captures = 0, graph_replays = 0;

  // the launches before the gauge sampling (ds: read dt and the fill modes from there)
  void launch_pre(int lev, double t, double dt, const Substep2* ds) {
    LevelPlan& L = plan[lev];
    const bool kids = lev + 1 <= p.mxnest && lstart[lev + 1] != 0;
    if (batched) {
      // bound and saveqc of the whole level, their stages sharing launches
      run_prog_pair(L.bound, bound_modes(lev, t), ds ? &ds->modes : nullptr, kids ? &L.saveqc : nullptr);
    } else {
      run_prog(L.bound, bound_modes(lev, t), ds ? &ds->modes : nullptr);
      if (kids) { SrcMode M{}; run_prog(L.saveqc, M); }
    }
    if (lev > 1 && !L.qad.empty()) {
      launch_qad2(prob.solver, pool.d, regs.d, d_patches.d, L.d_qad.d, (int)L.qad.size(), prob, nvar, lc, dt, st, f32,
                  ds ? &ds->dt : nullptr);
      ++nkernels;
    }
  }
  // the patch step (plain = one launch per patch, batched = one launch per level), the
  // store swap and the CFL read-back; timed: bracket the step with ev_a / ev_b
  void launch_post(int lev, double dt, const Substep2* ds, bool timed) {
    LevelPlan& L = plan[lev];
    AMR_CUDA(cudaMemsetAsync(d_cfl, 0, sizeof(unsigned long long), st));
    if (timed) AMR_CUDA(cudaEventRecord(ev_a, st));
    StepArgs a{};
    a.pool = pool.d; a.regs = regs.d; a.patches = d_patches.d; a.fsv = L.d_fsv.d; a.fad = L.d_fad.d;
    a.dt = dt; a.dt_dev = ds ? &ds->dt : nullptr; a.dx = hxposs[lev]; a.dy = hyposs[lev]; a.cflmax = d_cfl; a.sp = sp;
    if (batched) {
      a.work = L.d_work.d; a.nwork = (int)L.work.size(); a.queue = nullptr;
      if (batch_window_us > 0 && !use_graphs && !sp.split) {
        // the level step goes out in one launch with the steps other solves submit meanwhile
        StepBatcher::get().submit(batch_member, a, (int)L.work.size(), st, batch_window_us);
        ++batch_submits;
        batch_members_seen += batch_member.batch_size;
        if (batch_member.batch_size > 1) ++batch_shared;
      } else {
        launch_step2(prob.solver, a, (int)L.work.size(), st, f32);
      }
      ++nkernels;
    } else {
      for (size_t k = 0; k < L.plist.size(); ++k) {
        a.work = L.d_work.d + L.patch_work_lo[k];
        a.nwork = L.patch_work_hi[k] - L.patch_work_lo[k];
        a.queue = nullptr;
        launch_step2(prob.solver, a, a.nwork, st, f32);
        ++nkernels;
      }
    }
    if (timed) AMR_CUDA(cudaEventRecord(ev_b, st));
    launch_flip(d_patches.d, L.d_plist.d, (int)L.plist.size(), st);
    ++nkernels;
    AMR_CUDA(cudaMemcpyAsync(h_cfl, d_cfl, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  }
  // captures the level's two graphs if the current ones do not fit the plans and buffers
  void ensure_graphs(int lev) {
    LevelGraph& G = lgraph[lev];
    const void* ptrs[4] = {pool.d, regs.d, d_patches.d, d_cfl};
    bool ok = G.pre && G.gen == plan_gen[lev] && G.batched == (int)batched;
    for (int k = 0; k < 4 && ok; ++k) ok = G.ptrs[k] == ptrs[k];
    if (ok) return;
    HPROF("graph_capture");
    G.reset();
    const Substep2* ds = d_sub + lev;
    const double t = node[lgrids[lev][0]].time, dt = possk[lev];
    for (int part = 0; part < 2; ++part) {
      cudaGraph_t g = nullptr;
      const long long k0 = nkernels;
      AMR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      if (part == 0) launch_pre(lev, t, dt, ds);
      else launch_post(lev, dt, ds, false);
      AMR_CUDA(cudaStreamEndCapture(st, &g));
      AMR_CUDA(cudaGraphInstantiate(part == 0 ? &G.pre : &G.post, g, 0));
      AMR_CUDA(cudaGraphDestroy(g));
      (part == 0 ? G.kpre : G.kpost) = nkernels - k0;
      nkernels = k0;
    }
    G.gen = plan_gen[lev]; G.batched = (int)batched;
    for (int k = 0; k < 4; ++k) G.ptrs[k] = ptrs[k];
    ++graph_captures;
  }
  // gauges (gauges_module.f90:313-452): sampled before the step on the finest covering grid
  void sample_gauges(int lev) {
    if (record_gauges && !p.gauges.empty()) {
      std::vector<GaugeJob> jobs;
      const double hx = hxposs[lev], hy = hyposs[lev];
      for (size_t i = 0; i < p.gauges.size(); ++i) {
        const int m = mbestsrc[i];
        if (m == 0 || node[m].level != lev) continue;
        const GaugeSpec& G = p.gauges[i];
        const double tg = node[m].time;
        if (tg < G.t1 || tg > G.t2) continue;
        if (tg - glast[i] < G.min_inc) continue;
        const double xlow = node[m].xlo - ng * hx, ylow = node[m].ylo - ng * hy;
        GaugeJob J{};
        J.patch = m; J.ii = (int)(0.5 + (G.x - xlow) / hx); J.jj = (int)(0.5 + (G.y - ylow) / hy);
        const double xc = xlow + (J.ii - 0.5) * hx, yc = ylow + (J.jj - 0.5) * hy;
        J.xoff = (G.x - xc) / hx; J.yoff = (G.y - yc) / hy;
        J.slot = gslots++;
        jobs.push_back(J);
        grows.push_back(GaugeRow{G.num, lev, tg, J.slot});
        glast[i] = tg;
      }
      if (!jobs.empty()) {
        if ((size_t)gslots * nvar > d_gauge_out.cap) {
          DBuf<double> nb; nb.ensure(std::max<size_t>((size_t)gslots * nvar * 2, 4096));
          if (d_gauge_out.d) AMR_CUDA(cudaMemcpyAsync(nb.d, d_gauge_out.d, sizeof(double) * d_gauge_out.cap, cudaMemcpyDeviceToDevice, st));
          d_gauge_out.free(); d_gauge_out = nb;
        }
        DBuf<GaugeJob> dj; dj.upload(jobs, st, stg);
        launch_gauges2(pool.d, d_patches.d, dj.d, (int)jobs.size(), nvar, d_gauge_out.d, st, f32);
        sync_stream();
        dj.free();
      }
    }
  }

  // ================================================================ level substep (advanc.f:10-142)
  // launched directly, or replayed from captured graphs
  double advanc(int lev) {
    HPROF("advanc");
    ensure(lev, NEED_BOUND | NEED_SAVEQC | NEED_STEP);
    LevelPlan& L = plan[lev];
    const double t = node[lgrids[lev][0]].time;
    const double dt = possk[lev];
    if (use_graphs) {
      ensure_graphs(lev);
      Substep2& h = h_sub[lev];
      h.modes = bound_modes(lev, t); h.dt = dt;
      AMR_CUDA(cudaMemcpyAsync(d_sub + lev, &h, sizeof(Substep2), cudaMemcpyHostToDevice, st));
      AMR_CUDA(cudaGraphLaunch(lgraph[lev].pre, st));
      sample_gauges(lev);
      if (profile) AMR_CUDA(cudaEventRecord(ev_a, st));
      AMR_CUDA(cudaGraphLaunch(lgraph[lev].post, st));
      if (profile) AMR_CUDA(cudaEventRecord(ev_b, st));
      nkernels += lgraph[lev].kpre + lgraph[lev].kpost;
      graph_replays += 2;
    } else {
      PhaseTimer tph(hprof);
      tph.next("adv_pre");
      launch_pre(lev, t, dt, nullptr);
      tph.next("adv_gauges");
      sample_gauges(lev);
      tph.next("adv_post");
      launch_post(lev, dt, nullptr, profile);
    }
    {
      HPROF("advanc_compile");
      compile_while_busy(lev);
    }
    {
      HPROF("advanc_sync");
      sync_stream();
    }
    const unsigned long long cbits = *h_cfl;
    double cmax;
    std::memcpy(&cmax, &cbits, sizeof(double));
    // a step block whose bulk copies of its tile did not complete flags the level's
    // Courant number as infinite (no wave speed makes it so)
    if (std::isinf(cmax)) throw std::runtime_error("level step: a tile's staging copies did not complete");
    if (profile) {
      float ms = 0;
      AMR_CUDA(cudaEventElapsedTime(&ms, ev_a, ev_b));
      step_kernel_ms += ms;
      for (int m : lgrids[lev]) step_kernel_cells += (double)node[m].nx() * node[m].ny();
    }
    for (int m : lgrids[lev]) {
      node[m].cur ^= 1;
      node[m].time = node[m].time + dt;
      const double cells = (double)node[m].nx() * node[m].ny();
      rvol += cells; rvoll[lev] += cells;
    }
    cfl_level = cmax;
    cflmax_run = std::max(cflmax_run, cmax);
    ++nsteps_launched;
    stepped = true;
    (void)L;
    return cmax > 0.0 ? dt * p.cfl_desired / cmax : RINF;
  }

  // advanc without device allocation: the bound and saveqc programs run with their
  // scratch rects in the fixed device array (noalloc2d.cu); no gauge sampling, no
  // profiling events, no host timers. Returns dtnew like advanc.
  void run_prog_fixed(FillProg& P, const SrcMode& modes, const double* scratch) {
    if (P.zero_scratch && P.scratch_len > 0 && P.nstages > 0)
      AMR_CUDA(cudaMemsetAsync(const_cast<double*>(scratch), 0, sizeof(double) * P.scratch_len, st));
    for (int s = 0; s < P.nstages; ++s) {
      if (P.ch_hi[s] > P.ch_lo[s]) {
        FillArgs a{};
        a.pool = pool.d; a.regs = regs.d; a.patches = d_patches.d; a.rects = P.d_rects.d; a.ops = P.d_ops.d;
        a.chunks = P.d_chunks.d + P.ch_lo[s]; a.nchunks = P.ch_hi[s] - P.ch_lo[s]; a.nvar = nvar; a.modes = modes;
        a.lc = lc; a.xlower = xlower; a.ylower = ylower;
        launch_fill_fixed(a, scratch, P.scratch_off, st);
        ++nkernels;
      }
      if (P.bc_hi[s] > P.bc_lo[s]) {
        BcArgs b{};
        b.pool = pool.d; b.patches = d_patches.d; b.rects = P.d_rects.d; b.ops = P.d_bcs.d + P.bc_lo[s];
        b.nops = P.bc_hi[s] - P.bc_lo[s]; b.nvar = nvar;
        launch_bc_fixed(b, 0, scratch, P.scratch_off, st);
        launch_bc_fixed(b, 1, scratch, P.scratch_off, st);
        nkernels += 2;
      }
    }
  }
  double advanc_fixed(int lev, const double* scratch) {
    // compiling a plan would allocate (pool rectangles, device lists): every C-ABI exit
    // compiles all of them (ensure_all), so a marked plan here is a broken promise
    if (dirty[lev] & (NEED_BOUND | NEED_SAVEQC | NEED_STEP))
      throw std::invalid_argument("amrgpu_level_advance_noalloc: the level's device programs are not compiled");
    LevelPlan& L = plan[lev];
    const bool kids = lev + 1 <= p.mxnest && lstart[lev + 1] != 0;
    if (L.bound.scratch_len > NOALLOC_SCRATCH_DOUBLES || (kids && L.saveqc.scratch_len > NOALLOC_SCRATCH_DOUBLES))
      throw std::invalid_argument("ghost-fill scratch of this level exceeds the fixed array (4194304 doubles)");
    const double t = node[lgrids[lev][0]].time;
    const double dt = possk[lev];
    SrcMode M = modes_for(lev, t);
    for (int l = 1; l <= lev; ++l)
      if (M.mode[l] < 0 && !lgrids[l].empty()) M.mode[l] = 0;
    run_prog_fixed(L.bound, M, scratch);
    if (kids) { SrcMode Z{}; run_prog_fixed(L.saveqc, Z, scratch); }
    if (lev > 1 && !L.qad.empty()) {
      launch_qad2(prob.solver, pool.d, regs.d, d_patches.d, L.d_qad.d, (int)L.qad.size(), prob, nvar, lc, dt, st, f32);
      ++nkernels;
    }
    AMR_CUDA(cudaMemsetAsync(d_cfl, 0, sizeof(unsigned long long), st));
    StepArgs a{};
    a.pool = pool.d; a.regs = regs.d; a.patches = d_patches.d; a.fsv = L.d_fsv.d; a.fad = L.d_fad.d;
    a.dt = dt; a.dx = hxposs[lev]; a.dy = hyposs[lev]; a.cflmax = d_cfl; a.sp = sp;
    a.work = L.d_work.d; a.nwork = (int)L.work.size(); a.queue = nullptr;
    launch_step2(prob.solver, a, (int)L.work.size(), st, f32);
    launch_flip(d_patches.d, L.d_plist.d, (int)L.plist.size(), st);
    nkernels += 2;
    unsigned long long cbits = 0;
    AMR_CUDA(cudaMemcpyAsync(&cbits, d_cfl, sizeof(cbits), cudaMemcpyDeviceToHost, st));
    sync_stream();
    double cmax;
    std::memcpy(&cmax, &cbits, sizeof(double));
    for (int m : lgrids[lev]) {
      node[m].cur ^= 1;
      node[m].time = node[m].time + dt;
      const double cells = (double)node[m].nx() * node[m].ny();
      rvol += cells; rvoll[lev] += cells;
    }
    cfl_level = cmax;
    cflmax_run = std::max(cflmax_run, cmax);
    ++nsteps_launched;
    stepped = true;
    return cmax > 0.0 ? dt * p.cfl_desired / cmax : RINF;
  }

  void update(int lev) {
    HPROF("update");
    ensure(lev, NEED_UPDATE);
    LevelPlan& L = plan[lev];
    const double area = hxposs[lev] * hyposs[lev];
    launch_upbnd(pool.d, regs.d, d_patches.d, L.d_upc.d, (int)L.upc.size(), L.d_upt.d, area, nvar, st, f32);
    launch_average(pool.d, d_patches.d, L.d_avg.d, (int)L.avg.size(), intratx[lev], intraty[lev], nvar, st, f32, p.mcapa);
    nkernels += 2;
  }

  // ================================================================ regrid (regrid.f / grdfit2.f)
  void setIndices(int ist[3], int iend[3], int jst[3], int jend[3], int ilo, int ihi, int jlo, int jhi, int ish[3], int jsh[3], int lev) {
    ist[0] = ilo; ist[1] = 0; ist[2] = iregsz[lev]; iend[0] = -1; iend[1] = iregsz[lev] - 1; iend[2] = ihi;
    jst[0] = jlo; jst[1] = 0; jst[2] = jregsz[lev]; jend[0] = -1; jend[1] = jregsz[lev] - 1; jend[2] = jhi;
    if (xperdom) { ish[0] = iregsz[lev]; ish[1] = 0; ish[2] = -iregsz[lev]; } else ish[0] = ish[1] = ish[2] = 0;
    if (yperdom) { jsh[0] = jregsz[lev]; jsh[1] = 0; jsh[2] = -jregsz[lev]; } else jsh[0] = jsh[1] = jsh[2] = 0;
  }

  void set_phys_bndry(std::vector<int8_t>& f, const IBox& B, int lev) {
    const int mb = B.mb;
    if (B.ilo - mb < 0 && !xperdom) for (int j = B.jlo - mb; j <= B.jhi + mb; ++j) for (int i = B.ilo - mb; i <= -1; ++i) f[B.idx(i, j)] = 1;
    if (B.ihi + mb >= iregsz[lev] && !xperdom) for (int j = B.jlo - mb; j <= B.jhi + mb; ++j) for (int i = iregsz[lev]; i <= B.ihi + mb; ++i) f[B.idx(i, j)] = 1;
    if (B.jlo - mb < 0 && !yperdom) for (int j = B.jlo - mb; j <= -1; ++j) for (int i = B.ilo - mb; i <= B.ihi + mb; ++i) f[B.idx(i, j)] = 1;
    if (B.jhi + mb >= jregsz[lev] && !yperdom) for (int j = jregsz[lev]; j <= B.jhi + mb; ++j) for (int i = B.ilo - mb; i <= B.ihi + mb; ++i) f[B.idx(i, j)] = 1;
  }
  void shrink(const std::vector<int8_t>& in, std::vector<int8_t>& out, const IBox& B, int lev) {
    const int mb = B.mb;
    out.assign((size_t)B.ni() * B.nj(), 0);
    for (int j = B.jlo - mb + 1; j <= B.jhi + mb - 1; ++j)
      for (int i = B.ilo - mb + 1; i <= B.ihi + mb - 1; ++i) {
        bool ok = true;
        for (int dj = -1; dj <= 1 && ok; ++dj) for (int di = -1; di <= 1; ++di) if (in[B.idx(i + di, j + dj)] <= 0) { ok = false; break; }
        out[B.idx(i, j)] = ok ? in[B.idx(i, j)] : 0;
      }
    set_phys_bndry(out, B, lev);
  }
  // setdomflags.f: cells of the lcheck-level buffered box that are properly nested in lbase
  std::vector<int8_t> nesting_mask(const HPatch& g, int mbuff, int lbase, int lcheck) {
    int gs[12], ge[12], hs[12], he[12];
    gs[lcheck] = g.ilo; ge[lcheck] = g.ihi; hs[lcheck] = g.jlo; he[lcheck] = g.jhi;
    for (int lc_ = lcheck - 1; lc_ >= lbase; --lc_) {
      int a = (int)std::floor((double)gs[lc_ + 1] / intratx[lc_]), b = (int)std::floor((double)hs[lc_ + 1] / intraty[lc_]);
      int c = (int)std::ceil((double)ge[lc_ + 1] / intratx[lc_]) - 1, d = (int)std::ceil((double)he[lc_ + 1] / intraty[lc_]) - 1;
      if (c * intratx[lc_] < ge[lc_ + 1]) c += 1;
      if (d * intraty[lc_] < he[lc_ + 1]) d += 1;
      gs[lc_] = a; hs[lc_] = b; ge[lc_] = c; he[lc_] = d;
    }
    IBox B{gs[lbase], ge[lbase], hs[lbase], he[lbase], mbuff};
    std::vector<int8_t> base((size_t)B.ni() * B.nj(), 0);
    const GridIndex& XB = GI(lbase);
    std::vector<int> hits;
    {
      const bool bx = (B.ilo <= 0 || B.ihi >= iregsz[lbase] - 1), by = (B.jlo <= 0 || B.jhi >= jregsz[lbase] - 1);
      if ((xperdom && bx) || (yperdom && by)) { hits.resize(XB.size()); for (size_t r = 0; r < hits.size(); ++r) hits[r] = (int)r; }
      else XB.query2(B.ilo - mbuff, B.ihi + mbuff, B.jlo - mbuff, B.jhi + mbuff, hits);
    }
    for (int r : hits) {
      const HPatch& b = node[XB.id(r)];
      const bool bx = (B.ilo <= 0 || B.ihi >= iregsz[lbase] - 1), by = (B.jlo <= 0 || B.jhi >= jregsz[lbase] - 1);
      if ((xperdom && bx) || (yperdom && by)) {
        int ist[3], iend[3], jst[3], jend[3], ish[3], jsh[3];
        setIndices(ist, iend, jst, jend, B.ilo - mbuff, B.ihi + mbuff, B.jlo - mbuff, B.jhi + mbuff, ish, jsh, lbase);
        for (int a = 0; a < 3; ++a) {
          const int i1 = std::max(B.ilo - mbuff, ist[a]), i2 = std::min(B.ihi + mbuff, iend[a]);
          for (int c = 0; c < 3; ++c) {
            const int j1 = std::max(B.jlo - mbuff, jst[c]), j2 = std::min(B.jhi + mbuff, jend[c]);
            if (!(i1 <= i2 && j1 <= j2)) continue;
            const int ixlo = std::max(b.ilo, i1 + ish[a]), ixhi = std::min(b.ihi, i2 + ish[a]);
            const int jxlo = std::max(b.jlo, j1 + jsh[c]), jxhi = std::min(b.jhi, j2 + jsh[c]);
            if (ixlo > ixhi || jxlo > jxhi) continue;
            for (int jj = jxlo - jsh[c]; jj <= jxhi - jsh[c]; ++jj) for (int ii = ixlo - ish[a]; ii <= ixhi - ish[a]; ++ii) base[B.idx(ii, jj)] = 1;
          }
        }
      } else {
        const int ixlo = std::max(b.ilo, B.ilo - mbuff), ixhi = std::min(b.ihi, B.ihi + mbuff);
        const int jxlo = std::max(b.jlo, B.jlo - mbuff), jxhi = std::min(b.jhi, B.jhi + mbuff);
        if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
        for (int jj = jxlo; jj <= jxhi; ++jj) for (int ii = ixlo; ii <= ixhi; ++ii) base[B.idx(ii, jj)] = 1;
      }
    }
    set_phys_bndry(base, B, lbase);
    std::vector<int8_t> cur;
    shrink(base, cur, B, lbase);
    for (int lev = lbase + 1; lev <= lcheck; ++lev) {
      IBox F{gs[lev], ge[lev], hs[lev], he[lev], mbuff};
      const int rx = intratx[lev - 1], ry = intraty[lev - 1];
      std::vector<int8_t> up((size_t)F.ni() * F.nj(), 0);
      for (int j = B.jlo; j <= B.jhi; ++j)
        for (int i = B.ilo; i <= B.ihi; ++i)
          for (int mj = 1; mj <= ry; ++mj)
            for (int mi = 1; mi <= rx; ++mi) {
              const int is = std::max(std::min(i * rx - 1 + mi, F.ihi + mbuff), F.ilo - mbuff);
              const int js = std::max(std::min(j * ry - 1 + mj, F.jhi + mbuff), F.jlo - mbuff);
              up[F.idx(is, js)] = cur[B.idx(i, j)];
            }
      for (int j = F.jlo - mbuff; j <= F.jhi + mbuff; ++j) {
        for (int i = F.ihi + 1; i <= F.ihi + mbuff; ++i) up[F.idx(i, j)] = cur[B.idx(i / rx, j / ry)];
        for (int i = F.ilo - mbuff; i <= F.ilo - 1; ++i) up[F.idx(i, j)] = cur[B.idx(i / rx, j / ry)];
      }
      for (int i = F.ilo; i <= F.ihi; ++i) {
        for (int j = F.jlo - mbuff; j <= F.jlo - 1; ++j) up[F.idx(i, j)] = cur[B.idx(i / rx, j / ry)];
        for (int j = F.jhi + 1; j <= F.jhi + mbuff; ++j) up[F.idx(i, j)] = cur[B.idx(i / rx, j / ry)];
      }
      std::vector<int8_t> nx_;
      shrink(up, nx_, F, lev);
      cur.swap(nx_);
      B = F;
    }
    return cur;
  }

  bool base_check(const HPatch& n, int lbase, int thisBuff) {
    HPROF("base_check");
    const int levnew = n.level;
    const bool bx = (n.ilo == 0 || n.ihi == iregsz[levnew] - 1), by = (n.jlo == 0 || n.jhi == jregsz[levnew] - 1);
    int iclo = n.ilo, ichi = n.ihi, jclo = n.jlo, jchi = n.jhi;
    for (int lev = levnew - 1; lev >= lbase; --lev) {
      iclo = iclo / intratx[lev] - 1; ichi = ichi / intratx[lev] + 1; jclo = jclo / intraty[lev] - 1; jchi = jchi / intraty[lev] + 1;
    }
    if (!(xperdom && bx) && !(yperdom && by)) {
      iclo = std::max(iclo, 0); jclo = std::max(jclo, 0); ichi = std::min(ichi, iregsz[lbase] - 1); jchi = std::min(jchi, jregsz[lbase] - 1);
    }
    const int li = ichi - iclo + 1, lj = jchi - jclo + 1;
    std::vector<int8_t> M((size_t)li * lj, 0);
    auto at = [&](int i, int j) -> int8_t& { return M[(size_t)(i - iclo) + (size_t)li * (j - jclo)]; };
    if (n.ilo == 0 && !xperdom) for (int j = jclo; j <= jchi; ++j) { at(iclo, j) = 1; at(iclo + 1, j) = 1; }
    if (n.ihi == iregsz[levnew] - 1 && !xperdom) for (int j = jclo; j <= jchi; ++j) { at(ichi, j) = 1; at(ichi - 1, j) = 1; }
    if (n.jlo == 0 && !yperdom) for (int i = iclo; i <= ichi; ++i) { at(i, jclo) = 1; at(i, jclo + 1) = 1; }
    if (n.jhi == jregsz[levnew] - 1 && !yperdom) for (int i = iclo; i <= ichi; ++i) { at(i, jchi) = 1; at(i, jchi - 1) = 1; }
    const GridIndex& XB = GI(lbase);
    std::vector<int> hits;
    if ((xperdom && bx) || (yperdom && by)) { hits.resize(XB.size()); for (size_t r = 0; r < hits.size(); ++r) hits[r] = (int)r; }
    else XB.query2(iclo - thisBuff, ichi + thisBuff, jclo - thisBuff, jchi + thisBuff, hits);
    for (int r : hits) {
      const int mp = XB.id(r);
      const int iblo = node[mp].ilo - thisBuff, ibhi = node[mp].ihi + thisBuff, jblo = node[mp].jlo - thisBuff, jbhi = node[mp].jhi + thisBuff;
      if (!(xperdom && bx) && !(yperdom && by)) {
        const int a = std::max(iclo, iblo), b = std::min(ichi, ibhi), c = std::max(jclo, jblo), d = std::min(jchi, jbhi);
        for (int j = c; j <= d; ++j) for (int i = a; i <= b; ++i) at(i, j) = 1;
        continue;
      }
      int ist[3], iend[3], jst[3], jend[3], ish[3], jsh[3];
      setIndices(ist, iend, jst, jend, iclo, ichi, jclo, jchi, ish, jsh, lbase);
      for (int a = 0; a < 3; ++a) {
        const int i1 = std::max(iclo, ist[a]), i2 = std::min(ichi, iend[a]);
        for (int c = 0; c < 3; ++c) {
          const int j1 = std::max(jclo, jst[c]), j2 = std::min(jchi, jend[c]);
          if (!(i1 <= i2 && j1 <= j2)) continue;
          const int xl = std::max(i1 + ish[a], iblo), xh = std::min(i2 + ish[a], ibhi), yl = std::max(j1 + jsh[c], jblo), yh = std::min(j2 + jsh[c], jbhi);
          for (int j = yl; j <= yh; ++j) for (int i = xl; i <= xh; ++i) at(i - ish[a], j - jsh[c]) = 1;
        }
      }
    }
    for (int8_t v : M) if (v == 0) return false;
    return true;
  }

  // errest.f:4-63 for the grids G of level lcheck, launched on the stream: the big step
  // (prepbigstep.f: 2*dt, 2*h on the old values coarsened by 2), the regular step
  // (prepregstep.f: dt, h on the values just flagged, ghost cells included) and errf1.f's
  // estimate of component 1, one byte est >= tol per 2x2 block of interior cells (patch k's
  // blocks from boff[k], i fastest). Both steps run the level step kernel on "virtual
  // patches": pool arrays with descriptors of their own and no flux registers. The step
  // results only feed the estimate (stepgrid's Courant number and dtnew are dropped: the
  // next advanc.f resets cfl_level). Freed by richardson_release after the stream syncs.
  void richardson_launch(int lcheck, const std::vector<int>& G, int use_old, std::vector<long long>& boff) {
    HPROF("richardson");
    if (p.naux > 0) throw std::runtime_error("Richardson estimation needs num_aux = 0 (no auxcoarsen)");
    const int np = (int)G.size();
    const double hx = hxposs[lcheck], hy = hyposs[lcheck], dt = possk[lcheck];
    const double tpre = node[G[0]].time - dt;
    FillProg& P = rich_prog;
    P.clear();
    P.zero_scratch = true;
    P.scratch_len = 0;
    for (int l = 1; l <= lcheck; ++l) GI(l);
    std::vector<FillProg> part(np);
    pool_host.run(np, [&](int k) { compile_bigstep_patch(part[k], lcheck, G[k]); });
    std::vector<int> rect_of(np);
    for (int k = 0; k < np; ++k) { rect_of[k] = (int)P.rects.size(); merge_prog(P, part[k]); }
    upload_prog(P);
    // virtual patches: k the coarsened values, np+k the regular step; buffers in one block
    std::vector<PatchDev> vp(2 * (size_t)np);
    std::vector<long long> vo(2 * (size_t)np + 1, 0);
    boff.assign(np + 1, 0);
    for (int k = 0; k < np; ++k) {
      const HPatch& g = node[G[k]];
      const long long mi2 = g.nx() / 2 + 2 * ng, mj2 = g.ny() / 2 + 2 * ng;
      vo[k + 1] = vo[k] + 2 * Arena::rnd(nvar * mi2 * mj2);
      boff[k + 1] = boff[k] + (long long)(g.nx() / 2) * (g.ny() / 2);
    }
    for (int k = 0; k < np; ++k) vo[np + k + 1] = vo[np + k] + Arena::rnd((long long)nvar * mitot(G[k]) * mjtot(G[k]));
    rich_len = std::max<long long>(vo[2 * np], 1);
    rich_buf = palloc(rich_len);
    std::vector<StepWork> work;
    auto tiles = [&](int v, int mx, int my) {
      for (int tj = 1; tj <= my; tj += TILE2)
        for (int ti = 1; ti <= mx; ti += TILE2) work.push_back(StepWork{v, ti, tj, 0, 0, 0, 0});
    };
    for (int k = 0; k < np; ++k) {
      const HPatch& g = node[G[k]];
      PatchDev B{};
      const int nx2 = g.nx() / 2, ny2 = g.ny() / 2;
      B.mitot = nx2 + 2 * ng; B.mjtot = ny2 + 2 * ng; B.mktot = 1;
      B.q[0] = rich_buf + vo[k]; B.q[1] = B.q[0] + Arena::rnd((long long)nvar * B.mitot * B.mjtot);
      B.cur = 0; B.ilo = 0; B.ihi = nx2 - 1; B.jlo = 0; B.jhi = ny2 - 1;
      B.ffl = -1; B.level = lcheck; B.aux = -1;
      vp[k] = B;
      tiles(k, nx2, ny2);
    }
    const int nbig = (int)work.size();
    for (int k = 0; k < np; ++k) {
      const HPatch& g = node[G[k]];
      PatchDev R{};
      const int in_cur = use_old ? 1 - g.cur : g.cur;
      R.q[0] = in_cur == 0 ? g.q0 : g.q1; R.q[1] = rich_buf + vo[np + k];
      R.cur = 0; R.ilo = g.ilo; R.ihi = g.ihi; R.jlo = g.jlo; R.jhi = g.jhi;
      R.mitot = mitot(G[k]); R.mjtot = mjtot(G[k]); R.mktot = 1;
      R.ffl = -1; R.level = lcheck; R.aux = -1;
      vp[np + k] = R;
      tiles(np + k, g.nx(), g.ny());
    }
    const int nreg = (int)work.size() - nbig;
    rich_vp.upload(vp, st, stg);
    rich_work.upload(work, st, stg);
    rich_rect.upload(rect_of, st, stg);
    rich_off.upload(boff, st, stg);
    rich_out.ensure(std::max<long long>(boff[np], 1));
    rich_cfl.ensure(1);
    // the ghost ring at tpre, then coarsen.f
    run_prog(P, bound_modes(lcheck, tpre));
    launch_coarsen2(pool.d, P.d_rects.d, rich_rect.d, rich_vp.d, np, nvar, st, f32);
    StepArgs a{};
    a.pool = pool.d; a.regs = regs.d; a.patches = rich_vp.d; a.fsv = nullptr; a.fad = nullptr;
    a.cflmax = rich_cfl.d; a.sp = sp; a.queue = nullptr; a.dt_dev = nullptr;
    a.sp.split = 0;  // errest's big and regular steps call the unsplit stepgrid (prepbigstep.f:60, prepregstep.f:23)
    if (nbig > 0) {
      a.work = rich_work.d; a.nwork = nbig;
      a.dt = 2.0 * dt; a.dx = 2.0 * hx; a.dy = 2.0 * hy;
      launch_step2(prob.solver, a, nbig, st, f32);
    }
    if (nreg > 0) {
      a.work = rich_work.d + nbig; a.nwork = nreg;
      a.dt = dt; a.dx = hx; a.dy = hy;
      launch_step2(prob.solver, a, nreg, st, f32);
    }
    const double order = (double)((1 << (sp.order + 1)) - 2);
    launch_errf2(pool.d, rich_vp.d, np, ng, order, p.tol, rich_off.d, rich_out.d, st, f32);
    nkernels += 3 + (nbig > 0) + (nreg > 0);
  }
  void richardson_release() {
    pfree(rich_prog.scratch_off, rich_prog.scratch_alloc);
    rich_prog.scratch_off = -1;
    pfree(rich_buf, rich_len);
    rich_buf = -1;
  }

  // flagger.f + bufnst2.f + colate2.f: the sorted, unique flagged points of level lcheck
  std::vector<Pt> flag_points(int lcheck, int lbase) {
    const int mbuff = std::max(ng, p.ibuff + 1);
    std::vector<int>& G = lgrids[lcheck];
    const double t = node[G[0]].time;
    int use_old = 0;
    {
      HPROF("flag_bound");
      if (start_time + possk[lcheck] != t) bound_level(lcheck, t);
      else use_old = 1;
    }
    // device gradient test
    const auto tf0 = std::chrono::steady_clock::now();
    std::vector<long long> off(G.size() + 1, 0);
    for (size_t k = 0; k < G.size(); ++k) off[k + 1] = off[k] + (long long)node[G[k]].nx() * node[G[k]].ny();
    DBuf<int8_t>& dout = fl_out; dout.ensure(std::max<long long>(off.back(), 1));
    DBuf<long long>& doff = fl_off; doff.upload(off, st, stg);
    DBuf<int>& dpl = fl_pl; dpl.upload(G, st, stg);
    launch_flags2(pool.d, d_patches.d, dpl.d, doff.d, (int)G.size(), use_old, p.flag_component, p.tolsp, nvar, dout.d, st, f32);
    std::vector<int8_t> hflag(off.back());
    if (off.back()) AMR_CUDA(cudaMemcpyAsync(hflag.data(), dout.d, off.back(), cudaMemcpyDeviceToHost, st));
    std::vector<long long> roff;
    std::vector<int8_t> rbits;
    if (p.flag_richardson) {
      richardson_launch(lcheck, G, use_old, roff);
      rbits.resize(roff.back());
      if (roff.back()) AMR_CUDA(cudaMemcpyAsync(rbits.data(), rich_out.d, roff.back(), cudaMemcpyDeviceToHost, st));
    }
    sync_stream();
    if (p.flag_richardson) richardson_release();
    const auto tf1 = std::chrono::steady_clock::now();
    tr_flags += std::chrono::duration<double>(tf1 - tf0).count();
    const double dx = hxposs[lcheck], dy = hyposs[lcheck];
    std::vector<Pt> pts;
    int numbad = 0;
    // projec2.f boxes of the level lcheck+2 grids just created, indexed; wrapping ones are tried on every patch
    std::vector<int> pnew, pwrap;
    GridIndex XP;
    if (lcheck + 2 <= p.mxnest) {
      std::vector<std::array<int, 6>> pb;
      for (int mk = newstl[lcheck + 2]; mk != 0; mk = node[mk].levelptr) {
        const HPatch& c = node[mk];
        const int istc = (c.ilo / intratx[lcheck + 1] - 1) / intratx[lcheck] - 1, jstc = (c.jlo / intraty[lcheck + 1] - 1) / intraty[lcheck] - 1;
        const int iendc = (c.ihi / intratx[lcheck + 1] + 1) / intratx[lcheck] + 1, jendc = (c.jhi / intraty[lcheck + 1] + 1) / intraty[lcheck] + 1;
        const bool bx = (istc <= 0 || iendc >= iregsz[lcheck] - 1), by = (jstc <= 0 || jendc >= jregsz[lcheck] - 1);
        if ((xperdom && bx) || (yperdom && by)) pwrap.push_back(mk);
        else { pnew.push_back(mk); pb.push_back({istc, iendc, jstc, jendc, 0, 0}); }
      }
      std::vector<int> ids(pb.size());
      for (size_t r = 0; r < ids.size(); ++r) ids[r] = (int)r;
      XP.build(ids, [&](int r) { return pb[r]; });
    }
    GI(lbase);  // built here: the per-patch work below only reads the index
    std::vector<std::vector<Pt>> ptsp(G.size());
    ScopedTimer tpp(hprof, "flag_patches");
    pool_host.run((int)G.size(), [&](int k) {
      HPatch& g = node[G[k]];
      const int mx = g.nx(), my = g.ny();
      IBox B{g.ilo, g.ihi, g.jlo, g.jhi, mbuff};
      std::vector<int8_t> f((size_t)B.ni() * B.nj(), FLAG_UNSET);
      std::vector<int> phits;
      // flagregions2.f90
      std::vector<int> mnl, mxl;
      if (!p.regions.empty()) { mnl.assign((size_t)mx * my, 0); mxl.assign((size_t)mx * my, 0); }
      const double xu = g.xlo + mx * dx, yu = g.ylo + my * dy;
      for (const RegionSpec& r : p.regions) {
        if (t < r.t1 || t > r.t2) continue;
        if (g.xlo >= r.x2 || xu <= r.x1) continue;
        const int i1 = std::max((int)std::floor((r.x1 - g.xlo) / dx) + 1, 1), i2 = std::min((int)std::floor((r.x2 - g.xlo) / dx) + 1, mx);
        if (g.ylo >= r.y2 || yu <= r.y1) continue;
        const int j1 = std::max((int)std::floor((r.y1 - g.ylo) / dy) + 1, 1), j2 = std::min((int)std::floor((r.y2 - g.ylo) / dy) + 1, my);
        for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
          mnl[(size_t)(j - 1) * mx + i - 1] = std::max(mnl[(size_t)(j - 1) * mx + i - 1], r.minlevel);
          mxl[(size_t)(j - 1) * mx + i - 1] = std::max(mxl[(size_t)(j - 1) * mx + i - 1], r.maxlevel);
        }
      }
      const int8_t* gf = hflag.data() + off[k];
      for (int j = 1; j <= my; ++j)
        for (int i = 1; i <= mx; ++i) {
          const int a = mnl.empty() ? 0 : mnl[(size_t)(j - 1) * mx + i - 1], b = mxl.empty() ? 0 : mxl[(size_t)(j - 1) * mx + i - 1];
          if (a > b) throw std::runtime_error("region minimum level exceeds its maximum level");
          int8_t v = FLAG_UNSET;
          if (b != 0) { if (lcheck < a) v = FLAG_DO; else if (lcheck >= b) v = FLAG_DONT; }
          if (v == FLAG_UNSET && p.flag_gradient && gf[(size_t)(j - 1) * mx + (i - 1)]) v = FLAG_DO;
          f[B.idx(g.ilo + i - 1, g.jlo + j - 1)] = v;
        }
      // errf1.f:55-95: a block with a flag still unset gets DOFLAG on all four cells when
      // est >= tol. The reference indexes the flag array (nx + 2*mbuff wide) with the fine
      // grid's ghost width, so a block's flags sit mbuff - nghost cells below and left of
      // the cells whose values it compares; they are placed the same way here (cells that
      // land in the buffer zone are dropped by shiftset2.f, as there)
      if (p.flag_richardson) {
        const int8_t* rb = rbits.data() + roff[k];
        const int nxc = mx / 2, nyc = my / 2, sh = ng - mbuff;
        for (int jc = 0; jc < nyc; ++jc)
          for (int ic = 0; ic < nxc; ++ic) {
            if (!rb[(size_t)jc * nxc + ic]) continue;
            const int i0 = g.ilo + sh + 2 * ic, j0 = g.jlo + sh + 2 * jc;
            int8_t* c[4] = {&f[B.idx(i0, j0)], &f[B.idx(i0 + 1, j0)], &f[B.idx(i0, j0 + 1)], &f[B.idx(i0 + 1, j0 + 1)]};
            if (*c[0] == FLAG_UNSET || *c[1] == FLAG_UNSET || *c[2] == FLAG_UNSET || *c[3] == FLAG_UNSET)
              for (int8_t* q : c) *q = FLAG_DO;
          }
      }
      // projec2.f: cells under level lcheck+2 grids just created
      if (lcheck + 2 <= p.mxnest) {
        std::vector<int> cand;
        XP.query2(g.ilo - mbuff, g.ihi + mbuff, g.jlo - mbuff, g.jhi + mbuff, phits);
        for (int r : phits) cand.push_back(pnew[r]);
        cand.insert(cand.end(), pwrap.begin(), pwrap.end());
        for (int mk : cand) {
          const HPatch& c = node[mk];
          int istc = (c.ilo / intratx[lcheck + 1] - 1) / intratx[lcheck] - 1, jstc = (c.jlo / intraty[lcheck + 1] - 1) / intraty[lcheck] - 1;
          int iendc = (c.ihi / intratx[lcheck + 1] + 1) / intratx[lcheck] + 1, jendc = (c.jhi / intraty[lcheck + 1] + 1) / intraty[lcheck] + 1;
          const bool bx = (istc <= 0 || iendc >= iregsz[lcheck] - 1), by = (jstc <= 0 || jendc >= jregsz[lcheck] - 1);
          auto markp = [&](int a0, int a1, int b0, int b1) {
            const int xl = std::max(a0, g.ilo - mbuff), xh = std::min(a1, g.ihi + mbuff), yl = std::max(b0, g.jlo - mbuff), yh = std::min(b1, g.jhi + mbuff);
            for (int j = yl; j <= yh; ++j) for (int i = xl; i <= xh; ++i) if (f[B.idx(i, j)] <= FLAG_DONT) f[B.idx(i, j)] = FLAG_BADPRO;
          };
          if (!(xperdom && bx) && !(yperdom && by)) {
            istc = std::max(istc, 0); jstc = std::max(jstc, 0); iendc = std::min(iendc, iregsz[lcheck]); jendc = std::min(jendc, jregsz[lcheck]);
            markp(istc, iendc, jstc, jendc);
          } else {
            int ist[3], iend[3], jst[3], jend[3], ish[3], jsh[3];
            setIndices(ist, iend, jst, jend, istc, iendc, jstc, jendc, ish, jsh, lcheck);
            for (int a = 0; a < 3; ++a) for (int c2 = 0; c2 < 3; ++c2) {
              const int i1 = std::max(istc, ist[a]), i2 = std::min(iendc, iend[a]), j1 = std::max(jstc, jst[c2]), j2 = std::min(jendc, jend[c2]);
              if (!(i1 <= i2 && j1 <= j2)) continue;
              markp(i1 + ish[a], i2 + ish[a], j1 + jsh[c2], j2 + jsh[c2]);
            }
          }
        }
      }
      // shiftset2.f: buffer by ibuff in every direction
      // Only "flagged or not" survives buffering (colate2 tests > DONTFLAG), so the
      // (2*ibuff+1)^2 stamp is applied as a row pass and a column pass.
      std::vector<int8_t> row((size_t)B.ni() * B.nj(), 0), buf((size_t)B.ni() * B.nj(), FLAG_DONT);
      for (int j = g.jlo; j <= g.jhi; ++j)
        for (int i = g.ilo; i <= g.ihi; ++i)
          if (f[B.idx(i, j)] > 0) for (int mm = i - p.ibuff; mm <= i + p.ibuff; ++mm) row[B.idx(mm, j)] = 1;
      for (int j = g.jlo; j <= g.jhi; ++j)
        for (int i = g.ilo - p.ibuff; i <= g.ihi + p.ibuff; ++i)
          if (row[B.idx(i, j)]) for (int kk = j - p.ibuff; kk <= j + p.ibuff; ++kk) buf[B.idx(i, kk)] = FLAG_DO;
      int nf = 0;
      for (int8_t v : buf) if (v > FLAG_DONT) ++nf;
      g.numflags = nf;
      // colate2.f: nested flags with periodic wrap (the point order is irrelevant:
      // drivesort sorts them and drops duplicates)
      std::vector<Pt>& out = ptsp[k];
      out.clear();
      if (nf != 0) {
        const std::vector<int8_t> dom2 = nesting_mask(g, mbuff, lbase, lcheck);
        int jmin = g.jlo - mbuff, jmax = g.jhi + mbuff, imin = g.ilo - mbuff, imax = g.ihi + mbuff;
        if (!xperdom) { imin = std::max(imin, 0); imax = std::min(g.ihi + mbuff, iregsz[lcheck] - 1); }
        if (!yperdom) { jmin = std::max(jmin, 0); jmax = std::min(g.jhi + mbuff, jregsz[lcheck] - 1); }
        for (int j = jmin; j <= jmax; ++j)
          for (int i = imin; i <= imax; ++i) {
            if (buf[B.idx(i, j)] <= FLAG_DONT || dom2[B.idx(i, j)] != 1) continue;
            int iw = i, jw = j;
            if (xperdom) { if (i < 0) iw = i + iregsz[lcheck]; if (i >= iregsz[lcheck]) iw = i - iregsz[lcheck]; }
            if (yperdom) { if (j < 0) jw = j + jregsz[lcheck]; if (j >= jregsz[lcheck]) jw = j - jregsz[lcheck]; }
            out.push_back(Pt{iw, jw});
          }
      }
    });
    for (int m : G) numbad += node[m].numflags;
    ScopedTimer tcol(hprof, "colate");
    if (numbad == 0) return pts;
    size_t tot = 0;
    for (size_t k = 0; k < G.size(); ++k) tot += ptsp[k].size();
    pts.reserve(tot);
    for (size_t k = 0; k < G.size(); ++k) pts.insert(pts.end(), ptsp[k].begin(), ptsp[k].end());
    {
      HPROF("sort_unique");
      sort_unique(pts, iregsz[lcheck], mbuff);
    }
    tr_host += std::chrono::duration<double>(std::chrono::steady_clock::now() - tf1).count();
    if (std::getenv("AMRB_DEBUG")) {
      long long gsum = 0;
      for (int8_t v : hflag) gsum += v;
      std::fprintf(stderr, "FLAGS lcheck=%d lbase=%d t=%.17g use_old=%d grad=%lld npts=%zu:", lcheck, lbase, t, use_old, gsum, pts.size());
      for (size_t k = 0; k < pts.size() && k < 12; ++k) std::fprintf(stderr, " (%d,%d)", pts[k].i, pts[k].j);
      std::fprintf(stderr, "\n");
    }
    return pts;
  }

  // ---------------------------------------------------------------- clustering
  // Berger-Rigoutsos bisection (smartbis.f:25-177, signs.f:16-71, findcut.f:7-130,
  // moment.f:16-75) driven by signatures made on the device. The level's points (the
  // buffered, nested, wrapped and deduplicated flags of flag_points) are scattered into a
  // one-plane device array; a cluster is a box of it and its points the flagged cells
  // inside. Each wave of the bisection sends the boxes of all undecided clusters to the
  // device, which counts the points per i and per j of every box; only those counts come
  // back, and the host takes from them the count, the bounding box, the efficiency and the
  // cut. Every decision depends only on these counts, as the reference's do on its points.
  struct Clu2 { SigBox box; int n = 0; int lo[2] = {0, 0}, hi[2] = {0, 0}; };
  DBuf<int8_t> sig_mask;
  DBuf<int> sig_pts, sig_off, sig_hist;
  DBuf<SigBox> sig_boxes;
  LvlDims sig_dims{0, 0, 1};
  // signs.f on the device for the boxes of clus (1-based array indices = level index + 1);
  // fills n, lo, hi; si / sj (optional): each cluster's counts at 1-based level positions
  void signatures(std::vector<Clu2>& clus, std::vector<std::vector<int>>* si, std::vector<std::vector<int>>* sj) {
    const int nb = (int)clus.size();
    if (nb == 0) return;
    std::vector<SigBox> bx(nb);
    std::vector<int> off(nb + 1, 0);
    int maxlen = 0;
    long long maxvol = 0;
    for (int b = 0; b < nb; ++b) {
      bx[b] = clus[b].box;
      const int ni = bx[b].hi[0] - bx[b].lo[0] + 1, nj = bx[b].hi[1] - bx[b].lo[1] + 1;
      off[b + 1] = off[b] + ni + nj + 1;
      maxlen = std::max(maxlen, ni + nj + 1);
      maxvol = std::max(maxvol, (long long)nj);  // i-rows of the box
    }
    sig_boxes.upload(bx, st, stg);
    sig_off.upload(off, st, stg);
    sig_hist.ensure((size_t)off[nb]);
    launch_signatures3(sig_mask.d, sig_dims, sig_boxes.d, nb, sig_off.d, off[nb], maxlen, maxvol, sig_hist.d, st);
    ++nkernels;
    std::vector<int> h((size_t)off[nb]);
    AMR_CUDA(cudaMemcpyAsync(h.data(), sig_hist.d, sizeof(int) * h.size(), cudaMemcpyDeviceToHost, st));
    sync_stream();
    if (si) { si->assign(nb, {}); sj->assign(nb, {}); }
    for (int b = 0; b < nb; ++b) {
      Clu2& c = clus[b];
      const int* hh = h.data() + off[b];
      for (int d = 0; d < 2; ++d) {
        const int len = c.box.hi[d] - c.box.lo[d] + 1;
        int first = -1, last = -1, sum = 0;
        for (int t = 0; t < len; ++t)
          if (hh[t]) { if (first < 0) first = t; last = t; sum += hh[t]; }
        if (d == 0) c.n = sum;
        c.lo[d] = first < 0 ? c.box.lo[d] : c.box.lo[d] + first;
        c.hi[d] = last < 0 ? c.box.hi[d] : c.box.lo[d] + last;
        if (si) {
          std::vector<int>& v = d == 0 ? (*si)[b] : (*sj)[b];
          v.assign((d == 0 ? sig_dims.is : sig_dims.js) + 2, 0);
          for (int t = 0; t < len; ++t) v[c.box.lo[d] + t] = hh[t];
        }
        hh += len;
      }
    }
  }
  // moment.f: rect (0-based level indices ilo, ihi, jlo, jhi) and efficiency of a cluster
  static double moment2(const Clu2& c, int rect[4]) {
    rect[0] = c.lo[0] - 1; rect[1] = c.hi[0] - 1; rect[2] = c.lo[1] - 1; rect[3] = c.hi[1] - 1;
    return (double)c.n / (double)((rect[1] - rect[0] + 1) * (rect[3] - rect[2] + 1));
  }
  // smartbis.f, breadth first over the device signatures; leaves in the reference's order
  // (the part at or above the cut first)
  std::vector<Clu2> bisect_on_device(const std::vector<Pt>& pts, int lcheck, double cutoff) {
    sig_dims = LvlDims{iregsz[lcheck], jregsz[lcheck], 1};
    sig_mask.ensure((size_t)sig_dims.size());
    std::vector<int> flat(2 * pts.size());
    for (size_t k = 0; k < pts.size(); ++k) { flat[2 * k] = pts[k].i; flat[2 * k + 1] = pts[k].j; }
    sig_pts.upload(flat, st, stg);
    launch_scatter_points2(sig_pts.d, (int)pts.size(), sig_mask.d, sig_dims, st);
    ++nkernels;
    struct Node { Clu2 c; int child = -1; };
    std::vector<Node> T(1);
    T[0].c.box = SigBox{{1, 1, 1}, {sig_dims.is, sig_dims.js, 1}};
    std::vector<int> wave{0};
    std::vector<std::vector<int>> si, sj;
    while (!wave.empty()) {
      std::vector<Clu2> cl(wave.size());
      for (size_t w = 0; w < wave.size(); ++w) cl[w] = T[wave[w]].c;
      signatures(cl, &si, &sj);
      std::vector<int> next;
      for (size_t w = 0; w < wave.size(); ++w) {
        T[wave[w]].c = cl[w];
        const Clu2& c = cl[w];
        if (c.n == 0) continue;
        int rect[4];
        if (moment2(c, rect) >= cutoff) continue;
        int dir = 0;
        const int cut = find_cut_sig(si[w], sj[w], sig_dims.is, sig_dims.js, dir);
        if (cut == 0) continue;
        const int d = dir - 1;
        Clu2 up, dn;
        up.box = dn.box = SigBox{{c.lo[0], c.lo[1], 1}, {c.hi[0], c.hi[1], 1}};
        up.box.lo[d] = cut;
        dn.box.hi[d] = cut - 1;
        const int id = (int)T.size();
        T[wave[w]].child = id;
        T.push_back(Node{up, -1});
        T.push_back(Node{dn, -1});
        next.push_back(id);
        next.push_back(id + 1);
      }
      wave.swap(next);
    }
    std::vector<Clu2> leaves;
    if (T[0].c.n == 0) return leaves;
    std::vector<int> stack{0};
    while (!stack.empty()) {
      const int id = stack.back();
      stack.pop_back();
      if (T[id].child < 0) { leaves.push_back(T[id].c); continue; }
      stack.push_back(T[id].child + 1);
      stack.push_back(T[id].child);
    }
    return leaves;
  }

  // grdfit2.f:20-150
  void grdfit(int lbase, int lcheck, double t) {
    std::vector<Pt> pts = flag_points(lcheck, lbase);
    if (pts.empty()) return;
    const int levnew = lcheck + 1;
    const double hxf = hxposs[levnew], hyf = hyposs[levnew];
    const auto tc0 = std::chrono::steady_clock::now();
    std::vector<Clu2> cl;
    {
      HPROF("bisect");
      cl = bisect_on_device(pts, lcheck, p.cut);
    }
    int icl = 0, prv = 0;
    while (icl < (int)cl.size()) {
      const int mnew = nodget();
      while (true) {
        int rect[4];
        moment2(cl[icl], rect);
        HPatch& n = node[mnew];
        n.ilo = rect[0] * intratx[lcheck]; n.jlo = rect[2] * intraty[lcheck];
        n.ihi = (rect[1] + 1) * intratx[lcheck] - 1; n.jhi = (rect[3] + 1) * intraty[lcheck] - 1;
        n.xlo = n.ilo * hxf + xlower; n.ylo = n.jlo * hyf + ylower;
        n.xhi = (n.ihi + 1) * hxf + xlower; n.yhi = (n.jhi + 1) * hyf + ylower;
        n.level = levnew; n.time = t;
        // nestck2.f:37-176
        bool n1 = (lbase == 1) ? true : base_check(n, lbase, 0);
        const int l2 = levnew - 2;
        bool n2;
        if (l2 <= 1) n2 = true;
        else if (l2 <= lbase) n2 = n1;
        else n2 = base_check(n, l2, std::max(ng, p.ibuff + 1));
        if (n1 && n2) break;
        if (cl[icl].n <= 1) throw std::runtime_error("a single flagged point cannot be properly nested");
        double rmid; int dir;
        if (n.xhi - n.xlo > n.yhi - n.ylo) { rmid = (n.ihi + n.ilo + 1) / 2.; rmid = rmid / intratx[levnew - 1]; dir = 1; }
        else { rmid = (n.jhi + n.jlo + 1) / 2.; rmid = rmid / intraty[levnew - 1]; dir = 2; }
        // points with centre (index + .5) below rmid first, then the rest (nestck2.f:130-160)
        const Clu2 c = cl[icl];
        const int d = dir - 1;
        int cut = c.lo[d] - 1;  // the largest 1-based array index whose point centre lies below rmid
        for (int a = c.lo[d]; a <= c.hi[d]; ++a) if ((a - 1) + 0.5 < rmid) cut = a;
        std::vector<Clu2> parts(2);
        parts[0].box = parts[1].box = SigBox{{c.lo[0], c.lo[1], 1}, {c.hi[0], c.hi[1], 1}};
        parts[0].box.hi[d] = cut;
        parts[1].box.lo[d] = cut + 1;
        signatures(parts, nullptr, nullptr);
        cl[icl] = parts[0];
        cl.insert(cl.begin() + icl + 1, parts[1]);
      }
      if (newstl[levnew] == 0) newstl[levnew] = mnew;
      else node[prv].levelptr = mnew;
      prv = mnew;
      ++icl;
    }
    birect(newstl[levnew]);
    tr_cluster += std::chrono::duration<double>(std::chrono::steady_clock::now() - tc0).count();
  }

  // filval.f90 for all new grids of level lev, then release the old grids (gfixup.f:49-163)
  void fill_new_level(int lev) {
    HPROF("fill_new_level");
    FillProg& P = newfill;
    P.clear();
    P.zero_scratch = true;
    P.rects.clear();
    P.scratch_len = 0;
    GI(lev - 1); GI(lev);
    std::vector<int> nl;
    for (int m = newstl[lev]; m != 0; m = node[m].levelptr) nl.push_back(m);
    std::vector<FillProg> part(nl.size());
    pool_host.run((int)nl.size(), [&](int k) { fill_new_patch(part[k], lev, nl[k]); });
    for (auto& q : part) merge_prog(P, q);
    upload_prog(P);
    SrcMode M{};
    run_prog(P, M);
    sync_stream();
    pfree(P.scratch_off, P.scratch_alloc);
    P.scratch_off = -1;
  }
  // filval.f90 for new patch m: coarse values around it, then copies from the old grids
  void fill_new_patch(FillProg& P, int lev, int m) {
    P.scratch_len = 0;
    const int rx = intratx[lev - 1], ry = intraty[lev - 1];
    const double dxc = hxposs[lev] * rx, dyc = hyposs[lev] * ry;
    {
      const HPatch& g = node[m];
      const int iclo = g.ilo / rx - 1, jclo = g.jlo / ry - 1, ichi = (g.ihi + 1) / rx - 1 + 1, jchi = (g.jhi + 1) / ry - 1 + 1;
      const int mic = g.nx() / rx + 2, mjc = g.ny() / ry + 2;
      const int R = P.add_rect(mic, mjc, nvar);
      Tgt C{-1, R, mic, mjc};
      const bool sxc = (iclo < 0) || (ichi >= iregsz[lev - 1]), syc = (jclo < 0) || (jchi >= jregsz[lev - 1]);
      if ((xperdom && sxc) || (yperdom && syc)) c_preicall(P, C, iclo, ichi, jclo, jchi, lev - 1, 0);
      else c_icall(P, C, iclo, ichi, jclo, jchi, lev - 1, 1, 1, 0);
      bool any;
      BcOp b = make_bc(C, dxc, dyc, g.xlo - dxc, g.xhi + dxc, g.ylo - dyc, g.yhi + dyc, any);
      if (any) P.add_bc(b, 0);
      // fine copies from the old grids of this level over the interior
      const int nx = g.nx(), ny = g.ny();
      std::vector<int8_t> cov((size_t)nx * ny, 0);
      const GridIndex& XO = GI(lev);
      std::vector<int> hits;
      XO.query2(g.ilo, g.ihi, g.jlo, g.jhi, hits);
      for (int r : hits) {
        const int o = XO.id(r);
        const HPatch& s = node[o];
        const int ixlo = std::max(s.ilo, g.ilo), ixhi = std::min(s.ihi, g.ihi), jxlo = std::max(s.jlo, g.jlo), jxhi = std::min(s.jhi, g.jhi);
        if (!(ixlo <= ixhi && jxlo <= jxhi)) continue;
        FillOp o2{};
        o2.kind = FILL_COPY; o2.dst_patch = m; o2.dst_rect = -1;
        o2.di0 = ixlo - g.ilo + ng; o2.dj0 = jxlo - g.jlo + ng; o2.ni = ixhi - ixlo + 1; o2.nj = jxhi - jxlo + 1;
        o2.src = o; o2.si0 = ixlo - s.ilo + ng; o2.sj0 = jxlo - s.jlo + ng; o2.level = -1;
        P.add_op(o2, 1);
        for (int j = jxlo; j <= jxhi; ++j) for (int i = ixlo; i <= ixhi; ++i) cov[(size_t)(j - g.jlo) * nx + (i - g.ilo)] = 1;
      }
      std::vector<int> rr;
      runs(cov, nx, ny, rr);
      int capa0 = -1;
      if (p.mcapa > 0 && !rr.empty()) {
        // filval.f90:90-96: setaux on the coarse patch (no ghost cells, lower corner one
        // coarse cell out); fixcapaq reads its kappa
        std::vector<double> ac;
        setaux(0, mic, mjc, g.xlo - dxc, g.ylo - dyc, dxc, dyc, ac);
        capa0 = (int)P.capa.size();
        P.capa.insert(P.capa.end(), ac.begin() + (size_t)(p.mcapa - 1) * mic * mjc, ac.begin() + (size_t)p.mcapa * mic * mjc);
      }
      for (size_t k = 0; k < rr.size(); k += 4) {
        FillOp o2{};
        o2.kind = FILL_FILVAL; o2.dst_patch = m; o2.dst_rect = -1;
        o2.di0 = rr[k] + ng; o2.dj0 = rr[k + 1] + ng; o2.ni = rr[k + 2]; o2.nj = rr[k + 3];
        o2.src = R; o2.si0 = g.ilo + rr[k]; o2.sj0 = g.jlo + rr[k + 1]; o2.level = lev; o2.cilo = iclo; o2.cjlo = jclo;
        P.add_op(o2, 1);
        if (capa0 >= 0) {
          // fixcapaq.f over the coarse cells of the interpolated region (old and new grids are
          // unions of coarse cells, so each coarse cell's fine block is all copied or all
          // interpolated and only the latter change)
          if (rr[k] % rx || rr[k + 1] % ry || rr[k + 2] % rx || rr[k + 3] % ry)
            throw std::runtime_error("filval: interpolated region not aligned with the coarse cells");
          FillOp o3 = o2;
          o3.kind = FILL_FIXCAPA; o3.ni = rr[k + 2] / rx; o3.nj = rr[k + 3] / ry; o3.capa0 = capa0;
          P.add_op(o3, 2);
        }
      }
    }
  }

  void regrid(int lbase) {
    const auto t0c = std::chrono::steady_clock::now();
    int lcheck = std::min(lfine, p.mxnest - 1);
    int lfnew = lbase;
    for (int i = 1; i <= p.mxnest; ++i) newstl[i] = 0;
    const double t = node[lstart[lbase]].time;
    while (lcheck >= lbase) {
      grdfit(lbase, lcheck, t);
      if (newstl[lcheck + 1] != 0) lfnew = std::max(lcheck + 1, lfnew);
      --lcheck;
    }
    // gfixup.f: registers of the changed levels are rebuilt below
    for (int lcheck2 = lbase + 1; lcheck2 <= p.mxnest; ++lcheck2) {
      for (int m = newstl[lcheck2]; m != 0; m = node[m].levelptr) alloc_patch(m);
      // descriptors must know the new patches before their fill runs
      std::vector<int> keep = lgrids[lcheck2];
      lgrids[lcheck2].clear();
      for (int m = newstl[lcheck2]; m != 0; m = node[m].levelptr) lgrids[lcheck2].push_back(m);
      int lf_save = lfine;
      lfine = std::max(lfine, lcheck2);
      sync_descriptors_with(keep, lcheck2);
      lfine = lf_save;
      lgrids[lcheck2] = keep;
      const auto tq0 = std::chrono::steady_clock::now();
      if (newstl[lcheck2] != 0) fill_new_level(lcheck2);
      tr_fill += std::chrono::duration<double>(std::chrono::steady_clock::now() - tq0).count();
      int m = lstart[lcheck2];
      while (m != 0) {
        const int mold = m;
        m = node[m].levelptr;
        free_patch(mold);
        node[mold].bnd.clear(); node[mold].listbc.clear();
        putnod(mold);
      }
      lstart[lcheck2] = newstl[lcheck2];
      touch(lcheck2);
      lgrids[lcheck2].clear();
      for (int q = lstart[lcheck2]; q != 0; q = node[q].levelptr) lgrids[lcheck2].push_back(q);
    }
    lfine = lfnew;
    for (int lev = lbase; lev <= p.mxnest; ++lev) { for (int m : lgrids[lev]) { node[m].has_cfl = false; node[m].listbc.clear(); } }
    const auto tp0 = std::chrono::steady_clock::now();
    for (int lev = lbase; lev <= lfine - 1; ++lev) { prepf(lev + 1); prepc(lev); }
    for (int lev = lbase + 1; lev <= p.mxnest; ++lev) arrange(lev);
    make_lists();
    for (int lev = lbase + 1; lev <= lfine; ++lev) make_bndry(lev);
    const auto tp1 = std::chrono::steady_clock::now();
    compile_all(lbase);
    {
      HPROF("regrid_final_sync");
      sync_stream();
    }
    const auto tp2 = std::chrono::steady_clock::now();
    tr_prep += std::chrono::duration<double>(tp1 - tp0).count();
    tr_compile += std::chrono::duration<double>(tp2 - tp1).count();
    t_regrid += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0c).count();
  }

  // descriptors for: all current levels plus the old and new patches of level `lev` (during gfixup)
  void sync_descriptors_with(const std::vector<int>& old_lev_grids, int lev) {
    h_patches.assign(id_hwm, PatchDev{});
    auto put = [&](int m) {
      const HPatch& g = node[m];
      PatchDev& d = h_patches[m];
      d.q[0] = g.q0; d.q[1] = g.q1; d.cur = g.cur; d.ffl = g.ffl; d.aux = g.aux;
      d.ilo = g.ilo; d.ihi = g.ihi; d.jlo = g.jlo; d.jhi = g.jhi;
      d.mitot = mitot(m); d.mjtot = mjtot(m); d.mktot = 1; d.level = g.level; d.lenbc = g.lenbc;
    };
    for (int l = 1; l <= p.mxnest; ++l) for (int m : lgrids[l]) put(m);
    for (int m : old_lev_grids) put(m);
    for (int l = 1; l < lev; ++l) for (int m = lstart[l]; m != 0; m = node[m].levelptr) put(m);
    d_patches.upload(h_patches, st, stg);
    (void)lev;
  }

  // ================================================================ init (amr2.f90, domain.f, setgrd.f)
  void init(const std::string& dir) {
    p.load(dir);
    if (p.ndim != 2) throw std::runtime_error("this solver handles 2D runs");
    if (write_output && p.output_format != 1 && p.output_format != 3)
      throw std::runtime_error("output_format must be 1 (ASCII) or 3 (binary): NetCDF and HDF5 output are not supported");
    if (p.nghost != 2) throw std::runtime_error("num_ghost must be 2");
    if (f32 && p.naux != 0) throw std::runtime_error("the FP32 form has no 2D aux arrays (capacity, face velocities)");
    // amr2.f90:258-263: Godunov splitting (stepgrid_dimSplit.f) or unsplit; Strang stops the reference
    if (p.dimsplit > 1) throw std::runtime_error("Strang splitting is not supported (dimensional_split must be 0 or 1)");
    // stepgrid.f:176-180 calls src2 after the step when method(5) = 1; the library's default
    // src2 (src/2d/src2.f90) does nothing, and no registered problem has a source term
    if (p.src_split > 1) throw std::runtime_error("source_split must be 0 or 1 (stepgrid.f calls src2 only for 1)");
    nvar = p.nvar; ng = p.nghost;
    setup_problem();
    xlower = p.lower[0]; ylower = p.lower[1]; xupper = p.upper[0]; yupper = p.upper[1];
    nxc = p.ncells[0]; nyc = p.ncells[1];
    xperdom = (p.mthbc[1] == 2 && p.mthbc[2] == 2);
    yperdom = (p.mthbc[3] == 2 && p.mthbc[4] == 2);
    for (int k = 1; k <= 10; ++k) { intratx[k] = p.ratx[k]; intraty[k] = p.raty[k]; kratio[k] = p.ratt[k]; }
    hxposs[1] = (xupper - xlower) / nxc;
    hyposs[1] = (yupper - ylower) / nyc;
    for (int lev = 2; lev <= p.mxnest; ++lev) { hxposs[lev] = hxposs[lev - 1] / (double)intratx[lev - 1]; hyposs[lev] = hyposs[lev - 1] / (double)intraty[lev - 1]; }
    possk[1] = p.dt_initial;
    iregsz[1] = nxc; jregsz[1] = nyc;
    for (int lev = 2; lev <= p.mxnest; ++lev) {
      iregsz[lev] = iregsz[lev - 1] * intratx[lev - 1];
      jregsz[lev] = jregsz[lev - 1] * intraty[lev - 1];
      possk[lev] = possk[lev - 1] / (double)kratio[lev - 1];
    }
    for (int l = 0; l < MAXLV + 2; ++l) {
      lc.hx[l] = l < 12 ? hxposs[l] : 0; lc.hy[l] = l < 12 ? hyposs[l] : 0;
      lc.iregsz[l] = iregsz[l]; lc.jregsz[l] = jregsz[l]; lc.intratx[l] = intratx[l]; lc.intraty[l] = intraty[l];
    }
    AMR_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    retain_pool_memory();
    AllocStreamScope alloc_scope(st);
    for (cudaEvent_t* e : {&ev_a, &ev_b, &ev_run0, &ev_run1}) AMR_CUDA(cudaEventCreate(e));
    long long est = (long long)nvar * (nxc + 4) * (nyc + 4) * 8 * std::max(1, p.mxnest) + (1 << 22);
    pool.init(est);
    regs.init(1 << 20);
    AMR_CUDA(cudaMalloc(&d_cfl, sizeof(unsigned long long)));
    AMR_CUDA(cudaMallocHost((void**)&h_cfl, sizeof(unsigned long long)));
    AMR_CUDA(cudaMalloc(&d_mass, sizeof(double)));
    AMR_CUDA(cudaMalloc(&d_sub, sizeof(Substep2) * 12));
    AMR_CUDA(cudaMallocHost((void**)&h_sub, sizeof(Substep2) * 12));
    node.assign(10001, HPatch());
    for (int k = 1; k <= 10000; ++k) node[k].nextfree = k + 1;
    node[10000].nextfree = 0;
    ndfree = 1;
    start_time = p.t0;
    if (p.restart) {
      // amr2.f90: the run continues from the checkpoint named in claw.data (restrt.f)
      const std::string f = p.restart_file;
      restart_from(!f.empty() && f[0] == '/' ? f : dir + "/" + f);
      return;
    }
    // domain.f
    const int ms = nodget();
    node[ms].xlo = xlower; node[ms].ylo = ylower; node[ms].yhi = yupper; node[ms].xhi = xupper;
    node[ms].level = 1; node[ms].levelptr = 0;
    node[ms].ilo = 0; node[ms].jlo = 0; node[ms].ihi = nxc - 1; node[ms].jhi = nyc - 1;
    lstart[1] = ms;
    touch(1);
    lfine = 1;
    birect(ms);
    ginit(lstart[1], start_time);
    arrange(1);
    make_lists();
    make_bndry(1);
    sync_descriptors();
    // setgrd.f
    record_gauges = false;
    if (p.mxnest > 1) {
      int levnew = 2;
      while (levnew <= p.mxnest) {
        const int levold = levnew - 1;
        if (lstart[levold] == 0) break;
        compile_all();
        // setgrd.f:41-53: Richardson estimation needs the level one step ahead before it
        // is flagged; that step is not counted as integration work
        if (p.flag_richardson) {
          advanc(levold);
          rvol = 0;
          for (double& r : rvoll) r = 0;
        }
        for (int i = 1; i <= p.mxnest; ++i) newstl[i] = 0;
        grdfit(levold, levold, start_time);
        int lfnew = levold;
        if (newstl[levnew] != 0) lfnew = levnew;
        if (newstl[levnew] != 0) ginit(newstl[levnew], start_time);
        lstart[levnew] = newstl[levnew];
        touch(levnew);
        lfine = lfnew;
        arrange(levnew);
        make_lists();
        make_bndry(levnew);
        ++levnew;
      }
      // store1 and store2 of the initial levels hold the same qinit data (both buffers were
      // filled), unless the Richardson steps above advanced them: setgrd.f:106-121 swaps the
      // stores, putting the initial values back in store1, and resets the times
      if (p.flag_richardson)
        for (int lev = 1; !(lev == p.mxnest || lev > lfine); ++lev)
          for (int m : lgrids[lev]) { node[m].cur ^= 1; node[m].time = start_time; }
      compile_all();
      for (int lev = lfine - 1; lev >= 1; --lev) update(lev);
      for (int lev = 1; lev <= lfine - 1; ++lev) { prepf(lev + 1); prepc(lev); }
    }
    compile_all();
    record_gauges = true;
    time = p.t0;
    mbestsrc.assign(p.gauges.size(), 0);
    glast.assign(p.gauges.size(), 0.0);
    for (size_t i = 0; i < p.gauges.size(); ++i) glast[i] = p.gauges[i].t1;
    frame = p.output_t0 ? 0 : 1;
    tmass0 = mass();
    if (p.output_t0) output(time);
    ensure_all();
    sync_stream();
  }

  // ginit.f: new grids at the initial time, qinit into both buffers
  void ginit(int msave, double t) {
    for (int m = msave; m != 0; m = node[m].levelptr) {
      alloc_patch(m);
      HPatch& g = node[m];
      g.time = t;
      std::vector<double> q;
      qinit(g.nx(), g.ny(), g.xlo, g.ylo, hxposs[g.level], hyposs[g.level], q);
      std::vector<float> qf;
      const void* src = q.data();
      if (f32) {  // the FP32 form stores the initial values rounded to float
        qf.assign(q.begin(), q.end());
        src = qf.data();
      }
      char* base = reinterpret_cast<char*>(pool.d);
      AMR_CUDA(cudaMemcpyAsync(base + elem() * g.q0, src, elem() * q.size(), cudaMemcpyHostToDevice, st));
      AMR_CUDA(cudaMemcpyAsync(base + elem() * g.q1, src, elem() * q.size(), cudaMemcpyHostToDevice, st));
      h2d_bytes += 2.0 * elem() * q.size();
      sync_stream();
    }
  }

  void setbestsrc() {
    for (size_t i = 0; i < p.gauges.size(); ++i) {
      mbestsrc[i] = 0;
      for (int lev = lfine; lev >= 1 && mbestsrc[i] == 0; --lev)
        for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
          const HPatch& g = node[m];
          if (p.gauges[i].x >= g.xlo && p.gauges[i].x <= g.xhi && p.gauges[i].y >= g.ylo && p.gauges[i].y <= g.yhi) { mbestsrc[i] = m; break; }
        }
    }
  }

  double mass() {
    ensure(1, NEED_STEP);
    AMR_CUDA(cudaMemsetAsync(d_mass, 0, sizeof(double), st));
    launch_mass2(pool.d, d_patches.d, plan[1].d_plist.d, (int)plan[1].plist.size(), d_mass, st, f32, p.mcapa);
    double m = 0;
    AMR_CUDA(cudaMemcpyAsync(&m, d_mass, sizeof(double), cudaMemcpyDeviceToHost, st));
    sync_stream();
    return m * hxposs[1] * hyposs[1];
  }

  // valout.f90: zero |q| < 1e-90 in place (the reference does) and optionally write fort.q / fort.t
  void output(double t);
  void write_aux(bool binary);

  // ================================================================ check.f / restrt.f
  // A checkpoint, taken at a coarse-step boundary, holds what the continued run reads:
  // the scheduler state (time, cycle, step sizes, regrid counters, level times, output
  // cursor), the grid table with its free list (grid numbers continue as they would have),
  // both solution buffers of every grid, and the gauge samples so far. Neighbour lists,
  // register lists, fill programs and step plans are compiled again from the grids; the
  // flux registers and saved coarse rings are not kept, because each entry that upbnd
  // will read is rewritten (fluxsv, saveqc, prepf) before it is read. The layout is this
  // library's own (little-endian, versioned).
  static constexpr char CHK_MAGIC[8] = {'A', 'M', 'R', 'B', '2', 'C', 'K', '1'};
  struct ChkHead {
    int nvar, f32, mxnest, lfine, ncycle, frame, nextout, iout, nnodes, ndfree, gslots, ngrows, ngauges, pad;
    int icheck[12], lstart[12];
    double time, start_time, tmass0, cflmax_run, rvol, rvoll[12], possk[12], tlevel[12];
  };
  struct ChkNode { int ilo, ihi, jlo, jhi, level, levelptr, nextfree, pad; double xlo, xhi, ylo, yhi, time; };
  void checkpoint(const std::string& path) {
    sync_stream();
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write checkpoint " + path);
    auto put = [&](const void* d, size_t n) {
      if (n && std::fwrite(d, 1, n, f) != n) { std::fclose(f); throw std::runtime_error("short write to " + path); }
    };
    ChkHead h{};
    h.nvar = nvar; h.f32 = f32 ? 1 : 0; h.mxnest = p.mxnest; h.lfine = lfine; h.ncycle = ncycle; h.frame = frame;
    h.nextout = tk_nextout; h.iout = tk_iout; h.nnodes = (int)node.size(); h.ndfree = ndfree; h.gslots = gslots;
    h.ngrows = (int)grows.size(); h.ngauges = (int)glast.size();
    for (int l = 0; l < 12; ++l) {
      h.icheck[l] = icheck[l]; h.lstart[l] = lstart[l]; h.rvoll[l] = rvoll[l]; h.possk[l] = possk[l];
      h.tlevel[l] = tick_started ? tk_tlevel[l] : time;
    }
    if (!tick_started) {
      h.iout = p.iout; h.nextout = 0;
      if (h.iout == 0) { h.iout = 999999999; h.nextout = p.nout > 0 ? 1 : 0; }
    }
    h.time = time; h.start_time = start_time; h.tmass0 = tmass0; h.cflmax_run = cflmax_run; h.rvol = rvol;
    put(CHK_MAGIC, 8);
    put(&h, sizeof h);
    std::vector<ChkNode> nodes(node.size());
    for (size_t m = 0; m < node.size(); ++m) {
      const HPatch& g = node[m];
      nodes[m] = ChkNode{g.ilo, g.ihi, g.jlo, g.jhi, g.level, g.levelptr, g.nextfree, 0, g.xlo, g.xhi, g.ylo, g.yhi, g.time};
    }
    put(nodes.data(), sizeof(ChkNode) * nodes.size());
    std::vector<char> buf;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
        const HPatch& g = node[m];
        const long long offs[2] = {g.cur == 0 ? g.q0 : g.q1, g.cur == 0 ? g.q1 : g.q0};
        for (long long off : offs) {
          buf.resize(elem() * g.nq);
          AMR_CUDA(cudaMemcpy(buf.data(), reinterpret_cast<char*>(pool.d) + elem() * off, buf.size(), cudaMemcpyDeviceToHost));
          put(buf.data(), buf.size());
        }
      }
    put(glast.data(), sizeof(double) * glast.size());
    put(grows.data(), sizeof(GaugeRow) * grows.size());
    if (gslots) {
      std::vector<double> gv((size_t)gslots * nvar);
      AMR_CUDA(cudaMemcpy(gv.data(), d_gauge_out.d, sizeof(double) * gv.size(), cudaMemcpyDeviceToHost));
      put(gv.data(), sizeof(double) * gv.size());
    }
    if (std::fclose(f) != 0) throw std::runtime_error("cannot close " + path);
  }
  // restrt.f: the grids and scheduler state of a checkpoint, in place of domain.f/setgrd.f
  void restart_from(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot read checkpoint " + path);
    auto get = [&](void* d, size_t n) {
      if (n && std::fread(d, 1, n, f) != n) { std::fclose(f); throw std::runtime_error("checkpoint " + path + " is truncated"); }
    };
    char magic[8];
    get(magic, 8);
    if (std::memcmp(magic, CHK_MAGIC, 8) != 0) { std::fclose(f); throw std::runtime_error(path + " is not a 2D checkpoint of this library"); }
    ChkHead h{};
    get(&h, sizeof h);
    if (h.nvar != nvar || h.f32 != (f32 ? 1 : 0) || h.mxnest != p.mxnest || h.ngauges != (int)p.gauges.size() || h.nnodes < 2 ||
        h.lfine < 1 || h.lfine > p.mxnest) {
      std::fclose(f);
      throw std::runtime_error("checkpoint " + path + " does not match this run (equations, precision, levels or gauges)");
    }
    std::vector<ChkNode> nodes((size_t)h.nnodes);
    get(nodes.data(), sizeof(ChkNode) * nodes.size());
    node.assign(nodes.size(), HPatch());
    for (size_t m = 0; m < nodes.size(); ++m) {
      const ChkNode& c = nodes[m];
      HPatch& g = node[m];
      g.ilo = c.ilo; g.ihi = c.ihi; g.jlo = c.jlo; g.jhi = c.jhi; g.level = c.level; g.levelptr = c.levelptr;
      g.nextfree = c.nextfree; g.xlo = c.xlo; g.xhi = c.xhi; g.ylo = c.ylo; g.yhi = c.yhi; g.time = c.time;
    }
    ndfree = h.ndfree; lfine = h.lfine;
    for (int l = 0; l < 12; ++l) {
      icheck[l] = h.icheck[l]; lstart[l] = h.lstart[l]; rvoll[l] = h.rvoll[l]; possk[l] = h.possk[l]; tk_tlevel[l] = h.tlevel[l];
    }
    ncycle = h.ncycle; frame = h.frame; tk_nextout = h.nextout; tk_iout = h.iout; tick_started = true;
    time = h.time; start_time = h.start_time; tmass0 = h.tmass0; cflmax_run = h.cflmax_run; rvol = h.rvol;
    std::vector<char> buf;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
        alloc_patch(m);
        HPatch& g = node[m];
        g.cur = 0;  // q0 takes store1, q1 store2
        for (long long off : {g.q0, g.q1}) {
          buf.resize(elem() * g.nq);
          get(buf.data(), buf.size());
          AMR_CUDA(cudaMemcpy(reinterpret_cast<char*>(pool.d) + elem() * off, buf.data(), buf.size(), cudaMemcpyHostToDevice));
        }
        h2d_bytes += 2.0 * elem() * g.nq;
      }
    glast.resize((size_t)h.ngauges);
    get(glast.data(), sizeof(double) * glast.size());
    grows.resize((size_t)h.ngrows);
    get(grows.data(), sizeof(GaugeRow) * grows.size());
    gslots = h.gslots;
    if (gslots) {
      std::vector<double> gv((size_t)gslots * nvar);
      get(gv.data(), sizeof(double) * gv.size());
      d_gauge_out.ensure(std::max<size_t>(gv.size() * 2, 4096));
      AMR_CUDA(cudaMemcpy(d_gauge_out.d, gv.data(), sizeof(double) * gv.size(), cudaMemcpyHostToDevice));
    }
    std::fclose(f);
    for (int lev = 1; lev <= p.mxnest; ++lev) touch(lev);
    make_lists();
    for (int lev = 1; lev <= lfine; ++lev) make_bndry(lev);
    sync_descriptors();
    for (int lev = 1; lev <= lfine - 1; ++lev) { prepf(lev + 1); prepc(lev); }
    compile_all();
    ensure_all();
    record_gauges = true;
    stepped = true;
    mbestsrc.assign(p.gauges.size(), 0);
    setbestsrc();
    sync_stream();
  }
  void checkpoint_file(const char* path) {
    if (path && *path) { checkpoint(path); return; }
    char fn[64];
    if (p.checkpt_style < 0) {
      std::snprintf(fn, sizeof(fn), "/fort.chk%s", chk_a ? "aaaaa" : "bbbbb");  // check_twofiles.f
      chk_a = !chk_a;
    } else std::snprintf(fn, sizeof(fn), "/fort.chk%05d", ncycle);
    checkpoint(outdir + fn);
  }
  bool chk_a = true;
  int tk_nextchk = 0;
  bool tk_dumpchk = false, final_chk_done = false;

  // ================================================================ tick.f
  void tick() {
    double dtnew[12];
    double* tlevel = tk_tlevel;
    int ntogo[12];
    if (!tick_started) {
      ncycle = 0;
      setbestsrc();
      tk_iout = p.iout; tk_nextout = 0;
      if (tk_iout == 0) { tk_iout = 999999999; tk_nextout = p.nout > 0 ? 1 : 0; }
      tlevel[1] = time;
      for (int i = 2; i <= p.mxnest; ++i) tlevel[i] = tlevel[1];
      tick_started = true;
    }
    if (tk_nextchk == 0) {
      // tick.f:73-81: checkpoint times still to come
      tk_nextchk = 1;
      while (tk_nextchk <= (int)p.tchk.size() && p.tchk[tk_nextchk - 1] <= time) ++tk_nextchk;
    }
    int& iout = tk_iout;
    int& nextout = tk_nextout;
    int cycles_this_call = 0;
    const double rvol0 = rvol;
    AMR_CUDA(cudaEventRecord(ev_run0, st));
    const auto tstart = std::chrono::steady_clock::now();
    while (!(ncycle >= p.nstop || time >= p.tfinal)) {
      double outtime = (p.nout > 0) ? (nextout <= p.nout ? p.tout[nextout - 1] : RINF) : p.tfinal;
      const double chktime = (tk_nextchk <= (int)p.tchk.size()) ? p.tchk[tk_nextchk - 1] : RINF;
      bool dumpout = false;
      if (time < outtime && time + (double)1.001f * possk[1] >= outtime) {
        possk[1] = outtime - time;
        for (int i = 2; i <= p.mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
        if (p.nout > 0) { ++nextout; dumpout = true; }
      }
      // tick.f:146-157: shorten the step to land on a checkpoint time
      if (time < chktime && time + possk[1] >= chktime) {
        possk[1] = chktime - time;
        for (int i = 2; i <= p.mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
        ++tk_nextchk;
        tk_dumpchk = true;
      } else tk_dumpchk = false;
      int level = 1;
      ntogo[level] = 1;
      for (int i = 1; i <= 10; ++i) dtnew[i] = RINF;
      while (true) {
        int lbase = -1;
        if (icheck[level] >= p.kcheck) lbase = level;
        else if (level + 1 >= p.mxnest) lbase = -1;
        else if (icheck[level + 1] >= p.kcheck) lbase = level + 1;
        else if (level + 2 >= p.mxnest) lbase = -1;
        else if (icheck[level + 2] >= p.kcheck) lbase = level + 2;
        if (lbase > 0) {
          if (!(lbase == p.mxnest || lbase > lfine)) { regrid(lbase); setbestsrc(); }
          for (int i = lbase; i <= lfine; ++i) icheck[i] = 0;
          for (int i = lbase + 1; i <= lfine; ++i) tlevel[i] = tlevel[lbase];
        }
        const double dtl = advanc(level);
#ifdef AMRB_DEBUG_HOOKS
        if (dbg_stop > 0 && ++dbg_count >= dbg_stop) throw DebugStop();
#endif
        ntogo[level] -= 1;
        dtnew[level] = std::min(dtnew[level], dtl);
        tlevel[level] = tlevel[level] + possk[level];
        icheck[level] += 1;
        if (level < lfine) {
          ++level;
          if (((possk[level - 1] - dtnew[level - 1]) / dtnew[level - 1]) > (double)0.05f) {
            const double dttemp = dtnew[level - 1] / kratio[level - 1];
            ntogo[level] = (int)((tlevel[level - 1] - tlevel[level]) / dttemp + (double)0.9f);
          } else ntogo[level] = kratio[level - 1];
          possk[level] = possk[level - 1] / ntogo[level];
          continue;
        }
        bool done = false;
        while (true) {
          if (level == 1) { done = true; break; }
          if (ntogo[level] > 0) {
            while ((possk[level] - dtnew[level]) / dtnew[level] > (double)0.05f) {
              ntogo[level] += 1;
              possk[level] = (tlevel[level - 1] - tlevel[level]) / ntogo[level];
            }
            break;
          }
          --level;
          update(level);
        }
        if (done) break;
      }
      time = time + possk[1];
      ++ncycle;
      if (p.vtime) {
        for (int i = 2; i <= lfine; ++i) { const int ii = lfine + 1 - i; dtnew[ii] = std::min(dtnew[ii], dtnew[ii + 1] * kratio[ii]); }
        dtnew[1] = std::min(dtnew[1], p.dt_max);
        possk[1] = dtnew[1];
        for (int i = 2; i <= p.mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
      }
      // tick.f:322-326
      if (((p.checkpt_style == 3 || p.checkpt_style == -3) && ncycle % p.checkpt_interval == 0) || tk_dumpchk) {
        checkpoint_file(nullptr);
        tk_dumpchk = true;
      }
      if ((ncycle % iout == 0) || dumpout) output(time);
      ++cycles_this_call;
      if (max_cycles > 0 && cycles_this_call >= max_cycles) break;
    }
    // tick.f:365-368: a final checkpoint unless the last step just wrote one
    if (finished() && p.checkpt_style != 0 && !tk_dumpchk && !final_chk_done) {
      checkpoint_file(nullptr);
      final_chk_done = true;
    }
    AMR_CUDA(cudaEventRecord(ev_run1, st));
    sync_stream();
    float ms = 0;
    AMR_CUDA(cudaEventElapsedTime(&ms, ev_run0, ev_run1));
    last_run_ms = ms;
    run_cells = rvol - rvol0;
    t_step += std::chrono::duration<double>(std::chrono::steady_clock::now() - tstart).count();
  }
  bool finished() const { return ncycle >= p.nstop || time >= p.tfinal; }

  // interior values of all grids (levels 1..lfine, list order), layout [m][j][i] per grid
  long long count_values() const {
    long long tot = 0;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) tot += (long long)nvar * node[m].nx() * node[m].ny();
    return tot;
  }
  // gather_values into out (room for count_values() doubles), copied there from the device
  void gather_into(double* out) {
    std::vector<int> pl;
    std::vector<long long> off(1, 0);
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) { pl.push_back(m); off.push_back(off.back() + (long long)nvar * node[m].nx() * node[m].ny()); }
    const long long tot = off.back();
    off.pop_back();
    if (tot == 0) return;
    DBuf<double> d; d.ensure(tot);
    DBuf<int> dp; dp.upload(pl, st, stg);
    DBuf<long long> doff; doff.upload(off, st, stg);
    launch_gather_interior2(pool.d, d_patches.d, dp.d, doff.d, (int)pl.size(), nvar, d.d, st, f32);
    AMR_CUDA(cudaMemcpyAsync(out, d.d, sizeof(double) * tot, cudaMemcpyDeviceToHost, st));
    sync_stream();
    d.free(); dp.free(); doff.free();
  }
  std::vector<double> gather_values() {
    std::vector<double> out((size_t)count_values());
    if (!out.empty()) gather_into(out.data());
    return out;
  }
};

}  // namespace amrb

namespace amrb {

// valout.f90:8-397 (ASCII): |q| < 1e-90 becomes 0 in place on the interior cells, with or
// without files; fort.qNNNN holds per grid (output order) its header and then j-rows of
// i-cells, one line of meqn e26.16 values per cell and a blank line after every row.
void Amr2Gpu::output(double t) {
  const bool binary = p.output_format == 3;  // valout.f90:172-176: nothing zeroed
  for (int lev = 1; lev <= lfine; ++lev) {
    ensure(lev, NEED_STEP);
    if (binary) continue;
    launch_zero_tiny(pool.d, d_patches.d, plan[lev].d_plist.d, (int)plan[lev].plist.size(), nvar, st, f32);
    ++nkernels;
  }
  if (write_output && binary) {
    // fort.q: the grid headers only; fort.b: every grid's whole array, q(m,i,j) with m fastest
    std::vector<int> pl;
    std::vector<long long> off(1, 0);
    FILE* f = open_output(outdir, "fort.q", frame);
    int ngrids = 0;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) {
        const HPatch& g = node[m];
        ++ngrids;
        const int n2[2] = {g.nx(), g.ny()};
        const double lo[2] = {g.xlo, g.ylo}, h[2] = {hxposs[lev], hyposs[lev]};
        write_grid_header(f, 2, m, lev, n2, lo, h);
        pl.push_back(m);
        off.push_back(off.back() + (long long)nvar * (g.nx() + 2 * ng) * (g.ny() + 2 * ng));
      }
    if (std::fclose(f) != 0) throw std::runtime_error("cannot close fort.q in " + outdir);
    std::vector<double> v((size_t)off.back());
    off.pop_back();
    if (!v.empty()) {
      DBuf<double> d; d.ensure(v.size());
      DBuf<int> dp; dp.upload(pl, st, stg);
      DBuf<long long> doff; doff.upload(off, st, stg);
      launch_gather_enlarged2(pool.d, d_patches.d, dp.d, doff.d, (int)pl.size(), nvar, d.d, stepped ? p.dimsplit : 0, st, f32);
      AMR_CUDA(cudaMemcpyAsync(v.data(), d.d, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, st));
      sync_stream();
      d.free(); dp.free(); doff.free();
    }
    write_raw(open_output(outdir, "fort.b", frame, "wb"), v, outdir);
    write_fort_t(outdir, frame, t, nvar, ngrids, p.naux, 2, ng);
  } else if (write_output) {
    const std::vector<double> v = gather_values();
    FILE* f = open_output(outdir, "fort.q", frame);
    size_t pos = 0;
    int ngrids = 0;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) {
        const HPatch& g = node[m];
        ++ngrids;
        const int n2[2] = {g.nx(), g.ny()};
        const double lo[2] = {g.xlo, g.ylo}, h[2] = {hxposs[lev], hyposs[lev]};
        write_grid_header(f, 2, m, lev, n2, lo, h);
        const size_t cells = (size_t)g.nx() * g.ny();
        for (int j = 0; j < g.ny(); ++j) {
          for (int i = 0; i < g.nx(); ++i) {
            for (int mm = 0; mm < nvar; ++mm) std::fputs(fort_e(v[pos + mm * cells + (size_t)j * g.nx() + i], 26, 16).c_str(), f);
            std::fputc('\n', f);
          }
          std::fputs("  \n", f);
        }
        pos += cells * nvar;
      }
    if (std::fclose(f) != 0) throw std::runtime_error("cannot close fort.q in " + outdir);
    write_fort_t(outdir, frame, t, nvar, ngrids, p.naux, 2, ng);
  }
  if (p.out_aux(t)) write_aux(binary);
  ++frame;
}

// src/2d/valout.f90:216-286: fort.aNNNN when aux output is due. The aux arrays do not change
// during a run, so they come from the host copies. ASCII: fort.q's headers and layout, after
// zeroing |aux| < 1e-90 of the interior cells in place (on the device too); binary: every
// grid's whole aux array, aux(m,i,j) with m fastest, nothing zeroed.
void Amr2Gpu::write_aux(bool binary) {
  const int na = p.naux;
  if (!binary)
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) {
        HPatch& g = node[m];
        const int mi = mitot(m), mj = mjtot(m);
        const size_t pl = (size_t)mi * mj;
        bool changed = false;
        for (int a = 0; a < na; ++a)
          for (int j = ng; j < mj - ng; ++j)
            for (int i = ng; i < mi - ng; ++i) {
              double& v = g.haux[a * pl + (size_t)j * mi + i];
              if (std::fabs(v) < 1e-90) {
                if (v != 0.0 || std::signbit(v)) changed = true;
                v = 0.0;
              }
            }
        if (changed) {
          upload_to(reinterpret_cast<char*>(pool.d) + sizeof(double) * g.aux, g.haux.data(), sizeof(double) * g.haux.size());
          // the saved coarse rings copy these values (saveqc.f reads them every step)
          for (int l = 1; l <= p.mxnest; ++l) dirty[l] |= NEED_SAVEQC;
        }
      }
  if (!write_output) return;
  if (binary) {
    std::vector<double> v;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) {
        const HPatch& g = node[m];
        const size_t pl = (size_t)mitot(m) * mjtot(m);
        for (size_t k = 0; k < pl; ++k)
          for (int a = 0; a < na; ++a) v.push_back(g.haux[a * pl + k]);
      }
    write_raw(open_output(outdir, "fort.a", frame, "wb"), v, outdir);
    return;
  }
  FILE* f = open_output(outdir, "fort.a", frame);
  for (int lev = 1; lev <= lfine; ++lev)
    for (int m : lgrids[lev]) {
      const HPatch& g = node[m];
      const int n2[2] = {g.nx(), g.ny()};
      const double lo[2] = {g.xlo, g.ylo}, h[2] = {hxposs[lev], hyposs[lev]};
      write_grid_header(f, 2, m, lev, n2, lo, h);
      const int mi = mitot(m), mj = mjtot(m);
      const size_t pl = (size_t)mi * mj;
      for (int j = ng; j < mj - ng; ++j) {
        for (int i = ng; i < mi - ng; ++i) {
          for (int a = 0; a < na; ++a) std::fputs(fort_e(g.haux[a * pl + (size_t)j * mi + i], 26, 16).c_str(), f);
          std::fputc('\n', f);
        }
        std::fputs("  \n", f);
      }
    }
  if (std::fclose(f) != 0) throw std::runtime_error("cannot close fort.a in " + outdir);
}

}  // namespace amrb

// ============================================================================ C ABI
#include "../../include/amrclaw_b200.h"

namespace amrb {

// The 2D solver behind the C ABI's solver interface.
class Solver2 : public AmrSolver {
 public:
  Amr2Gpu g;
  int num_dim() const override { return 2; }
  cudaStream_t stream() const override { return g.st; }
  void set_batched(bool on) override { g.batched = on; }
  void set_profile(bool on) override { g.profile = on; }
  void set_graphs(bool on) override {
    g.use_graphs = on;
    if (!on) for (auto& G : g.lgraph) G.reset();
  }
  void set_schedule(int s) override {
    if (s != 0) throw std::runtime_error("amrgpu_set_schedule: sweep schedules are built for the 3D path");
  }
  void write_checkpoint(const char* path) override { g.checkpoint_file(path); }
  void set_solver(const std::string& name, const std::vector<double>& v) override {
    g.set_solver(name, v);
    if (g.batch_window_us > 0) {  // the plugin picks the batch this solve's steps join
      StepBatcher::get().leave(g.batch_member);
      StepBatcher::get().join(g.batch_member, StepBatcher::make_key(g.prob.solver, g.f32));
    }
  }
  void set_pool_limit(long long bytes) override { set_arena_limits(g.pool, g.regs, bytes); }
  void set_step_batching(int window_us) override {
    if (window_us < 0) throw std::invalid_argument("amrgpu_set_step_batching: negative window");
    if ((window_us > 0) == (g.batch_window_us > 0)) { g.batch_window_us = window_us; return; }
    if (window_us > 0) StepBatcher::get().join(g.batch_member, StepBatcher::make_key(g.prob.solver, g.f32));
    else StepBatcher::get().leave(g.batch_member);
    g.batch_window_us = window_us;
  }
  void run(int max_cycles) override {
    g.max_cycles = max_cycles;
    g.tick();
    g.ensure_all();
  }
  double level_advance(int level, double* cfl) override {
    if (level < 1 || level > g.lfine) throw std::runtime_error("level out of range");
    const double d = g.advanc(level);
    if (cfl) *cfl = g.cfl_level;
    return d;
  }
  void update_level(int level) override {
    if (level < 1 || level >= g.lfine) throw std::runtime_error("level out of range");
    g.update(level);
    AMR_CUDA(cudaStreamSynchronize(g.st));
  }
  void regrid_from(int lbase) override {
    if (lbase < 1 || lbase > g.lfine || lbase >= g.p.mxnest) throw std::runtime_error("lbase out of range");
    g.regrid(lbase);
    g.setbestsrc();
    g.ensure_all();
  }
  void valout(const char* dir) override {
    const std::string keep = g.outdir;
    const bool kw = g.write_output;
    if (dir) { g.outdir = dir; g.write_output = true; }
    g.output(g.time);
    g.outdir = keep; g.write_output = kw;
  }
  double mass() override { return g.mass(); }
  std::vector<double> info() override {
    return {g.time, g.rvol, (double)g.ncycle, (double)g.lfine, g.t_step, g.t_regrid, g.tmass0,
            g.cflmax_run, (double)g.nkernels, (double)g.pool.peak * 8.0, (double)g.nsteps_launched,
            g.step_kernel_ms, g.step_kernel_cells, g.last_run_ms, g.run_cells, g.finished() ? 1.0 : 0.0, g.h2d_bytes,
            g.tr_flags, g.tr_host, g.tr_cluster, g.tr_fill, g.tr_prep, g.tr_compile, 2.0, g.f32 ? 32.0 : 64.0, (double)g.graph_captures, (double)g.graph_replays, 0.0, 0.0,
            8.0 * (double)(g.pool.cap + g.regs.cap), (double)g.batch_submits, (double)g.batch_shared,
            (double)g.batch_members_seen};
  }
  std::vector<int> grid_rows() override {
    std::vector<int> r;
    for (int lev = 1; lev <= g.lfine; ++lev)
      for (int m : g.lgrids[lev]) {
        const HPatch& h = g.node[m];
        r.insert(r.end(), {m, lev, h.ilo, h.ihi, h.jlo, h.jhi});
      }
    return r;
  }
  std::vector<double> values() override { return g.gather_values(); }
  long long value_count() override { return g.count_values(); }
  void values_into(double* out) override { g.gather_into(out); }
  std::vector<double> gauge_rows() override {
    const int nv = g.nvar;
    std::vector<double> vals((size_t)g.gslots * nv), out;
    if (g.gslots) AMR_CUDA(cudaMemcpy(vals.data(), g.d_gauge_out.d, sizeof(double) * vals.size(), cudaMemcpyDeviceToHost));
    // rows grouped by gauge, in recording order (as each gauge's file would list them)
    for (const auto& G : g.p.gauges)
      for (const auto& r : g.grows) {
        if (r.gauge != G.num) continue;
        out.push_back(r.gauge); out.push_back(r.level); out.push_back(r.t);
        for (int k = 0; k < nv; ++k) out.push_back(vals[(size_t)r.slot * nv + k]);
      }
    return out;
  }
};

}  // namespace amrb

struct amrgpu_ctx {
  std::unique_ptr<amrb::AmrSolver> s;
  amrb::Amr2Gpu* s2 = nullptr;  // the 2D solver, for the 2D-only entry points
  int nvar = 0;
  int device = -1;  // the CUDA device current when the context was created
};

static thread_local std::string g_err;

template <class F>
static int guarded(F&& f) {
  try {
    f();
    return AMRGPU_OK;
  } catch (amrb::PoolLimitError& e) {
    g_err = e.what();
    return AMRGPU_ENOMEM;
  } catch (std::exception& e) {
    g_err = e.what();
    return AMRGPU_ERROR;
  }
}
// the same, with the context's stream ordering its buffer reallocations
template <class F>
static int guarded(amrgpu_ctx* ctx, F&& f) {
  amrb::AllocStreamScope scope(ctx->s->stream());
  return guarded(std::forward<F>(f));
}

extern "C" {

const char* amrgpu_last_error(void) { return g_err.c_str(); }

int amrgpu_init(const char* rundir, const char* outdir, int write_output, amrgpu_ctx** out) {
  return amrgpu_init_precision(rundir, outdir, write_output, 64, out);
}

int amrgpu_init_precision(const char* rundir, const char* outdir, int write_output, int precision_bits, amrgpu_ctx** out) {
  if (!rundir || !out) { g_err = "amrgpu_init: null argument"; return AMRGPU_EINVAL; }
  *out = nullptr;
  if (precision_bits != 64 && precision_bits != 32) { g_err = "amrgpu_init: precision_bits must be 64 or 32"; return AMRGPU_EINVAL; }
  return guarded([&] {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw std::runtime_error("no CUDA device is visible");
    amrb::KeyFile c;
    if (!c.read(std::string(rundir) + "/claw.data")) throw std::runtime_error(std::string("cannot read ") + rundir + "/claw.data");
    const int nd = c.n("num_dim");
    std::unique_ptr<amrgpu_ctx> ctx(new amrgpu_ctx());
    ctx->nvar = c.n("num_eqn");
    AMR_CUDA(cudaGetDevice(&ctx->device));
    if (nd == 2) {
      auto* s2 = new amrb::Solver2();
      ctx->s.reset(s2);
      ctx->s2 = &s2->g;
      s2->g.outdir = outdir ? outdir : "";
      s2->g.write_output = write_output != 0;
      s2->g.f32 = precision_bits == 32;
      s2->g.init(rundir);
    } else if (nd == 3) {
      ctx->s.reset(amrb::make_solver3(rundir, outdir ? outdir : "", write_output != 0, precision_bits == 32));
    } else if (nd == 1) {
      if (precision_bits != 64) throw std::invalid_argument("amrgpu_init: the 1D path is FP64 only");
      ctx->s.reset(amrb::make_solver1(rundir, outdir ? outdir : "", write_output != 0));
    } else {
      throw std::runtime_error("num_dim must be 1, 2 or 3");
    }
    *out = ctx.release();
  });
}

int amrgpu_set_batched(amrgpu_ctx* ctx, int batched) {
  if (!ctx) return AMRGPU_EINVAL;
  ctx->s->set_batched(batched != 0);
  return AMRGPU_OK;
}

int amrgpu_set_graphs(amrgpu_ctx* ctx, int on) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { ctx->s->set_graphs(on != 0); });
}

int amrgpu_set_schedule(amrgpu_ctx* ctx, int schedule) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { ctx->s->set_schedule(schedule); });
}

int amrgpu_checkpoint(amrgpu_ctx* ctx, const char* path) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { ctx->s->write_checkpoint(path); });
}

int amrgpu_set_profile(amrgpu_ctx* ctx, int on) {
  if (!ctx) return AMRGPU_EINVAL;
  ctx->s->set_profile(on != 0);
  return AMRGPU_OK;
}

int amrgpu_set_solver(amrgpu_ctx* ctx, const char* name, const double* params, int n) {
  if (!ctx || !name || n < 0 || (n > 0 && !params)) { g_err = "amrgpu_set_solver: bad argument"; return AMRGPU_EINVAL; }
  try {
    ctx->s->set_solver(name, std::vector<double>(params, params + n));
    return AMRGPU_OK;
  } catch (std::invalid_argument& e) {
    g_err = e.what();
    return AMRGPU_EINVAL;
  } catch (std::exception& e) {
    g_err = e.what();
    return AMRGPU_ERROR;
  }
}

int amrgpu_set_pool_limit(amrgpu_ctx* ctx, long long bytes) {
  if (!ctx) { g_err = "amrgpu_set_pool_limit: null context"; return AMRGPU_EINVAL; }
  try {
    ctx->s->set_pool_limit(bytes);
    return AMRGPU_OK;
  } catch (std::invalid_argument& e) {
    g_err = e.what();
    return AMRGPU_EINVAL;
  } catch (std::exception& e) {
    g_err = e.what();
    return AMRGPU_ERROR;
  }
}

int amrgpu_set_step_batching(amrgpu_ctx* ctx, int window_us) {
  if (!ctx) { g_err = "amrgpu_set_step_batching: null context"; return AMRGPU_EINVAL; }
  try {
    ctx->s->set_step_batching(window_us);
    return AMRGPU_OK;
  } catch (std::invalid_argument& e) {
    g_err = e.what();
    return AMRGPU_EINVAL;
  } catch (std::exception& e) {
    g_err = e.what();
    return AMRGPU_ERROR;
  }
}

int amrgpu_run(amrgpu_ctx* ctx, int max_cycles) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { ctx->s->run(max_cycles); });
}

int amrgpu_level_advance(amrgpu_ctx* ctx, int level, double* dtnew_out, double* cfl_out) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] {
    double cfl = 0;
    const double d = ctx->s->level_advance(level, &cfl);
    if (dtnew_out) *dtnew_out = d;
    if (cfl_out) *cfl_out = cfl;
  });
}

int amrgpu_level_advance_noalloc(amrgpu_ctx* ctx, int level, double* dtnew_out, double* cfl_out) {
  if (!ctx) return AMRGPU_EINVAL;
  if (!ctx->s2) { g_err = "amrgpu_level_advance_noalloc: 2D runs only"; return AMRGPU_EINVAL; }
  if (ctx->s2->f32) { g_err = "amrgpu_level_advance_noalloc: FP64 contexts only"; return AMRGPU_EINVAL; }
  try {
    amrb::Amr2Gpu& s = *ctx->s2;
    if (level < 1 || level > s.lfine) { g_err = "level out of range"; return AMRGPU_EINVAL; }
    // the fixed array is looked up per device: the context's device must be the current one
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != ctx->device) {
      g_err = "amrgpu_level_advance_noalloc: call with the context's device current";
      return AMRGPU_EINVAL;
    }
    double* scratch = nullptr;
    std::string err;
    if (amrb::fixed_scratch_address(&scratch, err) != 0) { g_err = err; return AMRGPU_ERROR; }
    const double d = s.advanc_fixed(level, scratch);
    if (dtnew_out) *dtnew_out = d;
    if (cfl_out) *cfl_out = s.cfl_level;
    return AMRGPU_OK;
  } catch (std::invalid_argument& e) {
    g_err = e.what();
    return AMRGPU_EINVAL;
  } catch (std::exception& e) {
    g_err = e.what();
    return AMRGPU_ERROR;
  }
}

int amrgpu_update(amrgpu_ctx* ctx, int level) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { ctx->s->update_level(level); });
}

int amrgpu_regrid(amrgpu_ctx* ctx, int lbase) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { ctx->s->regrid_from(lbase); });
}

int amrgpu_valout(amrgpu_ctx* ctx, const char* dir) {
  if (!ctx) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { ctx->s->valout(dir); });
}

int amrgpu_mass(amrgpu_ctx* ctx, double* mass_out) {
  if (!ctx || !mass_out) return AMRGPU_EINVAL;
  return guarded(ctx, [&] { *mass_out = ctx->s->mass(); });
}

int amrgpu_info(amrgpu_ctx* ctx, double* out, int n) {
  if (!ctx || !out) return AMRGPU_EINVAL;
  return guarded(ctx, [&] {
    const std::vector<double> v = ctx->s->info();
    for (int k = 0; k < n && k < (int)v.size(); ++k) out[k] = v[k];
  });
}

int amrgpu_grids(amrgpu_ctx* ctx, int* out, int cap, int* n_out) {
  if (!ctx || !n_out) return AMRGPU_EINVAL;
  return guarded(ctx, [&] {
    const std::vector<int> r = ctx->s->grid_rows();
    const int w = 2 + 2 * ctx->s->num_dim();
    const int n = (int)(r.size() / w);
    if (out) std::memcpy(out, r.data(), sizeof(int) * (size_t)w * std::min(cap, n));
    *n_out = n;
  });
}

int amrgpu_values(amrgpu_ctx* ctx, double* out, long long cap, long long* n_out) {
  if (!ctx || !n_out) return AMRGPU_EINVAL;
  return guarded(ctx, [&] {
    // a size query gathers nothing; a buffer with room for every value receives the device
    // copy directly
    const long long n = ctx->s->value_count();
    if (out && cap >= n) ctx->s->values_into(out);
    else if (out) {
      const std::vector<double> v = ctx->s->values();
      std::memcpy(out, v.data(), sizeof(double) * std::min<long long>(cap, (long long)v.size()));
    }
    *n_out = n;
  });
}

int amrgpu_gauges(amrgpu_ctx* ctx, double* out, int cap_rows, int* n_out) {
  if (!ctx || !n_out) return AMRGPU_EINVAL;
  return guarded(ctx, [&] {
    const std::vector<double> v = ctx->s->gauge_rows();
    const int w = 3 + ctx->nvar;
    const int n = (int)(v.size() / w);
    if (out) std::memcpy(out, v.data(), sizeof(double) * (size_t)w * std::min(cap_rows, n));
    *n_out = n;
  });
}

int amrgpu_destroy(amrgpu_ctx* ctx) {
  delete ctx;
  return AMRGPU_OK;
}

#ifdef AMRB_DEBUG_HOOKS
// Debug builds only (-DAMRB_DEBUG_HOOKS): stop after the n-th level substep; read a patch.
int amrgpu_debug_run_substeps(amrgpu_ctx* ctx, int n) {
  amrb::Amr2Gpu& g = *ctx->s2;
  g.dbg_stop = n; g.dbg_count = 0; g.max_cycles = 0;
  int stopped = 0;
  try { g.tick(); } catch (amrb::Amr2Gpu::DebugStop&) { stopped = 1; }
  g.dbg_stop = 0;
  return stopped;
}
long amrgpu_debug_patch(amrgpu_ctx* ctx, int grid, int store, double* out, long cap) {
  amrb::Amr2Gpu& g = *ctx->s2;
  if (grid <= 0 || grid >= (int)g.node.size() || g.node[grid].q0 < 0) return 0;
  const auto& h = g.node[grid];
  const long n = (long)h.nq;
  const long long off = (store == 1) == (h.cur == 0) ? h.q0 : h.q1;
  if (out && cap >= n) {
    cudaStreamSynchronize(g.st);
    if (g.f32) {
      std::vector<float> t(n);
      cudaMemcpy(t.data(), reinterpret_cast<float*>(g.pool.d) + off, sizeof(float) * n, cudaMemcpyDeviceToHost);
      for (long k = 0; k < n; ++k) out[k] = t[k];
    } else {
      cudaMemcpy(out, g.pool.d + off, sizeof(double) * n, cudaMemcpyDeviceToHost);
    }
  }
  return n;
}
#endif

int amrgpu_num_dim(amrgpu_ctx* ctx) { return ctx ? ctx->s->num_dim() : 0; }

}  // extern "C"
