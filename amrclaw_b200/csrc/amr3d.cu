// Host orchestrator of the 3D B200 patch-advance path (3D Euler).
//
// Same organisation as the 2D orchestrator: patches live in a device pool with two
// solution buffers each (store1 / store2 as a ping-pong pair), flux registers in a
// second pool, and the host compiles per regrid the device programs of a level
// substep: ghost fill (src/3d/bound.f, filpatch.f, intfil.f, bc3amr.f90), saved
// coarse values (saveqc.f, cstore.f), the step work (step3.f, flux3.f) with its
// register epilogue (fluxsv.f, fluxad.f), qad jobs (qad.f) and the level sync
// (update.f, upbnd.f). The scheduler (tick.f) and the regrid decisions stay on the
// host; 3D regridding flags whole levels in int8 arrays as the reference does
// (flglvl.f, domprep.f, domshrink.f, domup.f, domcopy.f, spest.f, bufnst.f,
// projec.f, shiftset.f, colate.f, smartbis.f, findcut.f, moment.f, nestck.f,
// grdfit.f, birect.f, gfixup.f, filval.f) with the gradient test on the device.
#include "kernels3d.cuh"
#include "flags3d.cuh"
#include "valout.hpp"
#include "params.hpp"
#include "gridindex.hpp"
#include "workpool.hpp"
#include "hostutil.hpp"
#include "solver.hpp"
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <future>
#include <memory>
#include <vector>

namespace amrb {

namespace {

constexpr int G3 = 2;  // num_ghost

struct HPatch3 {
  int ilo = 0, ihi = 0, jlo = 0, jhi = 0, klo = 0, khi = 0, level = 0, levelptr = 0, nextfree = 0;
  double xlo = 0, xhi = 0, ylo = 0, yhi = 0, zlo = 0, zhi = 0, time = 0;
  long long q0 = -1, q1 = -1, nq = 0;
  long long ffl = -1, nffl = 0;
  long long aux = -1, na = 0;  // aux block: na values, then (time-modulated swirl) na setaux values
  int lenbc = 0;
  int cur = 0;
  bool has_cfl = false;
  std::vector<int> listbc;  // 6 ints per entry (setuse.f): i, j, k (enlarged, 1-based), side, kid, register
  int nx() const { return ihi - ilo + 1; }
  int ny() const { return jhi - jlo + 1; }
  int nz() const { return khi - klo + 1; }
};

struct Prog3 {
  std::vector<Rect3> rects;
  std::vector<Fill3Op> ops;
  std::vector<int> op_stage, op_owner;  // owner: index of the patch (in the level list) the op serves
  std::vector<Bc3Op> bcs;
  std::vector<int> bc_stage, bc_owner;
  std::vector<long long> bc_lines;  // per stage: the most boundary lines of one op (bc3 grid size)
  int nstages = 0, nowners = 0;
  long long scratch_off = -1, scratch_len = 0, scratch_alloc = 0;
  // the scratch starts at zero each run: programs whose rects come from icall copies
  // (saveqc.f, filval.f) leave uncovered cells at the reference's initial 0
  bool zero_scratch = false;
  DBuf<Rect3> d_rects;
  DBuf<Fill3Op> d_ops;
  DBuf<Fill3Chunk> d_chunks;
  DBuf<Bc3Op> d_bcs;
  std::vector<int> ch_lo, ch_hi, bc_lo, bc_hi;
  // [stage][owner] chunk and bc ranges, for replaying the program one patch at a time
  std::vector<int> own_ch_lo, own_ch_hi, own_bc_lo, own_bc_hi;
  void clear() {
    rects.clear(); ops.clear(); op_stage.clear(); op_owner.clear(); bcs.clear(); bc_stage.clear(); bc_owner.clear();
    nstages = 0; nowners = 0; scratch_len = 0; zero_scratch = false;
  }
  int add_rect(int ni, int nj, int nk, int nvar) {
    Rect3 r; r.off = scratch_len; r.ni = ni; r.nj = nj; r.nk = nk;
    scratch_len += Arena::rnd((long long)ni * nj * nk * nvar);
    rects.push_back(r);
    return (int)rects.size() - 1;
  }
  void add_op(const Fill3Op& o, int st, int owner = 0) {
    ops.push_back(o); op_stage.push_back(st); op_owner.push_back(owner); nstages = std::max(nstages, st + 1); nowners = std::max(nowners, owner + 1);
  }
  void add_bc(const Bc3Op& b, int st, int owner = 0) {
    bcs.push_back(b); bc_stage.push_back(st); bc_owner.push_back(owner); nstages = std::max(nstages, st + 1); nowners = std::max(nowners, owner + 1);
  }
  void free_dev() { d_rects.free(); d_ops.free(); d_chunks.free(); d_bcs.free(); }
};

// Appends program S after the ops already in D (rect indices and scratch offsets shifted).
void merge_prog(Prog3& D, const Prog3& S, int owner = 0) {
  const int r0 = (int)D.rects.size();
  const long long s0 = D.scratch_len;
  for (Rect3 r : S.rects) { r.off += s0; D.rects.push_back(r); }
  D.scratch_len += S.scratch_len;
  for (size_t k = 0; k < S.ops.size(); ++k) {
    Fill3Op o = S.ops[k];
    if (o.dst_patch < 0) o.dst_rect += r0;
    if (o.kind != F3_COPY) o.src += r0;
    D.add_op(o, S.op_stage[k], owner);
  }
  for (size_t k = 0; k < S.bcs.size(); ++k) {
    Bc3Op b = S.bcs[k];
    if (b.dst_patch < 0) b.dst_rect += r0;
    D.add_bc(b, S.bc_stage[k], owner);
  }
}

struct Plan3 {
  Prog3 bound, saveqc;
  std::vector<int> plist;
  std::vector<long long> sweep0, comp0, face0, cell0;
  long long items[3] = {0, 0, 0}, faces = 0, cells = 0, slots = 0;  // items: interfaces per direction
  // dimensionally split step: interfaces of the split pencils per direction and patch, the
  // enlarged cells of each patch in the split scratch, and per-patch views of both
  std::vector<long long> scomp0, ecell0;
  long long sitems[3] = {0, 0, 0}, ecells = 0;
  DBuf<long long> d_scomp0, d_ecell0, d_spp;
  std::vector<Fsv3> fsv;
  std::vector<long long> seg0;  // register segments (lenbc) prefix over plist; fad/qad lists are built from it on the device
  std::vector<long long> fsv0;  // fluxsv entries prefix over plist
  long long nseg = 0;
  std::vector<Upbnd3Cell> upc;
  std::vector<Upbnd3Term> upt;
  std::vector<Avg3> avg;
  long long avg_max = 0;  // cells of the largest averaging rectangle
  DBuf<int> d_plist;
  DBuf<long long> d_sweep0, d_comp0, d_face0, d_cell0;
  DBuf<Fsv3> d_fsv;
  DBuf<long long> d_seg0;
  DBuf<Fad3> d_fad;
  DBuf<Qad3Job> d_qad;
  DBuf<Upbnd3Cell> d_upc;
  DBuf<Upbnd3Term> d_upt;
  DBuf<Avg3> d_avg;
  // one-patch views of the sweep prefixes for the per-patch launches of the plain path:
  // per patch, (first, last) slot and (first, last) interface of each direction
  DBuf<long long> d_pp;
  void free_dev() {
    bound.free_dev(); saveqc.free_dev();
    d_plist.free(); d_sweep0.free(); d_comp0.free(); d_face0.free(); d_cell0.free(); d_fsv.free(); d_seg0.free(); d_fad.free(); d_qad.free();
    d_upc.free(); d_upt.free(); d_avg.free(); d_pp.free();
    d_scomp0.free(); d_ecell0.free(); d_spp.free();
  }
};

// a flagged cell (1-based level indices); the reference stores its centre (i-.5, j-.5, k-.5)

// read-only view of a level int8 array (the nesting domain read back for nestck.f)
struct LvlView {
  const int8_t* v; LvlDims d;
  int8_t operator()(int i, int j, int k) const { return v[d.at(i, j, k)]; }
};

struct Tgt3 { int patch, rect, ni, nj, nk; };

}  // namespace

class Amr3Gpu : public AmrSolver {
 public:
  RunParams p;
  Step3Params sp{};
  int nvar = 5;
  double xlower, ylower, zlower, xupper, yupper, zupper;
  // periodic directions (both sides of the direction have mthbc 2)
  bool xperdom = false, yperdom = false, zperdom = false;
  bool anyper() const { return xperdom || yperdom || zperdom; }
  int nxc, nyc, nzc;
  std::vector<HPatch3> node;
  int ndfree = 0, lfine = 1, id_hwm = 1;
  int lstart[12] = {0}, newstl[12] = {0}, listsp[12] = {0}, icheck[12] = {0};
  std::vector<int> lgrids[12];
  GridIndex gidx[12];
  bool gidx_ok[12] = {false};
  double hxposs[12] = {0}, hyposs[12] = {0}, hzposs[12] = {0}, possk[12] = {0};
  int iregsz[12] = {0}, jregsz[12] = {0}, kregsz[12] = {0};
  int intratx[12] = {0}, intraty[12] = {0}, intratz[12] = {0}, kratio[12] = {0};
  Arena pool, regs;
  Staging stg;
  WorkPool pool_host;
  HostProf hprof;
  DBuf<PatchDev> d_patches;
  std::vector<PatchDev> h_patches;
  Plan3 plan[12];
  Prog3 newfill;
  // Richardson estimation (errest.f) of the level being flagged: the ghost fill of the big
  // step, the virtual patches of both steps and their step prefixes
  Prog3 rich_prog;
  DBuf<PatchDev> rich_vp;
  DBuf<int> rich_rect, rich_plist;
  DBuf<long long> rich_pre;
  DBuf<unsigned long long> rich_cfl;
  long long rich_buf = -1, rich_len = 0;
  DBuf<double> d_stash, d_flux;
  DBuf<double> d_split;  // the split step's y-updated values (nvar x enlarged cells of the largest level)
  DBuf<int8_t> lv_a, lv_b, lv_n, lv_t1, lv_t2;   // level flag arrays (flglvl)
  DBuf<LvlBox> lv_boxes, lv_proj;
  DBuf<long long> lv_c0;
  DBuf<int> lv_plist;
  int8_t* lv_host = nullptr;                       // pinned read-back: flags, then the nesting domain
  size_t lv_host_cap = 0;
  DBuf<double> d_gauge_out;
  unsigned long long* d_cfl = nullptr;
  unsigned long long* h_cfl = nullptr;  // pinned
  double* d_mass = nullptr;
  cudaStream_t st = nullptr;
  LevelConst lc{};
  double time = 0, start_time = 0;
  int ncycle = 0;
  double rvol = 0, rvoll[12] = {0};
  double cfl_level = 0, cflmax_run = 0, tmass0 = 0;
  bool batched = true, profile = false, record_gauges = true;
  int max_cycles = 0;
  double t_regrid = 0, t_step = 0, step_kernel_ms = 0, step_kernel_cells = 0, last_run_ms = 0, run_cells = 0, h2d_bytes = 0;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_run0 = nullptr, ev_run1 = nullptr;
  bool tick_started = false;
  int tk_nextout = 0;
  double tk_tlevel[12] = {0};
  long long nkernels = 0, nsteps_launched = 0;
  int frame = 0;
  std::string outdir;
  bool write_output = false;
  // gauges
  std::vector<int> mbestsrc;
  std::vector<double> glast;
  struct GRow { int gauge, level; double t; int slot; };
  std::vector<GRow> grows;
  int gslots = 0;

  ~Amr3Gpu() override {
    if (st) cudaStreamSynchronize(st);
    for (auto& G : lgraph) G.reset();
    if (d_sub) cudaFree(d_sub);
    if (d_queue) cudaFree(d_queue);
    for (cudaEvent_t e : {ev_t0, ev_t1}) if (e) cudaEventDestroy(e);
    if (h_sub) cudaFreeHost(h_sub);
    for (auto& L : plan) L.free_dev();
    newfill.free_dev();
    rich_prog.free_dev();
    rich_vp.free(); rich_rect.free(); rich_plist.free(); rich_pre.free(); rich_cfl.free();
    pool.destroy(); regs.destroy();
    stg.destroy();
    d_patches.free(); d_stash.free(); d_flux.free(); d_split.free(); d_gauge_out.free(); d_aux_jobs.free(); d_aux_fac.free();
    for (DBuf<int8_t>* b : {&lv_a, &lv_b, &lv_n, &lv_t1, &lv_t2}) b->free();
    lv_boxes.free(); lv_proj.free(); lv_c0.free(); lv_plist.free();
    if (lv_host) cudaFreeHost(lv_host);
    if (d_cfl) cudaFree(d_cfl);
    if (h_cfl) cudaFreeHost(h_cfl);
    if (d_mass) cudaFree(d_mass);
    for (cudaEvent_t e : {ev_a, ev_b, ev_run0, ev_run1}) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {sweep_ss.fork, sweep_ss.join[0], sweep_ss.join[1]}) if (e) cudaEventDestroy(e);
    for (cudaStream_t x : sweep_ss.side) if (x) { cudaStreamSynchronize(x); cudaStreamDestroy(x); }
    if (st) cudaStreamDestroy(st);
  }
  SweepStreams sweep_ss{};  // the side streams of the sweep directions
  void sync_stream() { AMR_CUDA(cudaStreamSynchronize(st)); stg.reset(); }

  int mitot(int m) const { return node[m].nx() + 2 * G3; }
  int mjtot(int m) const { return node[m].ny() + 2 * G3; }
  int mktot(int m) const { return node[m].nz() + 2 * G3; }

  // ================================================================ setup
  void setup_problem() {
    if (p.problem == "euler_blast") {
      sp.solver = SOLVER3_EULER;
      if (p.nvar != 5 || p.mwaves != 3) throw std::runtime_error("3D Euler needs num_eqn = 5 and num_waves = 3");
      if (p.naux != 0) throw std::runtime_error("3D Euler: aux arrays are not used");
    } else if (p.problem == "advection_swirl") {
      sp.solver = SOLVER3_SWIRL;
      if (p.nvar != 1 || p.mwaves != 1) throw std::runtime_error("the swirl needs num_eqn = 1 and num_waves = 1");
      if (p.naux != 3 || p.auxtype.size() != 3 || p.auxtype[0] != "xleft" || p.auxtype[1] != "yleft" || p.auxtype[2] != "zleft")
        throw std::runtime_error("the swirl needs 3 aux arrays of types xleft, yleft, zleft");
      const std::string ic = p.ps("ic", "halfspace");
      if (ic != "halfspace" && ic != "sphere") throw std::runtime_error("swirl: ic must be halfspace or sphere");
      swirl_sphere = ic == "sphere";
      sph_x = p.pn("x0", 0.5); sph_y = p.pn("y0", 0.25); sph_z = p.pn("z0", 0.5); sph_r = p.pn("r0", 0.15);
      vel_period = p.pn("vel_period", 0.0);
      // the wall condition negates the momentum components (2..4) of the Euler state
      for (int d = 1; d <= 6; ++d)
        if (p.mthbc[d] != 1) throw std::runtime_error("the swirl takes extrapolation boundaries only");
    } else {
      throw std::runtime_error("3D device path: unknown problem '" + p.problem + "' (euler_blast or advection_swirl)");
    }
    if (p.nghost != G3) throw std::runtime_error("num_ghost must be 2");
    if (p.mcapa != 0) throw std::runtime_error("capacity functions are not supported in 3D");
    // amr3.f90:241-246: Godunov splitting (stepgrid_dimSplit.f) or unsplit; Strang stops the reference
    if (p.dimsplit > 1) throw std::runtime_error("Strang splitting is not supported (dimensional_split must be 0 or 1)");
    if (p.use_fwaves) throw std::runtime_error("f-waves are not supported in 3D");
    if (p.flag_richardson && p.naux > 0) throw std::runtime_error("Richardson estimation needs num_aux = 0 (no auxcoarsen)");
    // bufnst.f:21-24 adds store2's first component to the flags whenever tol > 0: without
    // errest.f having written flags there, that would be the old solution
    if (!p.flag_richardson && p.tol > 0) throw std::runtime_error("flag_richardson_tol > 0 needs flag_richardson");
    for (int d = 1; d <= 6; ++d)
      if (p.mthbc[d] != 1 && p.mthbc[d] != 2 && p.mthbc[d] != 3)
        throw std::runtime_error("3D device path: boundaries must be extrapolation, periodic or wall");
    for (int d = 0; d < 3; ++d)
      if ((p.mthbc[2 * d + 1] == 2) != (p.mthbc[2 * d + 2] == 2))
        throw std::runtime_error("3D device path: a periodic direction needs mthbc 2 on both of its sides");
    xperdom = p.mthbc[1] == 2; yperdom = p.mthbc[3] == 2; zperdom = p.mthbc[5] == 2;
    sp.gamma = p.pn("gamma", 1.4); sp.gamma1 = sp.gamma - 1.0;
    sp.efix = (int)p.pn("efix", 1.0);
    for (int k = 0; k < 3; ++k) sp.mthlim[k] = k < (int)p.mthlim.size() ? p.mthlim[k] : 0;
    sp.order = p.order;
    if (p.trans < 0) throw std::runtime_error("transverse_waves < 0 is not supported");
    sp.m3 = p.trans / 10; sp.m4 = p.trans - 10 * sp.m3;
    if (sp.m3 > 2 || sp.m4 > 2 || (sp.m3 < 2 && sp.m4 == 2) || (sp.m3 >= 1 && sp.order == 1 && sp.m3 == 2))
      throw std::runtime_error("unsupported transverse_waves / order combination");
  }
  double blast_x = 0, blast_y = 0, blast_z = 0, blast_r = 0.2, blast_pin = 5, blast_pout = 1;
  int flag_pressure = 1;
  // swirl: the initial condition is the half space x < 0.5 (tests/advection_3d_swirl/qinit.f)
  // or the sphere of radius r0 about (x0, y0, z0); vel_period > 0 scales the velocity
  // field by cos(pi t / vel_period) before each step (b4step3)
  bool swirl_sphere = false;
  double sph_x = 0.5, sph_y = 0.25, sph_z = 0.5, sph_r = 0.15, vel_period = 0.0;

  // setaux of the swirl (tests/advection_3d_swirl/setaux.f:2-85): u, v, w at the left x-,
  // y- and z-face of every cell of the enlarged patch, as one-dimensional factors
  void aux_factors(const HPatch3& g, double dx, double dy, double dz, double* f) const {
    const int mi = g.nx() + 2 * G3, mj = g.ny() + 2 * G3, mk = g.nz() + 2 * G3;
    const double pi = 4.0 * std::atan(1.0), pi2 = 2.0 * pi;
    const double dx2 = 0.5 * dx, dy2 = 0.5 * dy, dz2 = 0.5 * dz;
    // Each velocity is a product of one-dimensional factors, evaluated left to right:
    //   u(x,y,z) = ((2 sin^2(pi x)) sin(2 pi y)) sin(2 pi z)   at (xc - dx/2, yc, zc)
    //   v(x,y,z) = ((-sin(2 pi x)) sin^2(pi y)) sin(2 pi z)    at (xc, yc - dy/2, zc)
    //   w(x,y,z) = ((-sin(2 pi x)) sin(2 pi y)) sin^2(pi z)    at (xc, yc, zc - dz/2)
    // so the factors are computed once per index along each axis (here, with the host's
    // sin) and multiplied on the device in the same order: the products round as the
    // expressions of setaux.f do. Layout: ua, va, wa [mi], ub, vb, wb [mj], uc, vc, wc [mk].
    double *ua = f, *va = ua + mi, *wa = va + mi, *ub = wa + mi, *vb = ub + mj, *wb = vb + mj;
    double *uc = wb + mj, *vc = uc + mk, *wc = vc + mk;
    for (int i = 1 - G3; i <= g.nx() + G3; ++i) {
      const double xc = g.xlo + (i - 0.5) * dx;
      const double s = std::sin(pi * (xc - dx2));
      ua[i - 1 + G3] = 2.0 * (s * s);
      va[i - 1 + G3] = wa[i - 1 + G3] = -std::sin(pi2 * xc);
    }
    for (int j = 1 - G3; j <= g.ny() + G3; ++j) {
      const double yc = g.ylo + (j - 0.5) * dy;
      const double s = std::sin(pi * (yc - dy2));
      ub[j - 1 + G3] = wb[j - 1 + G3] = std::sin(pi2 * yc);
      vb[j - 1 + G3] = s * s;
    }
    for (int k = 1 - G3; k <= g.nz() + G3; ++k) {
      const double zc = g.zlo + (k - 0.5) * dz;
      const double s = std::sin(pi * (zc - dz2));
      uc[k - 1 + G3] = vc[k - 1 + G3] = std::sin(pi2 * zc);
      wc[k - 1 + G3] = s * s;
    }
  }
  // setaux of new patches (tests/advection_3d_swirl/setaux.f:2-85) into their aux blocks,
  // and into the unscaled copy the time-modulated b4step3 reads
  DBuf<Setaux3Job> d_aux_jobs;
  DBuf<double> d_aux_fac;
  void init_aux(const std::vector<int>& ms) {
    if (p.naux == 0 || ms.empty()) return;
    HPROF("init_aux3");
    std::vector<Setaux3Job> jobs(ms.size());
    long long nf = 0, maxc = 0;
    for (size_t k = 0; k < ms.size(); ++k) {
      const int m = ms[k];
      Setaux3Job& J = jobs[k];
      J.aux = node[m].aux; J.mi = mitot(m); J.mj = mjtot(m); J.mk = mktot(m); J.f0 = nf;
      nf += 3LL * (J.mi + J.mj + J.mk);
      maxc = std::max(maxc, (long long)J.mi * J.mj * J.mk);
    }
    std::vector<double> fac((size_t)nf);
    pool_host.run((int)ms.size(), [&](int k) {
      const HPatch3& g = node[ms[k]];
      aux_factors(g, hxposs[g.level], hyposs[g.level], hzposs[g.level], fac.data() + jobs[k].f0);
    });
    d_aux_jobs.upload(jobs, st, stg);
    d_aux_fac.upload(fac, st, stg);
    launch_setaux3(pool.d, d_aux_jobs.d, (int)jobs.size(), maxc, d_aux_fac.d, vel_period > 0.0 ? 2 : 1, st, f32);
    ++nkernels;
  }

  // qinit (Euler blast): rho = 1, u = 0, p = pin within r0 of the centre, pout outside; layout [m][k][j][i]
  void qinit(const HPatch3& g, double dx, double dy, double dz, std::vector<double>& q) {
    const int mi = g.nx() + 2 * G3, mj = g.ny() + 2 * G3, mk = g.nz() + 2 * G3;
    const long long pl = (long long)mi * mj * mk;
    q.assign((size_t)pl * nvar, 0.0);
    if (sp.solver == SOLVER3_SWIRL) {
      // tests/advection_3d_swirl/qinit.f:5-42 (q = 1 for x < 0.5), or the sphere
      for (int k = 1; k <= g.nz(); ++k) {
        const double zc = g.zlo + (k - 0.5) * dz;
        for (int j = 1; j <= g.ny(); ++j) {
          const double yc = g.ylo + (j - 0.5) * dy;
          for (int i = 1; i <= g.nx(); ++i) {
            const double xc = g.xlo + (i - 0.5) * dx;
            const long long at = ((long long)(k - 1 + G3) * mj + (j - 1 + G3)) * mi + (i - 1 + G3);
            if (swirl_sphere) {
              const double ddx = xc - sph_x, ddy = yc - sph_y, ddz = zc - sph_z;
              q[at] = (ddx * ddx + ddy * ddy + ddz * ddz <= sph_r * sph_r) ? 1.0 : 0.0;
            } else {
              q[at] = (xc < 0.5) ? 1.0 : 0.0;
            }
          }
        }
      }
      return;
    }
    const double g1 = sp.gamma - 1.0;
    for (int k = 1; k <= g.nz(); ++k) {
      const double zc = g.zlo + (k - 0.5) * dz;
      for (int j = 1; j <= g.ny(); ++j) {
        const double yc = g.ylo + (j - 0.5) * dy;
        for (int i = 1; i <= g.nx(); ++i) {
          const double xc = g.xlo + (i - 0.5) * dx;
          const double ddx = xc - blast_x, ddy = yc - blast_y, ddz = zc - blast_z;
          const double r = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
          const double pr = (r <= blast_r) ? blast_pin : blast_pout;
          const long long at = ((long long)(k - 1 + G3) * mj + (j - 1 + G3)) * mi + (i - 1 + G3);
          q[0 * pl + at] = 1.0; q[1 * pl + at] = 0.0; q[2 * pl + at] = 0.0; q[3 * pl + at] = 0.0;
          q[4 * pl + at] = pr / g1;
        }
      }
    }
  }

  // cos(pi t / vel_period): the b4step3 scale of the swirl velocities at the step's start time
  double b4step_factor(double t) const {
    const double pi = 4.0 * std::atan(1.0);
    return std::cos(pi * t / vel_period);
  }
  long long max_enlarged(int lev) const {
    long long mx = 0;
    for (int m : lgrids[lev]) mx = std::max(mx, (long long)mitot(m) * mjtot(m) * mktot(m));
    return mx;
  }

  // ================================================================ node store
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
    node[m] = HPatch3();
    return m;
  }
  void putnod(int m) { node[m].nextfree = ndfree; ndfree = m; }
  // Patch pool offsets count elements of the storage type: doubles, or floats in the FP32
  // form (two per pool double; the pool's 32-double rounding keeps them 256-byte aligned).
  bool f32 = false;
  long long palloc(long long n) { return f32 ? pool.alloc((n + 1) / 2) * 2 : pool.alloc(n); }
  void pfree(long long off, long long n) {
    if (off < 0) return;
    if (f32) pool.release(off / 2, (n + 1) / 2); else pool.release(off, n);
  }
  size_t elem() const { return f32 ? sizeof(float) : sizeof(double); }
  char* pool_bytes() const { return reinterpret_cast<char*>(pool.d); }

  void alloc_patch(int m) {
    id_hwm = std::max(id_hwm, m + 1);
    HPatch3& g = node[m];
    g.nq = (long long)nvar * mitot(m) * mjtot(m) * mktot(m);
    g.q0 = palloc(g.nq);
    g.q1 = palloc(g.nq);
    g.cur = 0;
    if (p.naux > 0) {
      g.na = (long long)p.naux * mitot(m) * mjtot(m) * mktot(m);
      g.aux = palloc(g.na * (vel_period > 0.0 ? 2 : 1));
    }
  }
  void free_patch(int m) {
    HPatch3& g = node[m];
    pfree(g.q0, g.nq); pfree(g.q1, g.nq);
    if (g.aux >= 0) pfree(g.aux, g.na * (vel_period > 0.0 ? 2 : 1));
    g.aux = -1; g.na = 0;
    g.q0 = g.q1 = -1;
    if (g.ffl >= 0) regs.release(g.ffl, g.nffl);
    g.ffl = -1; g.nffl = 0;
  }
  void put_desc(int m) {
    const HPatch3& g = node[m];
    PatchDev& d = h_patches[m];
    d.q[0] = g.q0; d.q[1] = g.q1; d.cur = g.cur; d.ffl = g.ffl;
    d.ilo = g.ilo; d.ihi = g.ihi; d.jlo = g.jlo; d.jhi = g.jhi; d.klo = g.klo; d.khi = g.khi;
    d.mitot = mitot(m); d.mjtot = mjtot(m); d.mktot = mktot(m); d.level = g.level; d.lenbc = g.lenbc;
    d.aux = g.aux;
  }
  void sync_descriptors(const std::vector<int>* extra = nullptr, int extra_levels_below = 0) {
    h_patches.assign(id_hwm, PatchDev{});
    for (int l = 1; l <= p.mxnest; ++l) for (int m : lgrids[l]) put_desc(m);
    if (extra) for (int m : *extra) put_desc(m);
    for (int l = 1; l < extra_levels_below; ++l) for (int m = lstart[l]; m != 0; m = node[m].levelptr) put_desc(m);
    d_patches.upload(h_patches, st, stg);
  }

  // ================================================================ lists
  void touch(int lev) { gidx_ok[lev] = false; }
  const GridIndex& GI(int lev) {
    if (!gidx_ok[lev]) {
      std::vector<int> l;
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) l.push_back(m);
      gidx[lev].build(l, [&](int m) { const HPatch3& g = node[m]; return std::array<int, 6>{g.ilo, g.ihi, g.jlo, g.jhi, g.klo, g.khi}; });
      gidx_ok[lev] = true;
    }
    return gidx[lev];
  }
  void make_lists() {
    for (int lev = 1; lev <= 11; ++lev) {
      lgrids[lev].clear();
      if (lev > p.mxnest) continue;
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) lgrids[lev].push_back(m);
    }
  }
  // regrid.f:122-159: cost nx*ny, most expensive first, quick_sort1.f tie breaking
  static void qsorti(std::vector<int>& ord, int n, const std::vector<long long>& a);
  void arrange(int lev) {
    std::vector<int> gl;
    for (int m = lstart[lev]; m != 0; m = node[m].levelptr) gl.push_back(m);
    const int n = (int)gl.size();
    if (n <= 1) return;
    std::vector<long long> cost(n + 1);
    std::vector<int> ord(n + 1);
    for (int i = 1; i <= n; ++i) cost[i] = (long long)node[gl[i - 1]].nx() * node[gl[i - 1]].ny();
    qsorti(ord, n, cost);
    lstart[lev] = gl[ord[n] - 1];
    int prev = lstart[lev];
    for (int i = 1; i <= n - 1; ++i) { node[prev].levelptr = gl[ord[n - i] - 1]; prev = node[prev].levelptr; }
    node[prev].levelptr = 0;
    touch(lev);
  }
  // birect.f:4-172
  void birect(int m1) {
    int m = m1;
    const int lev = node[m].level;
    const double hx = hxposs[lev], hy = hyposs[lev], hz = hzposs[lev];
    while (true) {
      const int nx = node[m].nx(), ny = node[m].ny(), nz = node[m].nz();
      if (nx + 2 * G3 > p.max1d || ny + 2 * G3 > p.max1d || nz + 2 * G3 > p.max1d) {
        const int dir = (nx + 2 * G3 > p.max1d) ? 0 : (ny + 2 * G3 > p.max1d) ? 1 : 2;
        const int n = dir == 0 ? nx : dir == 1 ? ny : nz;
        int nl = n / 2;
        const int r = lev > 1 ? (dir == 0 ? intratx[lev - 1] : dir == 1 ? intraty[lev - 1] : intratz[lev - 1]) : 2;
        nl = (nl / r) * r;
        const double mid = (dir == 0 ? node[m].xlo + nl * hx : dir == 1 ? node[m].ylo + nl * hy : node[m].zlo + nl * hz);
        const int mn = nodget();
        HPatch3& a = node[m]; HPatch3& b = node[mn];
        b = a;
        b.listbc.clear(); b.q0 = b.q1 = -1; b.ffl = -1;
        b.levelptr = a.levelptr; a.levelptr = mn;
        if (dir == 0) { b.ihi = a.ihi; a.ihi = a.ilo + nl - 1; b.ilo = a.ihi + 1; b.xlo = mid; a.xhi = mid; }
        else if (dir == 1) { b.jhi = a.jhi; a.jhi = a.jlo + nl - 1; b.jlo = a.jhi + 1; b.ylo = mid; a.yhi = mid; }
        else { b.khi = a.khi; a.khi = a.klo + nl - 1; b.klo = a.khi + 1; b.zlo = mid; a.zhi = mid; }
      } else {
        m = node[m].levelptr;
        if (m == 0) break;
      }
    }
  }

  // ================================================================ fill-program compiler
  Bc3Op make_bc(Tgt3 t, double hx, double hy, double hz, double xl, double xr, double yl, double yr, double zl, double zr, bool& any) {
    Bc3Op b{};
    b.dst_patch = t.patch; b.dst_rect = t.rect; b.nrow = t.ni; b.ncol = t.nj; b.nfil = t.nk;
    any = false;
    const double hxm = hx * .01, hym = hy * .01, hzm = hz * .01;
    if (xl < xlower - hxm) { b.nxl = (int)((xlower + hxm - xl) / hx); b.bxl = p.mthbc[1]; any = true; }
    if (xr > xupper + hxm) { const int n = (int)((xr - xupper + hxm) / hx); b.ibeg = std::max(t.ni - n + 1, 1); b.bxr = p.mthbc[2]; any = true; }
    if (yl < ylower - hym) { b.nyl = (int)((ylower + hym - yl) / hy); b.byl = p.mthbc[3]; any = true; }
    if (yr > yupper + hym) { const int n = (int)((yr - yupper + hym) / hy); b.jbeg = std::max(t.nj - n + 1, 1); b.byr = p.mthbc[4]; any = true; }
    if (zl < zlower - hzm) { b.nzl = (int)((zlower + hzm - zl) / hz); b.bzl = p.mthbc[5]; any = true; }
    if (zr > zupper + hzm) { const int n = (int)((zr - zupper + hzm) / hz); b.kbeg = std::max(t.nk - n + 1, 1); b.bzr = p.mthbc[6]; any = true; }
    return b;
  }

  // boxes of cells with mask == 0 (merged row runs per plane, then along k)
  static void runs3(const std::vector<int8_t>& mask, int ni, int nj, int nk, std::vector<std::array<int, 6>>& out) {
    out.clear();
    std::vector<std::array<int, 6>> prevk;
    for (int k = 0; k < nk; ++k) {
      std::vector<std::array<int, 6>> cur;  // i0, j0, k0, w, h, d
      std::vector<int> prevrow;             // runs of the previous row: i0, w, index into cur
      for (int j = 0; j < nj; ++j) {
        std::vector<int> row;
        int i = 0;
        while (i < ni) {
          if (mask[((size_t)k * nj + j) * ni + i] != 0) { ++i; continue; }
          int e = i;
          while (e < ni && mask[((size_t)k * nj + j) * ni + e] == 0) ++e;
          int idx = -1;
          for (size_t q = 0; q < prevrow.size(); q += 3)
            if (prevrow[q] == i && prevrow[q + 1] == e - i) { idx = prevrow[q + 2]; break; }
          if (idx >= 0) cur[idx][4] += 1;
          else { idx = (int)cur.size(); cur.push_back({i, j, k, e - i, 1, 1}); }
          row.push_back(i); row.push_back(e - i); row.push_back(idx);
          i = e;
        }
        prevrow.swap(row);
      }
      // extend boxes of the previous plane that match exactly
      std::vector<std::array<int, 6>> next;
      for (auto& b : cur) {
        bool merged = false;
        for (auto& pb : prevk)
          if (pb[0] == b[0] && pb[1] == b[1] && pb[3] == b[3] && pb[4] == b[4] && pb[2] + pb[5] == k) {
            pb[5] += 1; merged = true; next.push_back(pb); break;
          }
        if (!merged) next.push_back(b);
      }
      for (auto& pb : prevk) {
        bool kept = false;
        for (auto& n2 : next) if (n2[0] == pb[0] && n2[1] == pb[1] && n2[2] == pb[2] && n2[3] == pb[3] && n2[4] == pb[4]) kept = true;
        if (!kept) out.push_back(pb);
      }
      prevk.swap(next);
    }
    for (auto& b : prevk) out.push_back(b);
  }

  // filpatch.f:4-282 (with intfil.f, trimbd.f) as a program; returns the stage completing the region
  int c_filrecur(Prog3& P, int level, Tgt3 T, int nrowst, int ncolst, int nfilst, int ilo, int ihi, int jlo, int jhi, int klo,
                 int khi, bool patchOnly, int msrc) {
    const int ni = ihi - ilo + 1, nj = jhi - jlo + 1, nk = khi - klo + 1;
    std::vector<int8_t> used((size_t)ni * nj * nk, 0);
    auto U = [&](int i, int j, int k) -> int8_t& { return used[((size_t)(k - klo) * nj + (j - jlo)) * ni + (i - ilo)]; };
    std::vector<Fill3Op> copies;
    // the same-level grids that meet the region (intfil.f walks bndList of msrc, the grids
    // next to it; a level's grids are disjoint, so every cell has at most one source and
    // the order of the copies does not matter)
    std::vector<int> src;
    {
      const GridIndex& X = GI(level);
      std::vector<int> hits;
      X.query(ilo, ihi, jlo, jhi, klo, khi, hits);
      // init_bndryList.f keeps the grids that meet msrc grown by nghost in i and j (not k):
      // every source of a ghost strip of width nghost, but not all of a wider ring's
      const HPatch3* gm = msrc > 0 ? &node[msrc] : nullptr;
      for (int r : hits) {
        const int m = X.id(r);
        if (m == msrc) continue;
        if (gm) {
          const HPatch3& q = node[m];
          if (std::max(q.ilo, gm->ilo - G3) > std::min(q.ihi, gm->ihi + G3) || std::max(q.jlo, gm->jlo - G3) > std::min(q.jhi, gm->jhi + G3)) continue;
        }
        src.push_back(m);
      }
    }
    for (int m : src) {
      const HPatch3& g = node[m];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi);
      const int jxlo = std::max(g.jlo, jlo), jxhi = std::min(g.jhi, jhi);
      const int kxlo = std::max(g.klo, klo), kxhi = std::min(g.khi, khi);
      if (!((ixlo <= ixhi && jxlo <= jxhi) && kxlo <= kxhi)) continue;
      Fill3Op o{};
      o.kind = F3_COPY; o.dst_patch = T.patch; o.dst_rect = T.rect;
      o.di0 = nrowst - 1 + (ixlo - ilo); o.dj0 = ncolst - 1 + (jxlo - jlo); o.dk0 = nfilst - 1 + (kxlo - klo);
      o.ni = ixhi - ixlo + 1; o.nj = jxhi - jxlo + 1; o.nk = kxhi - kxlo + 1;
      o.src = m; o.si0 = ixlo - g.ilo + G3; o.sj0 = jxlo - g.jlo + G3; o.sk0 = kxlo - g.klo + G3; o.level = level;
      copies.push_back(o);
      for (int k = kxlo; k <= kxhi; ++k) for (int j = jxlo; j <= jxhi; ++j) for (int i = ixlo; i <= ixhi; ++i) U(i, j, k) = 1;
    }
    // intfil.f:211-260: cells outside the domain count as set (bounds use the destination offsets as the reference does)
    auto mark = [&](int i0, int i1, int j0, int j1, int k0, int k1) {
      for (int k = std::max(k0, klo); k <= std::min(k1, khi); ++k)
        for (int j = std::max(j0, jlo); j <= std::min(j1, jhi); ++j)
          for (int i = std::max(i0, ilo); i <= std::min(i1, ihi); ++i) U(i, j, k) = 1;
    };
    if (khi >= kregsz[level]) mark(ilo, ihi, jlo, jhi, std::max(kregsz[level], klo), khi);
    if (klo < 0) mark(ilo, ihi, jlo, jhi, klo, std::min(-1, nfilst + nk - 1));
    if (jhi >= jregsz[level]) mark(ilo, ihi, std::max(jregsz[level], jlo), jhi, klo, khi);
    if (jlo < 0) mark(ilo, ihi, jlo, std::min(-1, ncolst + nj - 1), klo, khi);
    if (ilo < 0) mark(ilo, std::min(-1, nrowst + ni - 1), jlo, jhi, klo, khi);
    if (ihi >= iregsz[level]) mark(std::max(iregsz[level], ilo), ihi, jlo, jhi, klo, khi);
    // trimbd.f: bounding box of the unset cells
    int il = 1 << 30, ir = -(1 << 30), jl = 1 << 30, jr = -(1 << 30), kl = 1 << 30, kr = -(1 << 30);
    for (int k = klo; k <= khi; ++k) for (int j = jlo; j <= jhi; ++j) for (int i = ilo; i <= ihi; ++i)
      if (!U(i, j, k)) { il = std::min(il, i); ir = std::max(ir, i); jl = std::min(jl, j); jr = std::max(jr, j); kl = std::min(kl, k); kr = std::max(kr, k); }
    int stage = 0;
    if (ir >= il) {
      if (level == 1) throw std::runtime_error("ghost fill: level 1 cells not covered");
      const int rx = intratx[level - 1], ry = intraty[level - 1], rz = intratz[level - 1];
      const int iplo = (il - rx + G3 * rx) / rx - G3, jplo = (jl - ry + G3 * ry) / ry - G3, kplo = (kl - rz + G3 * rz) / rz - G3;
      const int iphi = (ir + rx) / rx, jphi = (jr + ry) / ry, kphi = (kr + rz) / rz;
      const int nrowc = iphi - iplo + 1, ncolc = jphi - jplo + 1, nfilc = kphi - kplo + 1;
      if (nrowc > ni + 2 || ncolc > nj + 2 || nfilc > nk + 2) throw std::runtime_error("ghost fill: coarse box too large");
      const int R = P.add_rect(nrowc, ncolc, nfilc, nvar);
      // filpatch.f:168-179: a coarse box that leaves a periodic domain is filled by prefilrecur
      const bool sticks = iplo < 0 || jplo < 0 || kplo < 0 || iphi >= iregsz[level - 1] || jphi >= jregsz[level - 1] ||
                          kphi >= kregsz[level - 1];
      const Tgt3 C{-1, R, nrowc, ncolc, nfilc};
      const int cst = (anyper() && sticks) ? c_prefil3(P, level - 1, C, iplo, iphi, jplo, jphi, kplo, kphi, iplo, jplo, kplo)
                                           : c_filrecur(P, level - 1, C, 1, 1, 1, iplo, iphi, jplo, jphi, kplo, kphi, true, -1);
      stage = cst + 1;
      std::vector<std::array<int, 6>> boxes;
      runs3(used, ni, nj, nk, boxes);
      for (auto& b : boxes) {
        Fill3Op o{};
        o.kind = F3_INTERP; o.dst_patch = T.patch; o.dst_rect = T.rect;
        o.di0 = nrowst - 1 + b[0]; o.dj0 = ncolst - 1 + b[1]; o.dk0 = nfilst - 1 + b[2];
        o.ni = b[3]; o.nj = b[4]; o.nk = b[5];
        o.src = R; o.si0 = ilo + b[0]; o.sj0 = jlo + b[1]; o.sk0 = klo + b[2]; o.level = level;
        o.cilo = iplo; o.cjlo = jplo; o.cklo = kplo;
        P.add_op(o, stage);
      }
    }
    for (auto& o : copies) P.add_op(o, stage);
    if (patchOnly) {
      bool any;
      const double hx = hxposs[level], hy = hyposs[level], hz = hzposs[level];
      Bc3Op b = make_bc(T, hx, hy, hz, xlower + (double)ilo * hx, xlower + (double)(ihi + 1) * hx, ylower + (double)jlo * hy,
                        ylower + (double)(jhi + 1) * hy, zlower + (double)klo * hz, zlower + (double)(khi + 1) * hz, any);
      if (any) P.add_bc(b, stage);
    }
    return stage;
  }

  // prefilp.f / preicall.f: the three index ranges of one direction (below the domain,
  // inside, above) and the shift that maps each into the domain when it is periodic
  void per_ranges(bool per, int lo, int hi, int n, int st[3], int en[3], int sh[3]) const {
    if (per) {
      st[0] = lo; st[1] = 0; st[2] = n; en[0] = -1; en[1] = n - 1; en[2] = hi; sh[0] = n; sh[1] = 0; sh[2] = -n;
    } else {
      st[0] = n; st[1] = lo; st[2] = n; en[0] = -1; en[1] = hi; en[2] = -1; sh[0] = sh[1] = sh[2] = 0;
    }
  }
  // prefilp.f:1-141 (prefilrecur): region [ilo,ihi]x[jlo,jhi]x[klo,khi] of `level` split into
  // its 27 pieces; each non-empty piece is filled (filrecur, patch-only) into a scratch rect
  // of its own size at its periodically shifted place, then copied into T, whose array
  // starts at index (iglo, jglo, kglo). Returns the stage completing the region.
  int c_prefil3(Prog3& P, int level, Tgt3 T, int ilo, int ihi, int jlo, int jhi, int klo, int khi, int iglo, int jglo, int kglo) {
    int ist[3], iend[3], ish[3], jst[3], jend[3], jsh[3], kst[3], kend[3], ksh[3];
    per_ranges(xperdom, ilo, ihi, iregsz[level], ist, iend, ish);
    per_ranges(yperdom, jlo, jhi, jregsz[level], jst, jend, jsh);
    per_ranges(zperdom, klo, khi, kregsz[level], kst, kend, ksh);
    int done = 0;
    for (int a = 0; a < 3; ++a) {
      const int i1 = std::max(ilo, ist[a]), i2 = std::min(ihi, iend[a]);
      if (i1 > i2) continue;
      for (int b = 0; b < 3; ++b) {
        const int j1 = std::max(jlo, jst[b]), j2 = std::min(jhi, jend[b]);
        if (j1 > j2) continue;
        for (int c = 0; c < 3; ++c) {
          const int k1 = std::max(klo, kst[c]), k2 = std::min(khi, kend[c]);
          if (k1 > k2) continue;
          const int mi = i2 - i1 + 1, mj = j2 - j1 + 1, mk = k2 - k1 + 1;
          const int R = P.add_rect(mi, mj, mk, nvar);
          const int st_ = c_filrecur(P, level, Tgt3{-1, R, mi, mj, mk}, 1, 1, 1, i1 + ish[a], i2 + ish[a], j1 + jsh[b], j2 + jsh[b],
                                     k1 + ksh[c], k2 + ksh[c], true, -1);
          Fill3Op o{};
          o.kind = F3_PIECE; o.dst_patch = T.patch; o.dst_rect = T.rect;
          o.di0 = i1 - iglo; o.dj0 = j1 - jglo; o.dk0 = k1 - kglo; o.ni = mi; o.nj = mj; o.nk = mk;
          o.src = R; o.si0 = 0; o.sj0 = 0; o.sk0 = 0;
          P.add_op(o, st_ + 1);
          done = std::max(done, st_ + 1);
        }
      }
    }
    return done;
  }
  // preicall.f:1-141 / preintcopy.f: icall over the 27 pieces with periodic shifts, each
  // put at its place in T (iput = i1 - ilo + 1)
  void c_preicall3(Prog3& P, Tgt3 T, int ilo, int ihi, int jlo, int jhi, int klo, int khi, int level, int st_) {
    int ist[3], iend[3], ish[3], jst[3], jend[3], jsh[3], kst[3], kend[3], ksh[3];
    per_ranges(xperdom, ilo, ihi, iregsz[level], ist, iend, ish);
    per_ranges(yperdom, jlo, jhi, jregsz[level], jst, jend, jsh);
    per_ranges(zperdom, klo, khi, kregsz[level], kst, kend, ksh);
    for (int a = 0; a < 3; ++a) {
      const int i1 = std::max(ilo, ist[a]), i2 = std::min(ihi, iend[a]);
      if (i1 > i2) continue;
      for (int b = 0; b < 3; ++b) {
        const int j1 = std::max(jlo, jst[b]), j2 = std::min(jhi, jend[b]);
        if (j1 > j2) continue;
        for (int c = 0; c < 3; ++c) {
          const int k1 = std::max(klo, kst[c]), k2 = std::min(khi, kend[c]);
          if (k1 > k2) continue;
          c_icall(P, T, i1 + ish[a], i2 + ish[a], j1 + jsh[b], j2 + jsh[b], k1 + ksh[c], k2 + ksh[c], level, i1 - ilo + 1, j1 - jlo + 1,
                  k1 - klo + 1, st_);
        }
      }
    }
  }

  // bound.f:4-211 for one patch
  void compile_bound_patch(Prog3& P, int lev, int m) { bound_strips(P, lev, m, Tgt3{m, -1, mitot(m), mjtot(m), mktot(m)}, G3); }
  // bound.f with ghost width gw into target T (the enlarged array of patch m, or a scratch
  // rect of the same shape): the six strips, then the physical boundaries
  void bound_strips(Prog3& P, int lev, int m, Tgt3 T, int gw) {
    const HPatch3& g = node[m];
    const int mi = T.ni, mj = T.nj, mk = T.nk;
    const double hx = hxposs[lev], hy = hyposs[lev], hz = hzposs[lev];
    // bound.f:60-199: a strip that leaves a periodic domain is filled by prefilrecur (the
    // x strips also when the patch leaves a periodic y range, the z strips when it leaves
    // a periodic x or y range: their corners lie there)
    const bool xl = g.xlo - gw * hx < xlower, xr = g.xhi + gw * hx > xupper;
    const bool yl = g.ylo - gw * hy < ylower, yr = g.yhi + gw * hy > yupper;
    const bool zl = g.zlo - gw * hz < zlower, zr = g.zhi + gw * hz > zupper;
    const bool ystick = yperdom && (yl || yr), xstick = xperdom && (xl || xr);
    const int iglo = g.ilo - gw, jglo = g.jlo - gw, kglo = g.klo - gw;
    auto strip = [&](bool per, int nrs, int ncs, int nfs, int i0, int i1, int j0, int j1, int k0, int k1) {
      return per ? c_prefil3(P, lev, T, i0, i1, j0, j1, k0, k1, iglo, jglo, kglo)
                 : c_filrecur(P, lev, T, nrs, ncs, nfs, i0, i1, j0, j1, k0, k1, false, m);
    };
    int s = 0;
    s = std::max(s, strip((xperdom && xl) || ystick, 1, 1, gw + 1, g.ilo - gw, g.ilo - 1, g.jlo - gw, g.jhi + gw, g.klo, g.khi));
    s = std::max(s, strip((xperdom && xr) || ystick, mi - gw + 1, 1, gw + 1, g.ihi + 1, g.ihi + gw, g.jlo - gw, g.jhi + gw, g.klo, g.khi));
    s = std::max(s, strip(yperdom && yl, gw + 1, 1, gw + 1, g.ilo, g.ihi, g.jlo - gw, g.jlo - 1, g.klo, g.khi));
    s = std::max(s, strip(yperdom && yr, gw + 1, mj - gw + 1, gw + 1, g.ilo, g.ihi, g.jhi + 1, g.jhi + gw, g.klo, g.khi));
    s = std::max(s, strip((zperdom && zl) || xstick || ystick, 1, 1, 1, g.ilo - gw, g.ihi + gw, g.jlo - gw, g.jhi + gw, g.klo - gw,
                          g.klo - 1));
    s = std::max(s, strip((zperdom && zr) || xstick || ystick, 1, 1, mk - gw + 1, g.ilo - gw, g.ihi + gw, g.jlo - gw, g.jhi + gw,
                          g.khi + 1, g.khi + gw));
    bool any;
    Bc3Op b = make_bc(T, hx, hy, hz, g.xlo - gw * hx, g.xhi + gw * hx, g.ylo - gw * hy, g.yhi + gw * hy, g.zlo - gw * hz, g.zhi + gw * hz, any);
    if (any) P.add_bc(b, s);
  }
  // errest.f:35-76 for patch m: copysol.f puts the old interior in the middle of a scratch
  // rect with twice the ghost width, bound.f fills that ring at the previous time
  void compile_bigstep_patch(Prog3& P, int lev, int m) {
    const HPatch3& g = node[m];
    const int gw = 2 * G3, ni = g.nx() + 2 * gw, nj = g.ny() + 2 * gw, nk = g.nz() + 2 * gw;
    const int R = P.add_rect(ni, nj, nk, nvar);
    Fill3Op o{};
    o.kind = F3_COPY; o.dst_patch = -1; o.dst_rect = R;
    o.di0 = gw; o.dj0 = gw; o.dk0 = gw; o.ni = g.nx(); o.nj = g.ny(); o.nk = g.nz();
    o.src = m; o.si0 = G3; o.sj0 = G3; o.sk0 = G3; o.level = lev;  // the time mode of level lev picks the old values
    P.add_op(o, 0);
    bound_strips(P, lev, m, Tgt3{-1, R, ni, nj, nk}, gw);
  }
  void compile_bound(int lev) {
    HPROF("compile_bound3");
    Prog3& P = plan[lev].bound;
    P.clear();
    for (int l = 1; l <= lev; ++l) GI(l);
    const std::vector<int>& G = lgrids[lev];
    std::vector<Prog3> part(G.size());
    PhaseTimer tph(hprof);
    tph.next("cb_patches");
    pool_host.run((int)G.size(), [&](int k) { compile_bound_patch(part[k], lev, G[k]); });
    tph.next("cb_merge");
    for (size_t k = 0; k < part.size(); ++k) merge_prog(P, part[k], (int)k);
    tph.next("cb_upload");
    upload_prog(P);
  }

  // icall.f / intcopy.f: copies of store1 of the grids of `level` into a target
  void c_icall(Prog3& P, Tgt3 T, int ilo, int ihi, int jlo, int jhi, int klo, int khi, int level, int iput, int jput, int kput, int st_) {
    const GridIndex& X = GI(level);
    std::vector<int> hits;
    X.query(ilo, ihi, jlo, jhi, klo, khi, hits);
    for (int r : hits) {
      const int m = X.id(r);
      const HPatch3& g = node[m];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi), jxlo = std::max(g.jlo, jlo), jxhi = std::min(g.jhi, jhi);
      const int kxlo = std::max(g.klo, klo), kxhi = std::min(g.khi, khi);
      if (!((ixlo <= ixhi && jxlo <= jxhi) && kxlo <= kxhi)) continue;
      Fill3Op o{};
      o.kind = F3_COPY; o.dst_patch = T.patch; o.dst_rect = T.rect;
      o.di0 = ixlo - ilo + iput - 1; o.dj0 = jxlo - jlo + jput - 1; o.dk0 = kxlo - klo + kput - 1;
      o.ni = ixhi - ixlo + 1; o.nj = jxhi - jxlo + 1; o.nk = kxhi - kxlo + 1;
      o.src = m; o.si0 = ixlo - g.ilo + G3; o.sj0 = jxlo - g.jlo + G3; o.sk0 = kxlo - g.klo + G3; o.level = -1;
      P.add_op(o, st_);
    }
  }

  // saveqc.f:3-111 for the kids at level lev+1
  void compile_saveqc(int lev) {
    HPROF("compile_saveqc3");
    Prog3& P = plan[lev].saveqc;
    P.clear();
    P.zero_scratch = true;
    if (lev + 1 > p.mxnest || lstart[lev + 1] == 0) { upload_prog(P); return; }
    GI(lev);
    const double hxc = hxposs[lev], hyc = hyposs[lev], hzc = hzposs[lev];
    const int rx = intratx[lev], ry = intraty[lev], rz = intratz[lev];
    for (int k = lstart[lev + 1]; k != 0; k = node[k].levelptr) {
      const HPatch3& g = node[k];
      const int iclo = g.ilo / rx - 1, jclo = g.jlo / ry - 1, kclo = g.klo / rz - 1;
      const int ichi = (g.ihi + 1) / rx, jchi = (g.jhi + 1) / ry, kchi = (g.khi + 1) / rz;
      const int nrow = ichi - iclo + 1, ncol = jchi - jclo + 1, nfil = kchi - kclo + 1;
      const int R = P.add_rect(nrow, ncol, nfil, nvar);
      Tgt3 T{-1, R, nrow, ncol, nfil};
      // saveqc.f:72-91: the periodic copy where the ring leaves the domain. The reference
      // takes it only with all three directions periodic and leaves the ring's cells beyond
      // a periodic face unset otherwise; here (as in the CPU restatement) it is taken
      // whenever a direction is periodic, which is the reference with three or none
      const bool sticksout = iclo < 0 || ichi == iregsz[lev] || jclo < 0 || jchi == jregsz[lev] || kclo < 0 || kchi == kregsz[lev];
      if (sticksout && anyper()) c_preicall3(P, T, iclo, ichi, jclo, jchi, kclo, kchi, lev, 0);
      else c_icall(P, T, iclo, ichi, jclo, jchi, kclo, kchi, lev, 1, 1, 1, 0);
      bool any;
      Bc3Op b = make_bc(T, hxc, hyc, hzc, g.xlo - hxc, g.xhi + hxc, g.ylo - hyc, g.yhi + hyc, g.zlo - hzc, g.zhi + hzc, any);
      if (any) P.add_bc(b, 0);
      Fill3Op o{};
      o.kind = F3_RING; o.dst_patch = k; o.dst_rect = -1; o.ni = g.lenbc; o.nj = 1; o.nk = 1; o.src = R;
      P.add_op(o, 1);
    }
    upload_prog(P);
  }

  // the stable order by (stage, owner): a counting sort by stage, then (only where the
  // owners of a stage are not already ascending, which merge_prog's appends make them)
  // a stable sort by owner inside the stage
  static std::vector<int> stage_owner_order(const std::vector<int>& stage, const std::vector<int>& owner, int nstages) {
    const size_t n = stage.size();
    std::vector<int> start((size_t)std::max(nstages, 1) + 1, 0), idx(n);
    for (size_t i = 0; i < n; ++i) ++start[stage[i] + 1];
    for (int k = 0; k < nstages; ++k) start[k + 1] += start[k];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (size_t i = 0; i < n; ++i) idx[fill[stage[i]]++] = (int)i;
    for (int k = 0; k < nstages; ++k) {
      auto b = idx.begin() + start[k], e = idx.begin() + start[k + 1];
      bool asc = true;
      for (auto it = b; it != e && asc; ++it) if (it != b && owner[*(it - 1)] > owner[*it]) asc = false;
      if (!asc) std::stable_sort(b, e, [&](int x, int y) { return owner[x] < owner[y]; });
    }
    return idx;
  }
  void upload_prog(Prog3& P) {
    HPROF("upload_prog3");
    if (P.scratch_off >= 0) pfree(P.scratch_off, P.scratch_alloc);
    P.scratch_alloc = std::max<long long>(P.scratch_len, 1);
    P.scratch_off = palloc(P.scratch_alloc);
    std::vector<Rect3> rects = P.rects;
    for (auto& r : rects) r.off += P.scratch_off;
    P.d_rects.upload(rects, st, stg);
    // stage-major, then owner (patch) order: a stage's ops are one range, and so are one
    // patch's ops within a stage (ops of one owner keep their compile order)
    const std::vector<int> oidx = stage_owner_order(P.op_stage, P.op_owner, P.nstages);
    const int no = std::max(P.nowners, 1);
    std::vector<Fill3Op> ops;
    std::vector<Fill3Chunk> ch;
    P.ch_lo.assign(P.nstages, 0); P.ch_hi.assign(P.nstages, 0);
    P.own_ch_lo.assign((size_t)P.nstages * no, 0); P.own_ch_hi.assign((size_t)P.nstages * no, 0);
    int s = -1;
    for (int k : oidx) {
      const int stg_ = P.op_stage[k];
      while (s < stg_) { ++s; P.ch_lo[s] = (int)ch.size(); P.ch_hi[s] = (int)ch.size(); }
      const int id = (int)ops.size();
      ops.push_back(P.ops[k]);
      const size_t ow = (size_t)s * no + P.op_owner[k];
      if (P.own_ch_hi[ow] == P.own_ch_lo[ow]) P.own_ch_lo[ow] = P.own_ch_hi[ow] = (int)ch.size();
      const long long cells = (long long)P.ops[k].ni * P.ops[k].nj * P.ops[k].nk;
      for (long long c0 = 0; c0 < cells; c0 += 128) ch.push_back(Fill3Chunk{id, c0, (int)std::min<long long>(128, cells - c0)});
      P.ch_hi[s] = (int)ch.size();
      P.own_ch_hi[ow] = (int)ch.size();
    }
    while (s + 1 < P.nstages) { ++s; P.ch_lo[s] = P.ch_hi[s] = (int)ch.size(); }
    const std::vector<int> bidx = stage_owner_order(P.bc_stage, P.bc_owner, P.nstages);
    std::vector<Bc3Op> bcs;
    P.bc_lo.assign(P.nstages, 0); P.bc_hi.assign(P.nstages, 0); P.bc_lines.assign(P.nstages, 0);
    P.own_bc_lo.assign((size_t)P.nstages * no, 0); P.own_bc_hi.assign((size_t)P.nstages * no, 0);
    s = -1;
    for (int k : bidx) {
      const int stg_ = P.bc_stage[k];
      while (s < stg_) { ++s; P.bc_lo[s] = (int)bcs.size(); P.bc_hi[s] = (int)bcs.size(); }
      const size_t ow = (size_t)s * no + P.bc_owner[k];
      if (P.own_bc_hi[ow] == P.own_bc_lo[ow]) P.own_bc_lo[ow] = P.own_bc_hi[ow] = (int)bcs.size();
      bcs.push_back(P.bcs[k]);
      P.bc_hi[s] = (int)bcs.size();
      P.own_bc_hi[ow] = (int)bcs.size();
      const Bc3Op& o = P.bcs[k];
      P.bc_lines[s] = std::max(P.bc_lines[s], std::max((long long)o.ncol * o.nfil, std::max((long long)o.nrow * o.nfil, (long long)o.nrow * o.ncol)));
    }
    while (s + 1 < P.nstages) { ++s; P.bc_lo[s] = P.bc_hi[s] = (int)bcs.size(); }
    P.d_ops.upload(ops, st, stg);
    P.d_chunks.upload(ch, st, stg);
    P.d_bcs.upload(bcs, st, stg);
  }

  // one patch's part of a program (the per-patch bound.f call of the plain path)
  void run_prog_owner(Prog3& P, const SrcMode& modes, int owner, const SrcMode* modes_dev = nullptr) {
    const int no = std::max(P.nowners, 1);
    if (owner >= no) return;
    for (int s = 0; s < P.nstages; ++s) {
      const size_t ow = (size_t)s * no + owner;
      if (P.own_ch_hi[ow] > P.own_ch_lo[ow]) {
        Fill3Args a{};
        a.pool = pool.d; a.regs = regs.d; a.patches = d_patches.d; a.rects = P.d_rects.d; a.ops = P.d_ops.d;
        a.chunks = P.d_chunks.d + P.own_ch_lo[ow]; a.nchunks = P.own_ch_hi[ow] - P.own_ch_lo[ow]; a.nvar = nvar; a.modes = modes;
        a.modes_dev = modes_dev;
        a.lc = lc; a.xlower = xlower; a.ylower = ylower; a.zlower = zlower;
        launch_fill3(a, st, f32);
        ++nkernels;
      }
      if (P.own_bc_hi[ow] > P.own_bc_lo[ow]) {
        Bc3Args b{};
        b.pool = pool.d; b.patches = d_patches.d; b.rects = P.d_rects.d; b.ops = P.d_bcs.d + P.own_bc_lo[ow];
        b.nops = P.own_bc_hi[ow] - P.own_bc_lo[ow]; b.nvar = nvar;
        for (int ph = 0; ph < 3; ++ph) launch_bc3(b, ph, st, f32, P.bc_lines[s]);
        nkernels += 3;
      }
    }
  }

  void run_prog(Prog3& P, const SrcMode& modes, const SrcMode* modes_dev = nullptr) {
    if (P.zero_scratch && P.scratch_len > 0 && P.nstages > 0)
      AMR_CUDA(cudaMemsetAsync(pool_bytes() + elem() * P.scratch_off, 0, elem() * P.scratch_len, st));
    for (int s = 0; s < P.nstages; ++s) {
      if (P.ch_hi[s] > P.ch_lo[s]) {
        Fill3Args a{};
        a.pool = pool.d; a.regs = regs.d; a.patches = d_patches.d; a.rects = P.d_rects.d; a.ops = P.d_ops.d;
        a.chunks = P.d_chunks.d + P.ch_lo[s]; a.nchunks = P.ch_hi[s] - P.ch_lo[s]; a.nvar = nvar; a.modes = modes;
        a.modes_dev = modes_dev;
        a.lc = lc; a.xlower = xlower; a.ylower = ylower; a.zlower = zlower;
        launch_fill3(a, st, f32);
        ++nkernels;
      }
      if (P.bc_hi[s] > P.bc_lo[s]) {
        Bc3Args b{};
        b.pool = pool.d; b.patches = d_patches.d; b.rects = P.d_rects.d; b.ops = P.d_bcs.d + P.bc_lo[s];
        b.nops = P.bc_hi[s] - P.bc_lo[s]; b.nvar = nvar;
        for (int ph = 0; ph < 3; ++ph) launch_bc3(b, ph, st, f32, P.bc_lines[s]);
        nkernels += 3;
      }
    }
  }

  // ================================================================ step plan, registers, update plan
  void compile_step(int lev) {
    HPROF("compile_step3");
    Plan3& L = plan[lev];
    L.plist = lgrids[lev];
    const int np = (int)L.plist.size();
    L.sweep0.assign((size_t)3 * (np + 1), 0);
    L.comp0.assign((size_t)3 * (np + 1), 0);
    L.face0.assign(np + 1, 0); L.cell0.assign(np + 1, 0);
    long long slot = 0, comp = 0;
    for (int d = 0; d < 3; ++d) {
      comp = 0;
      for (int k = 0; k < np; ++k) {
        const HPatch3& g = node[L.plist[k]];
        const long long mx = g.nx(), my = g.ny(), mz = g.nz();
        const long long n1 = d == 0 ? mx : d == 1 ? my : mz;
        const long long pencils = d == 0 ? (my + 2) * (mz + 2) : d == 1 ? (mx + 2) * (mz + 2) : (mx + 2) * (my + 2);
        L.sweep0[(size_t)d * (np + 1) + k] = slot;
        L.comp0[(size_t)d * (np + 1) + k] = comp;
        slot += pencils * (n1 + 1);
        comp += pencils * (n1 + 3);
      }
      L.sweep0[(size_t)d * (np + 1) + np] = slot;
      L.comp0[(size_t)d * (np + 1) + np] = comp;
      L.items[d] = comp;
    }
    L.slots = slot;
    for (int k = 0; k < np; ++k) {
      const HPatch3& g = node[L.plist[k]];
      L.face0[k + 1] = L.face0[k] + (long long)(g.nx() + 1) * (g.ny() + 1) * (g.nz() + 1);
      L.cell0[k + 1] = L.cell0[k] + (long long)g.nx() * g.ny() * g.nz();
    }
    L.faces = L.face0[np]; L.cells = L.cell0[np];
    if (p.dimsplit) {
      L.scomp0.assign((size_t)3 * (np + 1), 0);
      L.ecell0.assign(np + 1, 0);
      for (int d = 0; d < 3; ++d) {
        long long c = 0;
        for (int k = 0; k < np; ++k) {
          const HPatch3& g = node[L.plist[k]];
          const long long n1 = d == 0 ? g.nx() : d == 1 ? g.ny() : g.nz();
          L.scomp0[(size_t)d * (np + 1) + k] = c;
          c += split_pencils(d, g.nx(), g.ny(), g.nz()) * (n1 + 3);
        }
        L.scomp0[(size_t)d * (np + 1) + np] = c;
        L.sitems[d] = c;
      }
      for (int k = 0; k < np; ++k) L.ecell0[k + 1] = L.ecell0[k] + (long long)mitot(L.plist[k]) * mjtot(L.plist[k]) * mktot(L.plist[k]);
      L.ecells = L.ecell0[np];
    }
    L.seg0.assign(np + 1, 0);
    std::vector<long long>& fsv0 = L.fsv0;
    fsv0.assign(np + 1, 0);
    for (int k = 0; k < np; ++k) {
      const HPatch3& g = node[L.plist[k]];
      L.seg0[k + 1] = L.seg0[k] + ((lev > 1 && g.ffl >= 0) ? g.lenbc : 0);
      fsv0[k + 1] = fsv0[k] + (g.has_cfl ? (long long)(g.listbc.size() / 6) : 0);
    }
    L.nseg = L.seg0[np];
    // fluxsv.f entries: one per listbc entry of the coarse patches, written in place
    L.fsv.resize(fsv0[np]);
    pool_host.run(np, [&](int k) {
      const int m = L.plist[k];
      const HPatch3& g = node[m];
      if (!g.has_cfl) return;
      Fsv3* out = L.fsv.data() + fsv0[k];
      for (size_t e = 0; e + 5 < g.listbc.size(); e += 6) {
        const int* b = &g.listbc[e];
        Fsv3 f{};
        f.patch = m; f.pidx = k; f.i = b[0] - G3; f.j = b[1] - G3; f.k = b[2] - G3; f.side = b[3];
        f.dst = node[b[4]].ffl + (long long)nvar * (b[5] - 1);
        *out++ = f;
      }
    });
    PhaseTimer tph(hprof);
    tph.next("cs_upload");
    L.d_plist.upload(L.plist, st, stg);
    L.d_sweep0.upload(L.sweep0, st, stg);
    L.d_comp0.upload(L.comp0, st, stg);
    L.d_face0.upload(L.face0, st, stg);
    L.d_cell0.upload(L.cell0, st, stg);
    {
      std::vector<long long> pp((size_t)12 * np, 0);
      for (int k = 0; k < np; ++k)
        for (int d = 0; d < 3; ++d) {
          pp[(size_t)12 * k + 2 * d] = L.sweep0[(size_t)d * (np + 1) + k];
          pp[(size_t)12 * k + 2 * d + 1] = L.sweep0[(size_t)d * (np + 1) + k + 1];
          pp[(size_t)12 * k + 6 + 2 * d] = L.comp0[(size_t)d * (np + 1) + k];
          pp[(size_t)12 * k + 6 + 2 * d + 1] = L.comp0[(size_t)d * (np + 1) + k + 1];
        }
      L.d_pp.upload(pp, st, stg);
    }
    if (p.dimsplit) {
      L.d_scomp0.upload(L.scomp0, st, stg);
      L.d_ecell0.upload(L.ecell0, st, stg);
      // per patch: (first, last) split interface of each direction, then (first, last) scratch cell
      std::vector<long long> spp((size_t)8 * np, 0);
      for (int k = 0; k < np; ++k) {
        for (int d = 0; d < 3; ++d) {
          spp[(size_t)8 * k + 2 * d] = L.scomp0[(size_t)d * (np + 1) + k];
          spp[(size_t)8 * k + 2 * d + 1] = L.scomp0[(size_t)d * (np + 1) + k + 1];
        }
        spp[(size_t)8 * k + 6] = L.ecell0[k];
        spp[(size_t)8 * k + 7] = L.ecell0[k + 1];
      }
      L.d_spp.upload(spp, st, stg);
    }
    L.d_fsv.upload(L.fsv, st, stg);
    L.d_seg0.upload(L.seg0, st, stg);
    L.d_fad.reserve(L.nseg);
    L.d_qad.reserve(L.nseg);
    if (lev > 1 && L.nseg > 0) {
      // the descriptors of this level must be on the device (compile_all uploads them first)
      launch_expand_fadqad3(L.d_plist.d, L.d_seg0.d, np, d_patches.d, intratx[lev - 1], intraty[lev - 1], intratz[lev - 1], L.nseg,
                            L.d_fad.d, L.d_qad.d, st);
      ++nkernels;
    }
    // staging and face-flux buffers sized for the largest level
    tph.next("cs_reserve");
    d_stash.reserve(std::max<size_t>(d_stash.n, (size_t)(L.slots * stash_values(nvar))));
    d_flux.reserve(std::max<size_t>(d_flux.n, (size_t)(L.faces * 6 * nvar)));
    if (p.dimsplit) d_split.reserve(std::max<size_t>(d_split.n, (size_t)(L.ecells * nvar)));
  }

  // update.f:4-192 + upbnd.f:4-94 for coarse level lev
  void compile_update(int lev) {
    HPROF("compile_update3");
    Plan3& L = plan[lev];
    L.upc.clear(); L.upt.clear(); L.avg.clear();
    if (lev < p.mxnest && lstart[lev + 1] != 0) {
      PhaseTimer tph(hprof);
      tph.next("cu_lists");
      const GridIndex& XF = GI(lev + 1);
      const int rx = intratx[lev], ry = intraty[lev], rz = intratz[lev];
      const std::vector<int>& G = lgrids[lev];
      struct Part { std::vector<Upbnd3Cell> upc; std::vector<Upbnd3Term> upt; std::vector<Avg3> avg; };
      std::vector<Part> part(G.size());
      pool_host.run((int)G.size(), [&](int n) { update_lists(G[n], XF, rx, ry, rz, part[n].upc, part[n].upt, part[n].avg); });
      tph.next("cu_merge");
      // the parts in coarse-grid order: offsets by prefix sums, copies in parallel
      const size_t np = part.size();
      std::vector<size_t> oc(np + 1, 0), ot(np + 1, 0), oa(np + 1, 0);
      for (size_t n = 0; n < np; ++n) {
        oc[n + 1] = oc[n] + part[n].upc.size();
        ot[n + 1] = ot[n] + part[n].upt.size();
        oa[n + 1] = oa[n] + part[n].avg.size();
      }
      L.upc.resize(oc[np]); L.upt.resize(ot[np]); L.avg.resize(oa[np]);
      pool_host.run((int)np, [&](int n) {
        const Part& q = part[n];
        for (size_t k = 0; k < q.upc.size(); ++k) { Upbnd3Cell c = q.upc[k]; c.first += (int)ot[n]; L.upc[oc[n] + k] = c; }
        std::copy(q.upt.begin(), q.upt.end(), L.upt.begin() + ot[n]);
        std::copy(q.avg.begin(), q.avg.end(), L.avg.begin() + oa[n]);
      });
    }
    L.avg_max = 0;
    for (const Avg3& a : L.avg) L.avg_max = std::max<long long>(L.avg_max, (long long)a.ni * a.nj * a.nk);
    L.d_upc.upload(L.upc, st, stg); L.d_upt.upload(L.upt, st, stg); L.d_avg.upload(L.avg, st, stg);
  }
  // update.f:4-192 and upbnd.f:4-94 for one coarse patch m: its register cells and the
  // rectangles its kids average into
  void update_lists(int m, const GridIndex& XF, int rx, int ry, int rz, std::vector<Upbnd3Cell>& upc, std::vector<Upbnd3Term>& upt,
                    std::vector<Avg3>& avg) {
    static const double chsign[7] = {0, 1., -1., -1., 1., 1., -1.};
    const HPatch3& g = node[m];
    if (g.has_cfl) {
      // upbnd.f: the entries of one coarse cell in listbc order, each side at most once
      // (the iused bit mask); cells are independent, so they are grouped by a sort
      // (a counting sort by cell over the enlarged patch: stable, so a cell's entries keep
      // their listbc order)
      const int mi = mitot(m), mj = mjtot(m), mk = mktot(m);
      const size_t ne = g.listbc.size() / 6;
      const long long ncell = (long long)mi * mj * mk;
      std::vector<int> start((size_t)ncell + 1, 0), ord(ne);
      auto cell_of = [&](size_t e) {
        const int* b = &g.listbc[6 * e];
        return ((long long)(b[2] - 1) * mj + (b[1] - 1)) * mi + (b[0] - 1);
      };
      for (size_t e = 0; e < ne; ++e) ++start[cell_of(e) + 1];
      for (long long c = 0; c < ncell; ++c) start[c + 1] += start[c];
      {
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (size_t e = 0; e < ne; ++e) ord[fill[cell_of(e)]++] = (int)e;
      }
      for (size_t a0 = 0; a0 < ne;) {
        const long long key = cell_of(ord[a0]);
        const size_t a1 = (size_t)start[key + 1];
        Upbnd3Cell c{};
        c.patch = m; c.ie = (int)(key % mi); c.je = (int)((key / mi) % mj); c.ke = (int)(key / ((long long)mi * mj));
        c.first = (int)upt.size();
        int used = 0;
        for (size_t q = a0; q < a1; ++q) {
          const int* b = &g.listbc[6 * ord[q]];
          const int side = b[3], norm = 1 << (side - 1);
          if ((used / norm) % 2 == 1) continue;
          upt.push_back(Upbnd3Term{node[b[4]].ffl + (long long)nvar * (b[5] - 1), chsign[side]});
          used += norm;
        }
        c.count = (int)upt.size() - c.first;
        upc.push_back(c);
        a0 = a1;
      }
    }
    std::vector<int> hits;
    XF.query(g.ilo * rx, g.ihi * rx + rx - 1, g.jlo * ry, g.jhi * ry + ry - 1, g.klo * rz, g.khi * rz + rz - 1, hits);
    for (int r : hits) {
      const int kk = XF.id(r);
      const HPatch3& f = node[kk];
      const int iclo = f.ilo / rx, jclo = f.jlo / ry, kclo = f.klo / rz, ichi = f.ihi / rx, jchi = f.jhi / ry, kchi = f.khi / rz;
      const int iplo = std::max(g.ilo, iclo), jplo = std::max(g.jlo, jclo), kplo = std::max(g.klo, kclo);
      const int iphi = std::min(g.ihi, ichi), jphi = std::min(g.jhi, jchi), kphi = std::min(g.khi, kchi);
      if (iplo > iphi || jplo > jphi || kplo > kphi) continue;
      Avg3 a{};
      a.cpatch = m; a.kpatch = kk;
      a.ci0 = iplo - g.ilo + G3; a.cj0 = jplo - g.jlo + G3; a.ck0 = kplo - g.klo + G3;
      a.ni = iphi - iplo + 1; a.nj = jphi - jplo + 1; a.nk = kphi - kplo + 1;
      a.fi0 = iplo * rx - f.ilo + G3; a.fj0 = jplo * ry - f.jlo + G3; a.fk0 = kplo * rz - f.klo + G3;
      avg.push_back(a);
    }
  }

  // prepf.f:4-41
  void prepf(int lev) {
    HPROF("prepf3");
    std::vector<std::pair<long long, long long>> zr;
    for (int k = lstart[lev]; k != 0; k = node[k].levelptr) {
      HPatch3& g = node[k];
      const int ik = g.nx() / intratx[lev - 1], jk = g.ny() / intraty[lev - 1], kk = g.nz() / intratz[lev - 1];
      g.lenbc = 2 * (ik * jk + jk * kk + kk * ik);
      if (g.ffl >= 0) regs.release(g.ffl, g.nffl);
      g.nffl = (long long)2 * nvar * g.lenbc;
      g.ffl = regs.alloc(g.nffl);
      zr.emplace_back(g.ffl, Arena::rnd(g.nffl));
    }
    std::sort(zr.begin(), zr.end());
    for (size_t a = 0; a < zr.size();) {
      long long lo = zr[a].first, hi = zr[a].first + zr[a].second;
      size_t b = a + 1;
      while (b < zr.size() && zr[b].first <= hi) { hi = std::max(hi, zr[b].first + zr[b].second); ++b; }
      AMR_CUDA(cudaMemsetAsync(regs.d + lo, 0, sizeof(double) * (hi - lo), st));
      a = b;
    }
  }
  // setuse.f:4-173
  void setuse(std::vector<int>& lb, int mkid, const HPatch3& p_, int iclo, int ichi, int jclo, int jchi, int kclo, int kchi) {
    auto put = [&](int i, int j, int k, int side, int lkid) { lb.insert(lb.end(), {i, j, k, side, mkid, lkid}); };
    const int ilo = p_.ilo, ihi = p_.ihi, jlo = p_.jlo, jhi = p_.jhi, klo = p_.klo, khi = p_.khi;
    const int ist = iclo - 1, iend = ichi + 1, jst = jclo - 1, jend = jchi + 1, kst = kclo - 1, kend = kchi + 1;
    const int ni = ichi - iclo + 1, nj = jchi - jclo + 1, nk = kchi - kclo + 1;
    if (!(ist < ilo))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = (k - kclo) * nj + std::max(jlo, jclo) - jclo + 1;
        for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) put(ist - ilo + G3 + 1, j - jlo + G3 + 1, k - klo + G3 + 1, 3, lkid++);
      }
    if (!(jend > jhi))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = nk * nj + (k - kclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + G3 + 1, jend - jlo + G3 + 1, k - klo + G3 + 1, 4, lkid++);
      }
    if (!(iend > ihi))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = nk * nj + nk * ni + (k - kclo) * nj + std::max(jlo, jclo) - jclo + 1;
        for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) put(iend - ilo + G3 + 1, j - jlo + G3 + 1, k - klo + G3 + 1, 1, lkid++);
      }
    if (!(jst < jlo))
      for (int k = std::max(klo, kclo); k <= std::min(khi, kchi); ++k) {
        int lkid = 2 * nk * nj + nk * ni + (k - kclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + G3 + 1, jst - jlo + G3 + 1, k - klo + G3 + 1, 2, lkid++);
      }
    if (!(kst < klo))
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) {
        int lkid = 2 * nk * nj + 2 * nk * ni + (j - jclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + G3 + 1, j - jlo + G3 + 1, kst - klo + G3 + 1, 6, lkid++);
      }
    if (!(kend > khi))
      for (int j = std::max(jlo, jclo); j <= std::min(jhi, jchi); ++j) {
        int lkid = 2 * nk * nj + 2 * nk * ni + nj * ni + (j - jclo) * ni + std::max(ilo, iclo) - iclo + 1;
        for (int i = std::max(ilo, iclo); i <= std::min(ihi, ichi); ++i) put(i - ilo + G3 + 1, j - jlo + G3 + 1, kend - klo + G3 + 1, 5, lkid++);
      }
  }
  // prepc.f:4-138
  void prepc(int lev) {
    HPROF("prepc3");
    int maxsp = 0;
    for (int k = lstart[lev + 1]; k != 0; k = node[k].levelptr) {
      const HPatch3& f = node[k];
      const int ik = f.nx() / intratx[lev], jk = f.ny() / intraty[lev], kk = f.nz() / intratz[lev];
      maxsp += 2 * (ik * jk + jk * kk + kk * ik);
    }
    listsp[lev] = maxsp;
    if (maxsp == 0) return;
    const GridIndex& XF = GI(lev + 1);
    const int rx = intratx[lev], ry = intraty[lev], rz = intratz[lev];
    std::vector<int> parents;
    for (int mp = lstart[lev]; mp != 0; mp = node[mp].levelptr) parents.push_back(mp);
    // each parent's list depends only on its own box and the kids: built concurrently
    pool_host.run((int)parents.size(), [&](int n) {
      HPatch3& g = node[parents[n]];
      g.listbc.clear();
      g.has_cfl = true;
      // the kids within one coarse cell of the patch, in level order; a patch on a periodic
      // face also meets kids through their periodic images, which can lie anywhere
      const int imax = iregsz[lev] - 1, jmax = jregsz[lev] - 1, kmax = kregsz[lev] - 1;
      const bool wrap = (xperdom && (g.ilo == 0 || g.ihi == imax)) || (yperdom && (g.jlo == 0 || g.jhi == jmax)) ||
                        (zperdom && (g.klo == 0 || g.khi == kmax));
      std::vector<int> kids;
      if (wrap) {
        for (int k = lstart[lev + 1]; k != 0; k = node[k].levelptr) kids.push_back(k);
      } else {
        std::vector<int> hits;
        XF.query((g.ilo - 1) * rx, (g.ihi + 2) * rx - 1, (g.jlo - 1) * ry, (g.jhi + 2) * ry - 1, (g.klo - 1) * rz, (g.khi + 2) * rz - 1, hits);
        for (int r : hits) kids.push_back(XF.id(r));
      }
      const int ni = iregsz[lev], nj = jregsz[lev], nk = kregsz[lev];
      for (int k : kids) {
        const HPatch3& f = node[k];
        const int iclo = f.ilo / rx, jclo = f.jlo / ry, kclo = f.klo / rz, ichi = f.ihi / rx, jchi = f.jhi / ry, kchi = f.khi / rz;
        const int iplo = std::max(g.ilo, iclo), jplo = std::max(g.jlo, jclo), kplo = std::max(g.klo, kclo);
        const int iphi = std::min(g.ihi, ichi), jphi = std::min(g.jhi, jchi), kphi = std::min(g.khi, kchi);
        if ((iplo <= iphi + 1 && jplo <= jphi + 1) && kplo <= kphi + 1) setuse(g.listbc, k, g, iclo, ichi, jclo, jchi, kclo, kchi);
        if (!wrap) continue;
        // prepc.f:84-122: fine grids touching a periodic boundary, through their images
        if (xperdom && g.ilo == 0 && ichi == imax) setuse(g.listbc, k, g, iclo - ni, ichi - ni, jclo, jchi, kclo, kchi);
        if (xperdom && iclo == 0 && g.ihi == imax) setuse(g.listbc, k, g, iclo + ni, ichi + ni, jclo, jchi, kclo, kchi);
        if (yperdom && g.jlo == 0 && jchi == jmax) setuse(g.listbc, k, g, iclo, ichi, jclo - nj, jchi - nj, kclo, kchi);
        if (yperdom && jclo == 0 && g.jhi == jmax) setuse(g.listbc, k, g, iclo, ichi, jclo + nj, jchi + nj, kclo, kchi);
        if (zperdom && g.klo == 0 && kchi == kmax) setuse(g.listbc, k, g, iclo, ichi, jclo, jchi, kclo - nk, kchi - nk);
        if (zperdom && kclo == 0 && g.khi == kmax) setuse(g.listbc, k, g, iclo, ichi, jclo, jchi, kclo + nk, kchi + nk);
      }
    });
  }

  // A regrid marks the plans of the levels it changed; every consumer ensures its own plan
  // before use, so a plan is never used stale. The marked plans are compiled while the GPU
  // runs the level substeps that follow (compile_while_busy), the rest on first use.
  enum { NEED_BOUND = 1, NEED_SAVEQC = 2, NEED_STEP = 4, NEED_UPDATE = 8 };
  int dirty[12] = {0};
  void compile_all(int lbase = 0) {
    HPROF("compile_all3");
    PhaseTimer tph(hprof);
    tph.next("ca_desc");
    sync_descriptors();
    tph.close();
    for (int lev = 1; lev <= p.mxnest; ++lev) {
      if (lev > lfine) { plan[lev].plist.clear(); dirty[lev] = 0; continue; }
      if (lev > lbase) dirty[lev] |= NEED_BOUND;
      if (lev >= lbase) dirty[lev] |= NEED_SAVEQC | NEED_STEP | NEED_UPDATE;
    }
  }
  void ensure(int lev, int what) {
    if (lev < 1 || lev > p.mxnest) return;
    const int todo = dirty[lev] & what;
    if (!todo) return;
    dirty[lev] &= ~todo;
    ++plan_gen[lev];
    if (todo & NEED_BOUND) compile_bound(lev);
    if (todo & NEED_SAVEQC) compile_saveqc(lev);
    if (todo & NEED_STEP) compile_step(lev);
    if (todo & NEED_UPDATE) compile_update(lev);
  }
  // While the substep of level lev runs on the GPU the host compiles marked plans, in the
  // order the next consumers want them: the finer levels' substeps, then the updates from
  // the finest down, then the rest. It stops once the stream has drained (what is left is
  // compiled on first use). No plan compiled here is one the substep in flight reads: that
  // substep's own plans were ensured before its launch, and compiling a plan touches only
  // that plan's buffers and scratch (uploads and stream-ordered reallocations queue behind
  // the substep; a pool growth waits for the device first).
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


  // ================================================================ level substep
  // intfil.f:115-154: which buffer of a source level serves time t (teps = possk/10)
  SrcMode modes_for(int level, double t) {
    SrcMode M{};
    for (int l = 1; l <= level; ++l) {
      if (lgrids[l].empty()) continue;
      const double gt = node[lgrids[l][0]].time;
      const double dt = possk[l];
      const double teps = dt / 10.0;
      const double ac = (gt - t) / dt, ai = 1.0 - ac;
      M.alphai[l] = ai; M.alphac[l] = ac;
      if (ai < -teps || ai > 1.0 + teps) { M.mode[l] = 0; continue; }
      if (std::fabs(ai - 1.0) < teps) M.mode[l] = 0;
      else if (std::fabs(ai) < teps) M.mode[l] = 1;
      else M.mode[l] = 2;
    }
    return M;
  }
  void bound_level(int lev, double t) {
    ensure(lev, NEED_BOUND);
    run_prog(plan[lev].bound, modes_for(lev, t));
  }

  // ---- scalars of a level substep that change from substep to substep; a captured graph
  // reads them from device memory, refreshed by one copy before each replay
  struct Substep3 { SrcMode modes; double dt; double b4c; };
  Substep3* d_sub = nullptr;  // [12] on the device
  Substep3* h_sub = nullptr;  // [12] pinned
  // a level's substep as two CUDA graphs around the gauge sampling: pre (ghost fill,
  // saveqc, and the batched path's qad) and post (CFL reset, b4step3, step kernels,
  // fluxsv/fluxad, flip, CFL read-back). Valid while the level's plans and the buffers
  // they point into stay the same.
  struct LevelGraph {
    cudaGraphExec_t pre = nullptr, post = nullptr;
    long long gen = -1;
    int batched = -1;
    const void* ptrs[7] = {};
    long long kpre = 0, kpost = 0;
    void reset() {
      if (pre) cudaGraphExecDestroy(pre);
      if (post) cudaGraphExecDestroy(post);
      pre = post = nullptr; gen = -1;
    }
  };
  LevelGraph lgraph[12];
  bool use_graphs = false;
  int tune_pending = -1;  // the schedule timed in the substep in flight
  // Sweep schedule of the batched path: per-direction launches (one block per tile) or
  // one persistent work-queue launch over the tiles of all three directions. 1 (the
  // default) and 2 force one schedule. 0 autotunes per level: the level's first substeps
  // alternate the two (step kernels timed with events, per cell-update) until each has
  // TUNE_RUNS samples, then the faster one is kept. On the 3D workloads measured the tuner
  // always kept per-direction launches, and its trial substeps of the queue cost time, so
  // it is not the default. Results are identical under every schedule.
  static constexpr int TUNE_RUNS = 2;
  int schedule = 1;
  struct Tune { int runs[2] = {0, 0}; double ns_per_cell[2] = {0, 0}; int choice = -1; };
  Tune tune[12];
  unsigned int* d_queue = nullptr;
  cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;
  // the schedule of level lev's next substep (0: per direction, 1: queue), and whether to time it
  // (capturing: for a graph, never timed; a level is captured once it is tuned)
  int pick_schedule(int lev, bool& timed, bool capturing) {
    timed = false;
    if (schedule == 1) return 0;
    if (schedule == 2) return 1;
    Tune& T = tune[lev];
    if (T.choice >= 0) return T.choice;
    if (capturing) return 0;
    timed = true;
    return T.runs[1] <= T.runs[0] ? 1 : 0;
  }
  bool tuned(int lev) const { return schedule != 0 || tune[lev].choice >= 0; }
  void tune_record(int lev, int sched, double cells) {
    float ms = 0;
    AMR_CUDA(cudaEventElapsedTime(&ms, ev_t0, ev_t1));
    Tune& T = tune[lev];
    T.ns_per_cell[sched] += 1e6 * ms / std::max(cells, 1.0);
    if (++T.runs[sched] >= TUNE_RUNS && T.runs[1 - sched] >= TUNE_RUNS)
      T.choice = T.ns_per_cell[1] <= T.ns_per_cell[0] ? 1 : 0;
  }
  long long plan_gen[12] = {0};
  long long graph_captures = 0, graph_replays = 0;
  int tune_choices(int which) const {
    int n = 0;
    for (const Tune& T : tune) n += T.choice == which;
    return n;
  }

  // the launches before the gauge sampling (ds: read dt and the fill modes from there)
  void launch_pre(int lev, double t, double dt, const Substep3* ds) {
    Plan3& L = plan[lev];
    const bool kids = lev + 1 <= p.mxnest && lstart[lev + 1] != 0;
    const SrcMode M = modes_for(lev, t);
    const SrcMode* Md = ds ? &ds->modes : nullptr;
    if (batched) {
      // every patch of the level in one launch per routine
      run_prog(L.bound, M, Md);
      if (kids) { SrcMode Z{}; run_prog(L.saveqc, Z); }
      if (lev > 1 && L.nseg > 0) {
        launch_qad3(pool.d, regs.d, d_patches.d, L.d_qad.d, (int)L.nseg, sp, nvar, hxposs[lev], hyposs[lev], hzposs[lev], dt, st, f32,
                    ds ? &ds->dt : nullptr);
        ++nkernels;
      }
    } else {
      // the reference's per-grid structure (advanc.f): bound for every grid, saveqc for the level
      const int np = (int)L.plist.size();
      for (int k = 0; k < np; ++k) run_prog_owner(L.bound, M, k, Md);
      if (kids) { SrcMode Z{}; run_prog(L.saveqc, Z); }
    }
  }
  // the launches after the gauge sampling; timed: bracket the step kernels with ev_a/ev_b
  void launch_post(int lev, double t, double dt, const Substep3* ds, bool timed) {
    Plan3& L = plan[lev];
    const double* dtd = ds ? &ds->dt : nullptr;
    const double* cd = ds ? &ds->b4c : nullptr;
    const double c = vel_period > 0.0 ? b4step_factor(t) : 1.0;
    Step3Args a{};
    a.pool = pool.d; a.patches = d_patches.d; a.sp = sp;
    a.stash = d_stash.d; a.stash_stride = L.slots; a.flux = d_flux.d; a.flux_stride = L.faces;
    a.dt = dt; a.dt_dev = dtd; a.dx = hxposs[lev]; a.dy = hyposs[lev]; a.dz = hzposs[lev]; a.cflmax = d_cfl;
    AMR_CUDA(cudaMemsetAsync(d_cfl, 0, sizeof(unsigned long long), st));
    const double hx = hxposs[lev], hy = hyposs[lev], hz = hzposs[lev];
    if (batched) {
      if (vel_period > 0.0) {
        launch_b4step3(pool.d, d_patches.d, L.d_plist.d, (int)L.plist.size(), p.naux, max_enlarged(lev), c, st, f32, cd);
        ++nkernels;
      }
      if (timed) AMR_CUDA(cudaEventRecord(ev_a, st));
      a.plist = L.d_plist.d; a.np = (int)L.plist.size();
      a.sweep0 = L.d_sweep0.d; a.comp0 = L.d_comp0.d; a.face0 = L.d_face0.d; a.cell0 = L.d_cell0.d;
      if (p.dimsplit) {
        // stepgrid_dimSplit.f: x, y, z sweeps with their updates, one launch each
        a.scomp0 = L.d_scomp0.d; a.ecell0 = L.d_ecell0.d; a.split = d_split.d;
        nkernels += launch_split3(a, L.sitems, st, f32);
      } else {
        bool tt = false;
        const int sched = pick_schedule(lev, tt, ds != nullptr);
        a.queue = sched == 1 ? d_queue : nullptr;
        if (tt) AMR_CUDA(cudaEventRecord(ev_t0, st));
        nkernels += launch_step3(a, L.items, L.faces, L.cells, st, f32, &sweep_ss);
        if (tt) { AMR_CUDA(cudaEventRecord(ev_t1, st)); tune_pending = sched; }
      }
      if (timed) AMR_CUDA(cudaEventRecord(ev_b, st));
      if (!L.fsv.empty()) {
        launch_fsv3(d_flux.d, L.faces, L.d_face0.d, d_patches.d, regs.d, L.d_fsv.d, (int)L.fsv.size(), nvar, dt, hx, hy, hz, st, f32, dtd);
        ++nkernels;
      }
      if (lev > 1 && L.nseg > 0) {
        launch_fad3(d_flux.d, L.faces, L.d_face0.d, d_patches.d, regs.d, L.d_fad.d, (int)L.nseg, nvar, dt, hx, hy, hz, st, f32, dtd);
        ++nkernels;
      }
    } else {
      // par_advanc per grid (qad, b4step3, stepgrid, fluxsv, fluxad), each grid its own
      // launches; the per-grid arrays are views of the level's
      const int np = (int)L.plist.size();
      if (timed) AMR_CUDA(cudaEventRecord(ev_a, st));
      for (int k = 0; k < np; ++k) {
        const long long q0 = L.seg0[k], nq = L.seg0[k + 1] - L.seg0[k];
        if (lev > 1 && nq > 0) {
          launch_qad3(pool.d, regs.d, d_patches.d, L.d_qad.d + q0, (int)nq, sp, nvar, hx, hy, hz, dt, st, f32, dtd);
          ++nkernels;
        }
        if (vel_period > 0.0) {
          const int m = L.plist[k];
          launch_b4step3(pool.d, d_patches.d, L.d_plist.d + k, 1, p.naux, (long long)mitot(m) * mjtot(m) * mktot(m), c, st, f32, cd);
          ++nkernels;
        }
        Step3Args b = a;
        b.plist = L.d_plist.d + k; b.np = 1;
        b.sweep0 = L.d_pp.d + (size_t)12 * k; b.comp0 = L.d_pp.d + (size_t)12 * k + 6;
        b.face0 = L.d_face0.d + k; b.cell0 = L.d_cell0.d + k;
        long long it[3];
        if (p.dimsplit) {
          b.scomp0 = L.d_spp.d + (size_t)8 * k; b.ecell0 = L.d_spp.d + (size_t)8 * k + 6; b.split = d_split.d;
          for (int d = 0; d < 3; ++d) it[d] = L.scomp0[(size_t)d * (np + 1) + k + 1] - L.scomp0[(size_t)d * (np + 1) + k];
          nkernels += launch_split3(b, it, st, f32);
        } else {
          for (int d = 0; d < 3; ++d) it[d] = L.comp0[(size_t)d * (np + 1) + k + 1] - L.comp0[(size_t)d * (np + 1) + k];
          nkernels += launch_step3(b, it, L.face0[k + 1] - L.face0[k], L.cell0[k + 1] - L.cell0[k], st, f32, &sweep_ss);
        }
        const long long f0 = L.fsv0[k], nf = L.fsv0[k + 1] - L.fsv0[k];
        if (nf > 0) {
          launch_fsv3(d_flux.d, L.faces, L.d_face0.d, d_patches.d, regs.d, L.d_fsv.d + f0, (int)nf, nvar, dt, hx, hy, hz, st, f32, dtd);
          ++nkernels;
        }
        if (lev > 1 && nq > 0) {
          launch_fad3(d_flux.d, L.faces, L.d_face0.d, d_patches.d, regs.d, L.d_fad.d + q0, (int)nq, nvar, dt, hx, hy, hz, st, f32, dtd);
          ++nkernels;
        }
      }
      if (timed) AMR_CUDA(cudaEventRecord(ev_b, st));
    }
    launch_flip(d_patches.d, L.d_plist.d, (int)L.plist.size(), st);
    ++nkernels;
    // into pinned memory, so the copy is queued and the host goes on compiling
    AMR_CUDA(cudaMemcpyAsync(h_cfl, d_cfl, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  }
  // captures the level's two graphs if the current ones do not fit the plans and buffers
  void ensure_graphs(int lev) {
    LevelGraph& G = lgraph[lev];
    const void* ptrs[7] = {pool.d, regs.d, d_patches.d, d_stash.d, d_flux.d, d_cfl, d_split.d};
    bool ok = G.pre && G.gen == plan_gen[lev] && G.batched == (int)batched;
    for (int k = 0; k < 7 && ok; ++k) ok = G.ptrs[k] == ptrs[k];
    if (ok) return;
    HPROF("graph_capture3");
    G.reset();
    const Substep3* ds = d_sub + lev;
    const double t = node[lgrids[lev][0]].time, dt = possk[lev];
    for (int part = 0; part < 2; ++part) {
      cudaGraph_t g = nullptr;
      const long long k0 = nkernels;
      AMR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      if (part == 0) launch_pre(lev, t, dt, ds);
      else launch_post(lev, t, dt, ds, false);
      AMR_CUDA(cudaStreamEndCapture(st, &g));
      AMR_CUDA(cudaGraphInstantiate(part == 0 ? &G.pre : &G.post, g, 0));
      AMR_CUDA(cudaGraphDestroy(g));
      (part == 0 ? G.kpre : G.kpost) = nkernels - k0;
      nkernels = k0;
    }
    G.gen = plan_gen[lev]; G.batched = (int)batched;
    for (int k = 0; k < 7; ++k) G.ptrs[k] = ptrs[k];
    ++graph_captures;
  }

  // advanc.f:4-139 with par_advanc (:166-303): the level substep, batched (every patch of
  // the level in one launch per routine) or plain (the reference's per-grid launches),
  // launched directly or replayed from captured graphs
  double advanc(int lev) {
    HPROF("advanc3");
    ensure(lev, NEED_BOUND | NEED_SAVEQC | NEED_STEP);
    PhaseTimer tph(hprof);
    Plan3& L = plan[lev];
    const double t = node[lgrids[lev][0]].time;
    const double dt = possk[lev];
    tph.next("adv_launch");
    // with graphs, a level's substeps launch directly until its sweep schedule is tuned
    if (use_graphs && (!batched || tuned(lev))) {
      ensure_graphs(lev);
      Substep3& h = h_sub[lev];
      h.modes = modes_for(lev, t); h.dt = dt; h.b4c = vel_period > 0.0 ? b4step_factor(t) : 1.0;
      AMR_CUDA(cudaMemcpyAsync(d_sub + lev, &h, sizeof(Substep3), cudaMemcpyHostToDevice, st));
      AMR_CUDA(cudaGraphLaunch(lgraph[lev].pre, st));
      sample_gauges(lev);
      if (profile) AMR_CUDA(cudaEventRecord(ev_a, st));
      AMR_CUDA(cudaGraphLaunch(lgraph[lev].post, st));
      if (profile) AMR_CUDA(cudaEventRecord(ev_b, st));
      nkernels += lgraph[lev].kpre + lgraph[lev].kpost;
      graph_replays += 2;
    } else {
      launch_pre(lev, t, dt, nullptr);
      sample_gauges(lev);
      launch_post(lev, t, dt, nullptr, profile);
    }
    for (int m : lgrids[lev]) { node[m].cur ^= 1; h_patches[m].cur = node[m].cur; }
    tph.next("adv_compile");
    compile_while_busy(lev);
    tph.next("adv_sync");
    sync_stream();
    const unsigned long long cbits = *h_cfl;
    tph.close();
    double cmax;
    std::memcpy(&cmax, &cbits, sizeof(double));
    if (profile) {
      float ms = 0;
      AMR_CUDA(cudaEventElapsedTime(&ms, ev_a, ev_b));
      step_kernel_ms += ms;
      step_kernel_cells += (double)L.cells;
    }
    if (tune_pending >= 0) { tune_record(lev, tune_pending, (double)L.cells); tune_pending = -1; }
    for (int m : lgrids[lev]) {
      node[m].time = node[m].time + dt;
      const double cells = (double)node[m].nx() * node[m].ny() * node[m].nz();
      rvol += cells; rvoll[lev] += cells;
    }
    cfl_level = cmax;
    cflmax_run = std::max(cflmax_run, cmax);
    ++nsteps_launched;
    stepped = true;
    return cmax > 0.0 ? dt * p.cfl_desired / cmax : RINF;
  }
  // one-patch views of the sweep prefixes for the plain path, 12 per patch:
  // stash slots [x0, x1, y0, y1, z0, z1], then interfaces [x0, x1, y0, y1, z0, z1]

  // update.f:4-192 (upbnd then averaging)
  void update(int lev) {
    HPROF("update3");
    ensure(lev, NEED_UPDATE);
    Plan3& L = plan[lev];
    const double vol = hxposs[lev] * hyposs[lev] * hzposs[lev];
    launch_upbnd3(pool.d, regs.d, d_patches.d, L.d_upc.d, (int)L.upc.size(), L.d_upt.d, vol, nvar, st, f32);
    launch_average3(pool.d, d_patches.d, L.d_avg.d, (int)L.avg.size(), L.avg_max, intratx[lev], intraty[lev], intratz[lev], nvar, st, f32);
    nkernels += 2;
  }

  // ================================================================ gauges (gauges_module.f90:302-460)
  void setbestsrc() {
    mbestsrc.assign(p.gauges.size(), 0);
    for (size_t i = 0; i < p.gauges.size(); ++i)
      for (int lev = lfine; lev >= 1 && mbestsrc[i] == 0; --lev)
        for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
          const HPatch3& g = node[m];
          const GaugeSpec& G = p.gauges[i];
          if (G.x >= g.xlo && G.x <= g.xhi && G.y >= g.ylo && G.y <= g.yhi && G.z >= g.zlo && G.z <= g.zhi) { mbestsrc[i] = m; break; }
        }
  }
  void sample_gauges(int lev) {
    if (!record_gauges || p.gauges.empty()) return;
    std::vector<Gauge3Job> jobs;
    const double hx = hxposs[lev], hy = hyposs[lev], hz = hzposs[lev];
    for (size_t i = 0; i < p.gauges.size(); ++i) {
      const int m = mbestsrc[i];
      if (m == 0 || node[m].level != lev) continue;
      const GaugeSpec& G = p.gauges[i];
      const double tg = node[m].time;
      if (tg < G.t1 || tg > G.t2) continue;
      if (tg - glast[i] < G.min_inc) continue;
      const double xlow = node[m].xlo - G3 * hx, ylow = node[m].ylo - G3 * hy, zlow = node[m].zlo - G3 * hz;
      Gauge3Job J{};
      J.patch = m;
      J.ii = (int)(0.5 + (G.x - xlow) / hx); J.jj = (int)(0.5 + (G.y - ylow) / hy); J.kk = (int)(0.5 + (G.z - zlow) / hz);
      J.xoff = (G.x - (xlow + (J.ii - 0.5) * hx)) / hx; J.yoff = (G.y - (ylow + (J.jj - 0.5) * hy)) / hy;
      J.zoff = (G.z - (zlow + (J.kk - 0.5) * hz)) / hz;
      J.slot = gslots++;
      jobs.push_back(J);
      grows.push_back(GRow{G.num, lev, tg, J.slot});
      glast[i] = tg;
    }
    if (jobs.empty()) return;
    if ((size_t)gslots * nvar > d_gauge_out.cap) {
      DBuf<double> nb; nb.ensure(std::max<size_t>((size_t)gslots * nvar * 2, 4096));
      if (d_gauge_out.d) AMR_CUDA(cudaMemcpyAsync(nb.d, d_gauge_out.d, sizeof(double) * d_gauge_out.cap, cudaMemcpyDeviceToDevice, st));
      sync_stream();
      d_gauge_out.free(); d_gauge_out = nb;
    }
    DBuf<Gauge3Job> dj; dj.upload(jobs, st, stg);
    launch_gauges3(pool.d, d_patches.d, dj.d, (int)jobs.size(), nvar, d_gauge_out.d, st, f32);
    sync_stream();
    dj.free();
  }

  // ================================================================ regrid: level flag arrays on the device
  // errest.f:4-141 for the grids G of level lcheck, launched on the stream: the big step
  // (2*dt, 2*h on the old values coarsened by 2, ghost ring of twice the width filled at
  // t-dt), the regular step (dt, h on the values spest.f flags: store1 with its ghost
  // cells just filled) and errf1.f's estimate of component 1; when tol > 0 the flagged
  // blocks add BADPT to the level array f (bufnst.f:21-24 with setflags.f). Both steps run
  // the level step kernels on "virtual patches": pool arrays with descriptors of their own
  // and no flux registers; their Courant numbers and dtnew are dropped (the next advanc.f
  // resets cfl_level). richardson_release frees the buffers after the stream syncs.
  void richardson_launch(int lcheck, const std::vector<int>& G, int8_t* f, LvlDims dl) {
    HPROF("richardson3");
    const int np = (int)G.size();
    const double hx = hxposs[lcheck], hy = hyposs[lcheck], hz = hzposs[lcheck], dt = possk[lcheck];
    const double tpre = node[G[0]].time - dt;
    Prog3& P = rich_prog;
    P.clear();
    P.zero_scratch = true;
    for (int l = 1; l <= lcheck; ++l) GI(l);
    std::vector<Prog3> part(np);
    pool_host.run(np, [&](int k) { compile_bigstep_patch(part[k], lcheck, G[k]); });
    std::vector<int> rect_of(np);
    for (int k = 0; k < np; ++k) { rect_of[k] = (int)P.rects.size(); merge_prog(P, part[k], k); }
    upload_prog(P);
    // virtual patches: k the coarsened values, np+k the regular step; buffers in one block
    std::vector<PatchDev> vp(2 * (size_t)np);
    std::vector<long long> vo(2 * (size_t)np + 1, 0);
    for (int k = 0; k < np; ++k) {
      const HPatch3& g = node[G[k]];
      const long long n2 = (long long)(g.nx() / 2 + 2 * G3) * (g.ny() / 2 + 2 * G3) * (g.nz() / 2 + 2 * G3);
      vo[k + 1] = vo[k] + 2 * Arena::rnd(nvar * n2);
    }
    for (int k = 0; k < np; ++k) vo[np + k + 1] = vo[np + k] + Arena::rnd((long long)nvar * mitot(G[k]) * mjtot(G[k]) * mktot(G[k]));
    rich_len = std::max<long long>(vo[2 * np], 1);
    rich_buf = palloc(rich_len);
    for (int k = 0; k < np; ++k) {
      const HPatch3& g = node[G[k]];
      PatchDev B{};
      const int nx2 = g.nx() / 2, ny2 = g.ny() / 2, nz2 = g.nz() / 2;
      B.mitot = nx2 + 2 * G3; B.mjtot = ny2 + 2 * G3; B.mktot = nz2 + 2 * G3;
      B.q[0] = rich_buf + vo[k]; B.q[1] = B.q[0] + Arena::rnd((long long)nvar * B.mitot * B.mjtot * B.mktot);
      B.cur = 0; B.ilo = 0; B.ihi = nx2 - 1; B.jlo = 0; B.jhi = ny2 - 1; B.klo = 0; B.khi = nz2 - 1;
      B.ffl = -1; B.level = lcheck; B.aux = -1;
      vp[k] = B;
      PatchDev R{};
      R.q[0] = g.cur == 0 ? g.q0 : g.q1; R.q[1] = rich_buf + vo[np + k];
      R.cur = 0; R.ilo = g.ilo; R.ihi = g.ihi; R.jlo = g.jlo; R.jhi = g.jhi; R.klo = g.klo; R.khi = g.khi;
      R.mitot = mitot(G[k]); R.mjtot = mjtot(G[k]); R.mktot = mktot(G[k]);
      R.ffl = -1; R.level = lcheck; R.aux = -1;
      vp[np + k] = R;
    }
    // step prefixes of both lists, as compile_step builds them for a level:
    // [sweep0 3*(n+1) | comp0 3*(n+1) | face0 n+1 | cell0 n+1] per list
    std::vector<long long> pre;
    long long items[2][3], slots[2], faces[2], cells[2], base[2];
    for (int li = 0; li < 2; ++li) {
      base[li] = (long long)pre.size();
      const int n = np, first = li * np;
      std::vector<long long> sw(3 * (size_t)(n + 1), 0), cp(3 * (size_t)(n + 1), 0), fc(n + 1, 0), ce(n + 1, 0);
      long long slot = 0;
      for (int d = 0; d < 3; ++d) {
        long long comp = 0;
        for (int k = 0; k < n; ++k) {
          const PatchDev& V = vp[first + k];
          const long long mx = V.ihi - V.ilo + 1, my = V.jhi - V.jlo + 1, mz = V.khi - V.klo + 1;
          const long long n1 = d == 0 ? mx : d == 1 ? my : mz;
          const long long pencils = d == 0 ? (my + 2) * (mz + 2) : d == 1 ? (mx + 2) * (mz + 2) : (mx + 2) * (my + 2);
          sw[(size_t)d * (n + 1) + k] = slot; cp[(size_t)d * (n + 1) + k] = comp;
          slot += pencils * (n1 + 1);
          comp += pencils * (n1 + 3);
        }
        sw[(size_t)d * (n + 1) + n] = slot; cp[(size_t)d * (n + 1) + n] = comp;
        items[li][d] = comp;
      }
      for (int k = 0; k < n; ++k) {
        const PatchDev& V = vp[first + k];
        const long long mx = V.ihi - V.ilo + 1, my = V.jhi - V.jlo + 1, mz = V.khi - V.klo + 1;
        fc[k + 1] = fc[k] + (mx + 1) * (my + 1) * (mz + 1);
        ce[k + 1] = ce[k] + mx * my * mz;
      }
      slots[li] = slot; faces[li] = fc[n]; cells[li] = ce[n];
      pre.insert(pre.end(), sw.begin(), sw.end());
      pre.insert(pre.end(), cp.begin(), cp.end());
      pre.insert(pre.end(), fc.begin(), fc.end());
      pre.insert(pre.end(), ce.begin(), ce.end());
    }
    std::vector<int> pl(2 * (size_t)np);
    for (int k = 0; k < 2 * np; ++k) pl[k] = k;
    rich_vp.upload(vp, st, stg);
    rich_rect.upload(rect_of, st, stg);
    rich_plist.upload(pl, st, stg);
    rich_pre.upload(pre, st, stg);
    rich_cfl.ensure(1);
    d_stash.reserve(std::max<size_t>(d_stash.n, (size_t)(std::max(slots[0], slots[1]) * stash_values(nvar))));
    d_flux.reserve(std::max<size_t>(d_flux.n, (size_t)(std::max(faces[0], faces[1]) * 6 * nvar)));
    // the ghost ring at tpre, coarsen.f, then the two steps
    run_prog(P, modes_for(lcheck, tpre));
    launch_coarsen3(pool.d, P.d_rects.d, rich_rect.d, rich_vp.d, np, nvar, st, f32);
    nkernels += 1;
    for (int li = 0; li < 2; ++li) {
      if (cells[li] == 0) continue;
      Step3Args a{};
      a.pool = pool.d; a.patches = rich_vp.d; a.sp = sp;
      a.plist = rich_plist.d + li * np; a.np = np;
      const long long* b = rich_pre.d + base[li];
      a.sweep0 = b; a.comp0 = b + 3 * (np + 1); a.face0 = b + 6 * (np + 1); a.cell0 = b + 7 * (np + 1);
      a.stash = d_stash.d; a.stash_stride = slots[li]; a.flux = d_flux.d; a.flux_stride = faces[li];
      a.dt = li == 0 ? 2.0 * dt : dt;
      a.dx = li == 0 ? 2.0 * hx : hx; a.dy = li == 0 ? 2.0 * hy : hy; a.dz = li == 0 ? 2.0 * hz : hz;
      a.cflmax = rich_cfl.d; a.queue = nullptr; a.dt_dev = nullptr;
      nkernels += launch_step3(a, items[li], faces[li], cells[li], st, f32);
    }
    if (p.tol > 0) {
      const double order = (double)((1 << (sp.order + 1)) - 2);
      launch_errf3(pool.d, rich_vp.d, np, order, p.tol, f, dl, st, f32);
      nkernels += 1;
    }
  }
  void richardson_release() {
    pfree(rich_prog.scratch_off, rich_prog.scratch_alloc);
    rich_prog.scratch_off = -1;
    pfree(rich_buf, rich_len);
    rich_buf = -1;
  }

  // flglvl.f:4-85 with domprep.f, domshrink.f, domup.f, domcopy.f, spest.f (+ flag2refine.f,
  // setflags.f), bufnst.f (+ projec.f, shiftset.f) and colate.f. The arrays live in device
  // memory; one read-back returns the flags (for the ordered point list) and the nesting
  // domain (for nestck.f). Returns the flagged cells in (k, j, i) order.
  // flglvl.f on the device: the level's flag array (lv_b) with buffering and nesting
  // applied (colate.f); only the nesting-domain array comes back to the host (nestck.f
  // reads it). The clusters are then found from device signatures (cluster_on_device).
  void flglvl(int lcheck, int lbase, LvlView& dom) {
    PhaseTimer tph(hprof);
    tph.next("flg_device");
    const LvlDims d0{iregsz[lbase], jregsz[lbase], kregsz[lbase]};
    const LvlDims dl{iregsz[lcheck], jregsz[lcheck], kregsz[lcheck]};
    const size_t need = (size_t)dl.size();
    for (DBuf<int8_t>* b : {&lv_a, &lv_b, &lv_n, &lv_t1, &lv_t2}) b->reserve(need);
    std::vector<LvlBox> boxes;
    for (int m = lstart[lbase]; m != 0; m = node[m].levelptr) {
      const HPatch3& g = node[m];
      boxes.push_back(LvlBox{g.ilo + 1, g.ihi + 1, g.jlo + 1, g.jhi + 1, g.klo + 1, g.khi + 1});
    }
    lv_boxes.upload(boxes, st, stg);
    const int per = (xperdom ? 1 : 0) | (yperdom ? 2 : 0) | (zperdom ? 4 : 0);
    launch_domprep(lv_a.d, d0, lv_boxes.d, (int)boxes.size(), st, per);
    launch_domshrink(lv_a.d, lv_b.d, d0, st, per);
    LvlDims dc = d0;
    for (int lev = lbase + 1; lev <= lcheck; ++lev) {
      const LvlDims df{dc.is * intratx[lev - 1], dc.js * intraty[lev - 1], dc.ks * intratz[lev - 1]};
      launch_domup(lv_b.d, dc, lv_a.d, df, intratx[lev - 1], intraty[lev - 1], intratz[lev - 1], st, per);
      launch_domshrink(lv_a.d, lv_b.d, df, st, per);
      dc = df;
    }
    // domcopy.f: the nesting domain keeps the shrunk array (its ring extended again: without
    // periodic directions that changes nothing); the shrunk array itself becomes the flag array
    AMR_CUDA(cudaMemcpyAsync(lv_n.d, lv_b.d, need, cudaMemcpyDeviceToDevice, st));
    if (per) launch_domcopy_borders(lv_n.d, dl, st, per);
    launch_zero_interior(lv_b.d, dl, st);
    // spest.f fills the ghost cells of every grid whether or not it flags by gradient:
    // errest.f steps those values
    if (p.flag_gradient || p.flag_richardson) bound_level(lcheck, node[lgrids[lcheck][0]].time);
    if (p.flag_gradient) {
      const std::vector<int>& G = lgrids[lcheck];
      std::vector<long long> c0(G.size() + 1, 0);
      for (size_t k = 0; k < G.size(); ++k) c0[k + 1] = c0[k] + (long long)node[G[k]].nx() * node[G[k]].ny() * node[G[k]].nz();
      lv_c0.upload(c0, st, stg);
      lv_plist.upload(G, st, stg);
      launch_flag_cells3(pool.d, d_patches.d, lv_plist.d, lv_c0.d, (int)G.size(), c0.back(), flag_pressure, sp.gamma1, p.tolsp, nvar,
                         lv_b.d, dl, st, f32);
    }
    if (p.flag_richardson) richardson_launch(lcheck, lgrids[lcheck], lv_b.d, dl);
    std::vector<LvlBox> proj;
    if (lcheck + 2 <= p.mxnest) {
      // projec.f: level lcheck+2's new grids, with one more cell on each side when ibuff = 0
      const int lrx = intratx[lcheck] * intratx[lcheck + 1], lry = intraty[lcheck] * intraty[lcheck + 1], lrz = intratz[lcheck] * intratz[lcheck + 1];
      for (int mk = newstl[lcheck + 2]; mk != 0; mk = node[mk].levelptr) {
        const HPatch3& c = node[mk];
        int ist = c.ilo / lrx, jst = c.jlo / lry, kst = c.klo / lrz;
        int iend = (c.ihi + lrx - 1) / lrx, jend = (c.jhi + lry - 1) / lry, kend = (c.khi + lrz - 1) / lrz;
        if (p.ibuff == 0) {
          if (ist * lrx == c.ilo) ist = ist - 1;
          if (jst * lry == c.jlo) jst = jst - 1;
          if (kst * lrz == c.klo) kst = kst - 1;
          if (iend * lrx == c.ihi + 1) iend = iend + 1;
          if (jend * lry == c.jhi + 1) jend = jend + 1;
          if (kend * lrz == c.khi + 1) kend = kend + 1;
        }
        // kept inside the array (0:is+1, ...); the ring is cleared right after
        proj.push_back(LvlBox{std::max(ist + 1, 0), std::min(iend + 1, dl.is + 1), std::max(jst + 1, 0), std::min(jend + 1, dl.js + 1),
                              std::max(kst + 1, 0), std::min(kend + 1, dl.ks + 1)});
      }
    }
    lv_proj.upload(proj, st, stg);
    launch_bufnst3(lv_b.d, dl, lv_proj.d, (int)proj.size(), p.ibuff, lv_t1.d, lv_t2.d, st);
    launch_colate3(lv_b.d, lv_n.d, dl, st);
    nkernels += 20;
    if (lv_host_cap < need) {
      if (lv_host) AMR_CUDA(cudaFreeHost(lv_host));
      lv_host_cap = need;
      AMR_CUDA(cudaMallocHost((void**)&lv_host, lv_host_cap));
    }
    AMR_CUDA(cudaMemcpyAsync(lv_host, lv_n.d, need, cudaMemcpyDeviceToHost, st));
    lv_dims = dl;
    tph.next("flg_sync");
    sync_stream();
    if (p.flag_richardson) richardson_release();
    dom = LvlView{lv_host, dl};
  }

  // ---------------------------------------------------------------- clustering
  // Berger-Rigoutsos bisection (smartbis.f:25-177, signs.f:4-86, findcut.f:4-198,
  // moment.f:4-70) driven by signatures made on the device: a cluster is a box of the
  // level's flag array, its points the flagged cells inside. Each wave of the bisection
  // sends the boxes of all undecided clusters to the device, which counts the flagged
  // cells per i, per j and per k of every box (launch_signatures3); only those counts come
  // back. From them the host takes the cluster's point count and bounding box (moment.f:
  // the first and last non-zero count per axis), its efficiency, and the cut (findcut.f).
  // A point of the reference is the cell centre (i-.5, j-.5, k-.5); every comparison it
  // makes on centres is the same comparison on the integer indices, and every decision
  // depends only on the counts, so the clusters are the reference's.
  struct Clu3 {
    SigBox box;   // where its points lie (a sub-box of its parent's bounding box)
    int n = 0;    // points
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // bounding box of the points (moment.f)
  };
  DBuf<SigBox> sig_boxes;
  DBuf<int> sig_off, sig_hist;
  LvlDims lv_dims{0, 0, 0};
  // signs.f on the device for the boxes of clus; fills n, lo, hi of each; scr (optional)
  // receives each cluster's counts per axis at their level indices (0..dims+1)
  void signatures(std::vector<Clu3>& clus, std::vector<std::array<std::vector<int>, 3>>* scr) {
    const int nb = (int)clus.size();
    if (nb == 0) return;
    std::vector<SigBox> bx(nb);
    std::vector<int> off(nb + 1, 0);
    int maxlen = 0;
    long long maxvol = 0;
    for (int b = 0; b < nb; ++b) {
      bx[b] = clus[b].box;
      const int len = (bx[b].hi[0] - bx[b].lo[0] + 1) + (bx[b].hi[1] - bx[b].lo[1] + 1) + (bx[b].hi[2] - bx[b].lo[2] + 1);
      off[b + 1] = off[b] + len;
      maxlen = std::max(maxlen, len);
      maxvol = std::max(maxvol, (long long)(bx[b].hi[1] - bx[b].lo[1] + 1) * (bx[b].hi[2] - bx[b].lo[2] + 1));  // i-rows
    }
    sig_boxes.upload(bx, st, stg);
    sig_off.upload(off, st, stg);
    sig_hist.reserve((size_t)off[nb]);
    launch_signatures3(lv_b.d, lv_dims, sig_boxes.d, nb, sig_off.d, off[nb], maxlen, maxvol, sig_hist.d, st);
    ++nkernels;
    std::vector<int> h((size_t)off[nb]);
    AMR_CUDA(cudaMemcpyAsync(h.data(), sig_hist.d, sizeof(int) * h.size(), cudaMemcpyDeviceToHost, st));
    sync_stream();
    const int dims[3] = {lv_dims.is, lv_dims.js, lv_dims.ks};
    if (scr) scr->assign(nb, {});
    for (int b = 0; b < nb; ++b) {
      Clu3& c = clus[b];
      const int* hh = h.data() + off[b];
      c.n = 0;
      for (int d = 0; d < 3; ++d) {
        const int len = c.box.hi[d] - c.box.lo[d] + 1;
        int first = -1, last = -1, sum = 0;
        for (int t = 0; t < len; ++t)
          if (hh[t]) { if (first < 0) first = t; last = t; sum += hh[t]; }
        if (d == 0) c.n = sum;
        c.lo[d] = first < 0 ? c.box.lo[d] : c.box.lo[d] + first;
        c.hi[d] = last < 0 ? c.box.hi[d] : c.box.lo[d] + last;
        if (scr) {
          std::vector<int>& v = (*scr)[b][d];
          v.assign(dims[d] + 2, 0);
          for (int t = 0; t < len; ++t) v[c.box.lo[d] + t] = hh[t];
        }
        hh += len;
      }
    }
  }
  // moment.f:4-70: bounding box (rect: ilo, ihi, jlo, jhi, klo, khi, 0-based) and efficiency
  static void moment(int rect[6], const Clu3& c, double& usage) {
    for (int d = 0; d < 3; ++d) { rect[2 * d] = c.lo[d] - 1; rect[2 * d + 1] = c.hi[d] - 1; }
    const int gpall = (rect[1] - rect[0] + 1) * (rect[3] - rect[2] + 1) * (rect[5] - rect[4] + 1);
    usage = (double)c.n / gpall;
  }
  // findcut.f on a cluster's signatures scr (counts at level indices 0..dims+1): a hole in
  // a signature, else the largest Laplacian sign change (ties to the middle)
  static void findcut(std::array<std::vector<int>, 3>& scr, const int dims[3], int& index, int& iside) {
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = 1; hi[d] = dims[d];
      for (int t = 1; t <= dims[d]; ++t) if (scr[d][t] != 0) { lo[d] = t; break; }
      for (int t = 1; t <= dims[d]; ++t) if (scr[d][dims[d] + 1 - t] != 0) { hi[d] = dims[d] + 1 - t; break; }
    }
    for (int d = 0; d < 3; ++d)
      for (int t = lo[d]; t <= hi[d]; ++t)
        if (scr[d][t] == 0) { index = t; iside = d + 1; return; }
    auto lap = [&](std::vector<int>& sc, int l0, int h0, int& locmax, int& idx, int& mid) {
      int pre = sc[l0];
      for (int t = l0 + 1; t <= h0 - 1; ++t) { const int cur = sc[t]; sc[t] = sc[t + 1] - 2 * cur + pre; pre = cur; }
      locmax = 0; idx = 0; mid = (l0 + h0) / 2;
      for (int t = l0 + 2; t <= h0 - 2 + 1; ++t) {
        const int t1 = sc[t - 1], t2 = sc[t], dd = std::abs(t1 - t2);
        if (t1 * t2 < 0) {
          if (dd > locmax) { locmax = dd; idx = t; }
          else if (dd == locmax && std::abs(t - mid) < std::abs(idx - mid)) idx = t;
        }
      }
    };
    int lv[3][4];
    for (int d = 0; d < 3; ++d) { lap(scr[d], lo[d], hi[d], lv[d][0], lv[d][2], lv[d][3]); lv[d][1] = d + 1; }
    for (int a = 0; a < 2; ++a)
      for (int b = a + 1; b < 3; ++b)
        if (lv[a][0] < lv[b][0]) for (int t = 0; t < 4; ++t) std::swap(lv[a][t], lv[b][t]);
    const int icount = (lv[0][0] > lv[1][0]) ? 1 : (lv[1][0] > lv[2][0]) ? 2 : 3;
    if (icount != 1)
      for (int a = 0; a < icount - 1; ++a)
        for (int b = a + 1; b < icount; ++b)
          if (std::abs(lv[a][2] - lv[a][3]) > std::abs(lv[b][2] - lv[b][3])) for (int t = 0; t < 4; ++t) std::swap(lv[a][t], lv[b][t]);
    index = lv[0][2];
    iside = lv[0][1];
    if (lv[0][0] < 2) index = 0;
  }
  // smartbis.f: bisect until every cluster's efficiency reaches cutoff or it has no cut;
  // breadth first (one signature wave per depth), then the leaves in the reference's
  // depth-first order: the part at or above the cut before the part below it
  std::vector<Clu3> cluster_on_device(double cutoff) {
    const int dims[3] = {lv_dims.is, lv_dims.js, lv_dims.ks};
    struct Node { Clu3 c; int child = -1; };  // child: the upper part; child+1 the lower part
    std::vector<Node> T(1);
    T[0].c.box = SigBox{{1, 1, 1}, {dims[0], dims[1], dims[2]}};
    std::vector<int> wave{0};
    std::vector<std::array<std::vector<int>, 3>> scr;
    while (!wave.empty()) {
      std::vector<Clu3> cl(wave.size());
      for (size_t w = 0; w < wave.size(); ++w) cl[w] = T[wave[w]].c;
      signatures(cl, &scr);
      std::vector<int> next;
      for (size_t w = 0; w < wave.size(); ++w) {
        T[wave[w]].c = cl[w];
        const Clu3& c = cl[w];
        if (c.n == 0) continue;  // only the whole array of a level without flags
        int rect[6];
        double usenew;
        moment(rect, c, usenew);
        int index = 0, iside = 0;
        if (usenew < cutoff) findcut(scr[w], dims, index, iside);
        if (usenew >= cutoff || index == 0) continue;
        const int d = iside - 1;
        Clu3 up, dn;
        up.box = dn.box = SigBox{{c.lo[0], c.lo[1], c.lo[2]}, {c.hi[0], c.hi[1], c.hi[2]}};
        up.box.lo[d] = index;
        dn.box.hi[d] = index - 1;
        const int id = (int)T.size();
        T[wave[w]].child = id;
        T.push_back(Node{up, -1});
        T.push_back(Node{dn, -1});
        next.push_back(id);
        next.push_back(id + 1);
      }
      wave.swap(next);
    }
    std::vector<Clu3> leaves;
    if (T[0].c.n == 0) return leaves;
    std::vector<int> stack{0};
    while (!stack.empty()) {
      const int id = stack.back();
      stack.pop_back();
      if (T[id].child < 0) { leaves.push_back(T[id].c); continue; }
      stack.push_back(T[id].child + 1);  // lower part after
      stack.push_back(T[id].child);      // upper part first
    }
    return leaves;
  }
  // nestck.f: a new grid must lie in the nesting domain of its base; otherwise split its
  // points at the middle of its longest side (points with centre below the middle first)
  // and retry: clus[icl] becomes the lower part and the upper part follows it
  bool nestck(int mnew, int lbase, std::vector<Clu3>& clus, int icl, const LvlView& dom) {
    if (lbase == 1) return true;
    const HPatch3& n = node[mnew];
    const int lev = n.level;
    const int rx = intratx[lev - 1], ry = intraty[lev - 1], rz = intratz[lev - 1];
    bool nested = true;
    for (int k = n.klo / rz + 1; k <= n.khi / rz + 1 && nested; ++k)
      for (int j = n.jlo / ry + 1; j <= n.jhi / ry + 1 && nested; ++j)
        for (int i = n.ilo / rx + 1; i <= n.ihi / rx + 1; ++i)
          if (dom(i, j, k) == 0) { nested = false; break; }
    if (nested) return true;
    if (clus[icl].n <= 1) throw std::runtime_error("nestck: a single point cannot be properly nested");
    double sidemx = std::max(n.xhi - n.xlo, n.yhi - n.ylo);
    sidemx = std::max(sidemx, n.zhi - n.zlo);
    double rmid; int d;
    if (n.xhi - n.xlo >= sidemx) { rmid = (double)(float)((n.ihi + n.ilo + 1) / 2.f); rmid = rmid / rx; d = 0; }
    else if (n.yhi - n.ylo >= sidemx) { rmid = (double)(float)((n.jhi + n.jlo + 1) / 2.f); rmid = rmid / ry; d = 1; }
    else { rmid = (double)(float)((n.khi + n.klo + 1) / 2.f); rmid = rmid / rz; d = 2; }
    // the largest index whose centre lies below rmid
    const Clu3 c = clus[icl];
    int cut = c.lo[d] - 1;
    for (int t = c.lo[d]; t <= c.hi[d]; ++t) if ((double)t - .5 < rmid) cut = t;
    std::vector<Clu3> parts(2);
    parts[0].box = parts[1].box = SigBox{{c.lo[0], c.lo[1], c.lo[2]}, {c.hi[0], c.hi[1], c.hi[2]}};
    parts[0].box.hi[d] = cut;
    parts[1].box.lo[d] = cut + 1;
    signatures(parts, nullptr);
    clus[icl] = parts[0];
    clus.insert(clus.begin() + icl + 1, parts[1]);
    return false;
  }
  // grdfit.f
  void grdfit(int lbase, int lcheck, double t) {
    LvlView i1flags{nullptr, LvlDims{0, 0, 0}};
    {
      HPROF("flglvl3");
      flglvl(lcheck, lbase, i1flags);
    }
    HPROF("cluster3");
    std::vector<Clu3> clus = cluster_on_device(p.cut);
    if (clus.empty()) return;
    const int levnew = lcheck + 1;
    const double hxf = hxposs[levnew], hyf = hyposs[levnew], hzf = hzposs[levnew];
    int prv = 0;
    for (size_t icl = 0; icl < clus.size(); ++icl) {
      const int mnew = nodget();
      while (true) {
        int rect[6]; double usage;
        moment(rect, clus[icl], usage);
        HPatch3& n = node[mnew];
        n.ilo = rect[0] * intratx[lcheck]; n.jlo = rect[2] * intraty[lcheck]; n.klo = rect[4] * intratz[lcheck];
        n.ihi = (rect[1] + 1) * intratx[lcheck] - 1; n.jhi = (rect[3] + 1) * intraty[lcheck] - 1; n.khi = (rect[5] + 1) * intratz[lcheck] - 1;
        n.xlo = n.ilo * hxf + xlower; n.ylo = n.jlo * hyf + ylower; n.zlo = n.klo * hzf + zlower;
        n.xhi = (n.ihi + 1) * hxf + xlower; n.yhi = (n.jhi + 1) * hyf + ylower; n.zhi = (n.khi + 1) * hzf + zlower;
        n.level = levnew; n.time = t;
        if (nestck(mnew, lbase, clus, (int)icl, i1flags)) break;
      }
      if (newstl[levnew] == 0) newstl[levnew] = mnew;
      else node[prv].levelptr = mnew;
      prv = mnew;
    }
    birect(newstl[levnew]);
  }

  // filval.f for the new grids of level lev: coarse box (icall + bc3amr), limited interpolation, copies from the old grids
  void fill_new_patch(Prog3& P, int lev, int m) {
    const HPatch3& g = node[m];
    const int rx = intratx[lev - 1], ry = intraty[lev - 1], rz = intratz[lev - 1];
    const double hxc = hxposs[lev] * rx, hyc = hyposs[lev] * ry, hzc = hzposs[lev] * rz;
    const int iclo = g.ilo / rx - 1, jclo = g.jlo / ry - 1, kclo = g.klo / rz - 1;
    const int ichi = (g.ihi + 1) / rx - 1 + 1, jchi = (g.jhi + 1) / ry - 1 + 1, kchi = (g.khi + 1) / rz - 1 + 1;
    const int mic = g.nx() / rx + 2, mjc = g.ny() / ry + 2, mkc = g.nz() / rz + 2;
    const int R = P.add_rect(mic, mjc, mkc, nvar);
    Tgt3 C{-1, R, mic, mjc, mkc};
    // filval.f:52-58: preintcopy with any periodic direction (the fine copy below is intcopy)
    if (anyper()) c_preicall3(P, C, iclo, ichi, jclo, jchi, kclo, kchi, lev - 1, 0);
    else c_icall(P, C, iclo, ichi, jclo, jchi, kclo, kchi, lev - 1, 1, 1, 1, 0);
    bool any;
    Bc3Op b = make_bc(C, hxc, hyc, hzc, g.xlo - hxc, g.xhi + hxc, g.ylo - hyc, g.yhi + hyc, g.zlo - hzc, g.zhi + hzc, any);
    if (any) P.add_bc(b, 0);
    Fill3Op o{};
    o.kind = F3_FILVAL; o.dst_patch = m; o.dst_rect = -1;
    o.di0 = G3; o.dj0 = G3; o.dk0 = G3; o.ni = g.nx(); o.nj = g.ny(); o.nk = g.nz();
    o.src = R; o.si0 = g.ilo; o.sj0 = g.jlo; o.sk0 = g.klo; o.level = lev; o.cilo = iclo; o.cjlo = jclo; o.cklo = kclo;
    P.add_op(o, 1);
    c_icall(P, Tgt3{m, -1, mitot(m), mjtot(m), mktot(m)}, g.ilo - G3, g.ihi + G3, g.jlo - G3, g.jhi + G3, g.klo - G3, g.khi + G3, lev, 1, 1, 1, 2);
  }
  void fill_new_level(int lev) {
    HPROF("fill_new_level3");
    Prog3& P = newfill;
    P.clear();
    P.zero_scratch = true;
    GI(lev - 1); GI(lev);
    std::vector<int> nl;
    for (int m = newstl[lev]; m != 0; m = node[m].levelptr) nl.push_back(m);
    std::vector<Prog3> part(nl.size());
    pool_host.run((int)nl.size(), [&](int k) { fill_new_patch(part[k], lev, nl[k]); });
    for (auto& q : part) merge_prog(P, q);
    upload_prog(P);
    run_prog(P, SrcMode{});
    sync_stream();
    pfree(P.scratch_off, P.scratch_alloc);
    P.scratch_off = -1;
  }

  // regrid.f:4-118 with gfixup.f
  void regrid(int lbase) {
    HPROF("regrid3");
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
    PhaseTimer tph(hprof);
    tph.next("rg_newlevels");
    for (int lev = lbase; lev <= p.mxnest; ++lev) for (int m : lgrids[lev]) { node[m].has_cfl = false; node[m].listbc.clear(); }
    for (int l2 = lbase + 1; l2 <= p.mxnest; ++l2) {
      std::vector<int> nl;
      tph.next("rg_alloc");
      for (int m = newstl[l2]; m != 0; m = node[m].levelptr) { alloc_patch(m); nl.push_back(m); }
      init_aux(nl);
      // descriptors: current levels (levels below l2 already replaced), the old grids of l2 and the new ones
      tph.next("rg_desc");
      sync_descriptors(&nl, 0);
      tph.next("rg_fill");
      if (newstl[l2] != 0) fill_new_level(l2);
      tph.next("rg_free");
      int m = lstart[l2];
      while (m != 0) {
        const int mold = m;
        m = node[m].levelptr;
        free_patch(mold);
        node[mold].listbc.clear();
        putnod(mold);
      }
      lstart[l2] = newstl[l2];
      touch(l2);
      lgrids[l2].clear();
      for (int q = lstart[l2]; q != 0; q = node[q].levelptr) lgrids[l2].push_back(q);
    }
    lfine = lfnew;
    tph.next("rg_prepf_prepc");
    for (int lev = lbase; lev <= lfine - 1; ++lev) { prepf(lev + 1); prepc(lev); }
    tph.next("rg_arrange_lists");
    for (int lev = lbase + 1; lev <= p.mxnest; ++lev) arrange(lev);
    make_lists();
    tph.next("rg_compile");
    compile_all(lbase);
    sync_stream();
    tph.close();
    t_regrid += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0c).count();
  }

  // ================================================================ init (amr3.f90, domain.f, setgrd.f, ginit.f)
  void ginit(int msave, double t) {
    for (int m = msave; m != 0; m = node[m].levelptr) {
      alloc_patch(m);
      HPatch3& g = node[m];
      g.time = t;
      std::vector<double> q;
      qinit(g, hxposs[g.level], hyposs[g.level], hzposs[g.level], q);
      std::vector<float> qf;
      const void* src = q.data();
      if (f32) {  // the FP32 form stores the initial values rounded to float
        qf.assign(q.begin(), q.end());
        src = qf.data();
      }
      AMR_CUDA(cudaMemcpyAsync(pool_bytes() + elem() * g.q0, src, elem() * q.size(), cudaMemcpyHostToDevice, st));
      AMR_CUDA(cudaMemcpyAsync(pool_bytes() + elem() * g.q1, src, elem() * q.size(), cudaMemcpyHostToDevice, st));
      h2d_bytes += 2.0 * elem() * q.size();
      init_aux({m});
      sync_stream();
    }
  }
  void init(const std::string& dir) {
    p.load(dir);
    if (p.ndim != 3) throw std::runtime_error("num_dim must be 3");
    if (write_output && p.output_format != 1 && p.output_format != 3)
      throw std::runtime_error("output_format must be 1 (ASCII) or 3 (binary): NetCDF and HDF5 output are not supported");
    nvar = p.nvar;
    blast_x = p.pn("x0", 0.0); blast_y = p.pn("y0", 0.0); blast_z = p.pn("z0", 0.0);
    blast_r = p.pn("r0", 0.2); blast_pin = p.pn("pin", 5.0); blast_pout = p.pn("pout", 1.0);
    flag_pressure = p.problem == "euler_blast" ? (int)p.pn("flag_pressure", 1.0) : 0;
    setup_problem();
    xlower = p.lower[0]; ylower = p.lower[1]; zlower = p.lower[2];
    xupper = p.upper[0]; yupper = p.upper[1]; zupper = p.upper[2];
    nxc = p.ncells[0]; nyc = p.ncells[1]; nzc = p.ncells[2];
    if ((nxc / 2) * 2 != nxc || (nyc / 2) * 2 != nyc || (nzc / 2) * 2 != nzc) throw std::runtime_error("cell counts must be even");
    for (int k = 1; k <= 10; ++k) { intratx[k] = p.ratx[k]; intraty[k] = p.raty[k]; intratz[k] = p.ratz[k]; kratio[k] = p.ratt[k]; }
    hxposs[1] = (xupper - xlower) / nxc; hyposs[1] = (yupper - ylower) / nyc; hzposs[1] = (zupper - zlower) / nzc;
    for (int lev = 2; lev <= p.mxnest; ++lev) {
      hxposs[lev] = hxposs[lev - 1] / (double)intratx[lev - 1];
      hyposs[lev] = hyposs[lev - 1] / (double)intraty[lev - 1];
      hzposs[lev] = hzposs[lev - 1] / (double)intratz[lev - 1];
    }
    possk[1] = p.dt_initial;
    iregsz[1] = nxc; jregsz[1] = nyc; kregsz[1] = nzc;
    for (int lev = 2; lev <= p.mxnest; ++lev) {
      iregsz[lev] = iregsz[lev - 1] * intratx[lev - 1];
      jregsz[lev] = jregsz[lev - 1] * intraty[lev - 1];
      kregsz[lev] = kregsz[lev - 1] * intratz[lev - 1];
      possk[lev] = possk[lev - 1] / (double)kratio[lev - 1];
    }
    for (int l = 0; l < MAXLV + 2; ++l) {
      lc.hx[l] = l < 12 ? hxposs[l] : 0; lc.hy[l] = l < 12 ? hyposs[l] : 0; lc.hz[l] = l < 12 ? hzposs[l] : 0;
      lc.iregsz[l] = iregsz[l]; lc.jregsz[l] = jregsz[l]; lc.kregsz[l] = kregsz[l];
      lc.intratx[l] = intratx[l]; lc.intraty[l] = intraty[l]; lc.intratz[l] = intratz[l];
    }
    AMR_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (cudaStream_t& x : sweep_ss.side) AMR_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    AMR_CUDA(cudaEventCreateWithFlags(&sweep_ss.fork, cudaEventDisableTiming));
    for (cudaEvent_t& e : sweep_ss.join) AMR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    retain_pool_memory();
    AllocStreamScope alloc_scope(st);
    for (cudaEvent_t* e : {&ev_a, &ev_b, &ev_run0, &ev_run1}) AMR_CUDA(cudaEventCreate(e));
    // room for the finer levels from the start (16x the level-1 storage): growing the pool
    // later moves it, which waits for the device
    pool.init((long long)nvar * (nxc + 4) * (nyc + 4) * (nzc + 4) * 32 + (1 << 22));
    regs.init(1 << 20);
    AMR_CUDA(cudaMalloc(&d_cfl, sizeof(unsigned long long)));
    AMR_CUDA(cudaMallocHost((void**)&h_cfl, sizeof(unsigned long long)));
    AMR_CUDA(cudaMalloc(&d_mass, sizeof(double)));
    AMR_CUDA(cudaMalloc(&d_sub, sizeof(Substep3) * 12));
    AMR_CUDA(cudaMalloc(&d_queue, sizeof(unsigned int)));
    AMR_CUDA(cudaEventCreate(&ev_t0)); AMR_CUDA(cudaEventCreate(&ev_t1));
    AMR_CUDA(cudaMallocHost((void**)&h_sub, sizeof(Substep3) * 12));
    stg.reserve((size_t)256 << 20);
    {
      // sweep staging and face fluxes: reserved at once for twice a level-1 sweep
      const long long n = (long long)nxc * nyc * nzc;
      d_stash.reserve((size_t)(stash_values(nvar) * 3 * (n + 4LL * (nxc * nyc + nyc * nzc + nxc * nzc))));
      d_flux.reserve((size_t)(6 * nvar * (n + 2LL * (nxc * nyc + nyc * nzc + nxc * nzc) + 8)));
      d_stash.n = d_flux.n = 0;
    }
    node.assign(10001, HPatch3());
    for (int k = 1; k <= 10000; ++k) node[k].nextfree = k + 1;
    node[10000].nextfree = 0;
    ndfree = 1;
    start_time = p.t0;
    glast.assign(p.gauges.size(), 0.0);
    for (size_t i = 0; i < p.gauges.size(); ++i) glast[i] = p.gauges[i].t1;
    if (p.restart) {
      // amr3.f90:466-480: the run continues from the checkpoint named in claw.data
      const std::string f = p.restart_file;
      restart_from(!f.empty() && f[0] == '/' ? f : dir + "/" + f);
      return;
    }
    // domain.f
    const int ms = nodget();
    HPatch3& g = node[ms];
    g.xlo = xlower; g.ylo = ylower; g.zlo = zlower; g.xhi = xupper; g.yhi = yupper; g.zhi = zupper;
    g.level = 1; g.levelptr = 0;
    g.ilo = 0; g.jlo = 0; g.klo = 0; g.ihi = nxc - 1; g.jhi = nyc - 1; g.khi = nzc - 1;
    lstart[1] = ms;
    touch(1);
    lfine = 1;
    birect(ms);
    ginit(lstart[1], start_time);
    arrange(1);
    make_lists();
    compile_all(0);
    // setgrd.f
    record_gauges = false;
    int levnew = 2;
    while (levnew <= p.mxnest) {
      const int levold = levnew - 1;
      if (lstart[levold] == 0) break;
      // setgrd.f:41-53: Richardson estimation needs the level one step ahead before it is
      // flagged; that step is not counted as integration work
      if (p.flag_richardson) {
        advanc(levold);
        rvol = 0;
        for (double& r : rvoll) r = 0;
      }
      for (int i = 1; i <= p.mxnest; ++i) newstl[i] = 0;
      grdfit(levold, levold, start_time);
      if (newstl[levnew] == 0) break;
      ginit(newstl[levnew], start_time);
      lstart[levnew] = newstl[levnew];
      touch(levnew);
      lfine = levnew;
      arrange(levnew);
      make_lists();
      compile_all(levold);
      ++levnew;
    }
    // setgrd.f:110-121 swaps store1/store2 after re-initialising store2. Both hold qinit
    // (both buffers were filled), unless the Richardson steps above advanced the levels:
    // then the swap puts the initial values back in store1, and the times are reset.
    if (p.flag_richardson)
      for (int lev = 1; !(lev == p.mxnest || lev > lfine); ++lev)
        for (int m : lgrids[lev]) { node[m].cur ^= 1; node[m].time = start_time; }
    // update.f runs before prepf/prepc, so no coarse patch has a register list yet (averaging only).
    make_lists();
    compile_all(0);
    for (int level = 1; level <= lfine - 1; ++level) update(lfine - level);
    for (int level = 1; level <= lfine - 1; ++level) { prepf(level + 1); prepc(level); }
    compile_all(0);
    sync_stream();
    record_gauges = true;
    time = start_time;
    tmass0 = mass();
    if (p.output_t0) output(time);
  }

  // ================================================================ check.f / restrt.f
  // A checkpoint, taken at a coarse-step boundary, holds what the continued run reads:
  // the scheduler state (time, cycle, step sizes, regrid counters, level times, output and
  // gauge cursors), the grid table with its free list (grid numbers continue as they
  // would have), both solution buffers and the aux block of every grid, and the gauge
  // samples so far. The fill programs, step plans and register lists are compiled again
  // from the grids. The flux registers and saved coarse rings are not kept: at a
  // coarse-step boundary each entry upbnd will read is rewritten (fluxsv, saveqc, prepf)
  // before it is read. The layout is this library's own (little-endian, versioned); the
  // reference dumps its raw alloc array instead.
  static constexpr char CHK_MAGIC[8] = {'A', 'M', 'R', 'B', '3', 'C', 'K', '1'};
  struct ChkHead {
    int nvar, naux, f32, mxnest, lfine, ncycle, frame, nextout, nnodes, ndfree, id_hwm, gslots, ngrows, ngauges;
    int icheck[12], lstart[12];
    double time, start_time, tmass0, cflmax_run, rvol, rvoll[12], possk[12], tlevel[12];
  };
  struct ChkNode {
    int ilo, ihi, jlo, jhi, klo, khi, level, levelptr, nextfree;
    double xlo, xhi, ylo, yhi, zlo, zhi, time;
  };
  void checkpoint(const std::string& path) {
    HPROF("checkpoint3");
    sync_stream();
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write checkpoint " + path);
    auto put = [&](const void* d, size_t n) {
      if (n && std::fwrite(d, 1, n, f) != n) { std::fclose(f); throw std::runtime_error("short write to " + path); }
    };
    ChkHead h{};
    h.nvar = nvar; h.naux = p.naux; h.f32 = f32 ? 1 : 0; h.mxnest = p.mxnest; h.lfine = lfine; h.ncycle = ncycle;
    h.frame = frame; h.nextout = tk_nextout; h.nnodes = (int)node.size(); h.ndfree = ndfree; h.id_hwm = id_hwm;
    h.gslots = gslots; h.ngrows = (int)grows.size(); h.ngauges = (int)glast.size();
    for (int l = 0; l < 12; ++l) {
      h.icheck[l] = icheck[l]; h.lstart[l] = lstart[l]; h.rvoll[l] = rvoll[l]; h.possk[l] = possk[l];
      h.tlevel[l] = tk_tlevel[l];
    }
    h.time = time; h.start_time = start_time; h.tmass0 = tmass0; h.cflmax_run = cflmax_run; h.rvol = rvol;
    if (!tick_started) for (int l = 1; l <= p.mxnest; ++l) h.tlevel[l] = time;
    put(CHK_MAGIC, 8);
    put(&h, sizeof h);
    std::vector<ChkNode> nodes(node.size());
    for (size_t m = 0; m < node.size(); ++m) {
      const HPatch3& g = node[m];
      nodes[m] = ChkNode{g.ilo, g.ihi, g.jlo, g.jhi, g.klo, g.khi, g.level, g.levelptr, g.nextfree,
                         g.xlo, g.xhi, g.ylo, g.yhi, g.zlo, g.zhi, g.time};
    }
    put(nodes.data(), sizeof(ChkNode) * nodes.size());
    // per grid, level by level in list order: store1, store2, aux block (storage precision)
    std::vector<char> buf;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
        const HPatch3& g = node[m];
        const long long offs[2] = {g.cur == 0 ? g.q0 : g.q1, g.cur == 0 ? g.q1 : g.q0};
        for (long long off : offs) {
          buf.resize(elem() * g.nq);
          AMR_CUDA(cudaMemcpy(buf.data(), pool_bytes() + elem() * off, buf.size(), cudaMemcpyDeviceToHost));
          put(buf.data(), buf.size());
        }
        if (g.aux >= 0) {
          buf.resize(elem() * g.na * (vel_period > 0.0 ? 2 : 1));
          AMR_CUDA(cudaMemcpy(buf.data(), pool_bytes() + elem() * g.aux, buf.size(), cudaMemcpyDeviceToHost));
          put(buf.data(), buf.size());
        }
      }
    put(glast.data(), sizeof(double) * glast.size());
    put(grows.data(), sizeof(GRow) * grows.size());
    if (gslots) {
      std::vector<double> gv((size_t)gslots * nvar);
      AMR_CUDA(cudaMemcpy(gv.data(), d_gauge_out.d, sizeof(double) * gv.size(), cudaMemcpyDeviceToHost));
      put(gv.data(), sizeof(double) * gv.size());
    }
    if (std::fclose(f) != 0) throw std::runtime_error("cannot close " + path);
  }
  // restrt.f: the grids and scheduler state of a checkpoint, in place of domain.f/setgrd.f
  void restart_from(const std::string& path) {
    HPROF("restart3");
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot read checkpoint " + path);
    auto get = [&](void* d, size_t n) {
      if (n && std::fread(d, 1, n, f) != n) { std::fclose(f); throw std::runtime_error("checkpoint " + path + " is truncated"); }
    };
    char magic[8];
    get(magic, 8);
    if (std::memcmp(magic, CHK_MAGIC, 8) != 0) { std::fclose(f); throw std::runtime_error(path + " is not a 3D checkpoint of this library"); }
    ChkHead h{};
    get(&h, sizeof h);
    if (h.nvar != nvar || h.naux != p.naux || h.f32 != (f32 ? 1 : 0) || h.mxnest != p.mxnest || h.ngauges != (int)glast.size() ||
        h.nnodes < 2 || h.lfine < 1 || h.lfine > p.mxnest) {
      std::fclose(f);
      throw std::runtime_error("checkpoint " + path + " does not match this run (equations, aux, precision, levels or gauges)");
    }
    std::vector<ChkNode> nodes((size_t)h.nnodes);
    get(nodes.data(), sizeof(ChkNode) * nodes.size());
    node.assign(nodes.size(), HPatch3());
    for (size_t m = 0; m < nodes.size(); ++m) {
      const ChkNode& c = nodes[m];
      HPatch3& g = node[m];
      g.ilo = c.ilo; g.ihi = c.ihi; g.jlo = c.jlo; g.jhi = c.jhi; g.klo = c.klo; g.khi = c.khi;
      g.level = c.level; g.levelptr = c.levelptr; g.nextfree = c.nextfree;
      g.xlo = c.xlo; g.xhi = c.xhi; g.ylo = c.ylo; g.yhi = c.yhi; g.zlo = c.zlo; g.zhi = c.zhi; g.time = c.time;
    }
    ndfree = h.ndfree; id_hwm = 0; lfine = h.lfine;
    for (int l = 0; l < 12; ++l) {
      icheck[l] = h.icheck[l]; lstart[l] = h.lstart[l]; rvoll[l] = h.rvoll[l]; possk[l] = h.possk[l]; tk_tlevel[l] = h.tlevel[l];
    }
    ncycle = h.ncycle; frame = h.frame; tk_nextout = h.nextout; tick_started = true;
    time = h.time; start_time = h.start_time; tmass0 = h.tmass0; cflmax_run = h.cflmax_run; rvol = h.rvol;
    std::vector<char> buf;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) {
        alloc_patch(m);  // cur = 0: q0 takes store1, q1 store2
        HPatch3& g = node[m];
        for (long long off : {g.q0, g.q1}) {
          buf.resize(elem() * g.nq);
          get(buf.data(), buf.size());
          AMR_CUDA(cudaMemcpy(pool_bytes() + elem() * off, buf.data(), buf.size(), cudaMemcpyHostToDevice));
        }
        if (g.aux >= 0) {
          buf.resize(elem() * g.na * (vel_period > 0.0 ? 2 : 1));
          get(buf.data(), buf.size());
          AMR_CUDA(cudaMemcpy(pool_bytes() + elem() * g.aux, buf.data(), buf.size(), cudaMemcpyHostToDevice));
        }
        h2d_bytes += 2.0 * elem() * g.nq;
      }
    get(glast.data(), sizeof(double) * glast.size());
    grows.resize((size_t)h.ngrows);
    get(grows.data(), sizeof(GRow) * grows.size());
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
    for (int level = 1; level <= lfine - 1; ++level) { prepf(level + 1); prepc(level); }
    compile_all(0);
    sync_stream();
    record_gauges = true;
    stepped = true;
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
  void write_checkpoint(const char* path) override { checkpoint_file(path); }

  // ================================================================ tick.f
  bool finished() const { return ncycle >= p.nstop || time >= p.tfinal; }
  void tick() {
    double dtnew[12];
    int ntogo[12];
    int cycles = 0;
    run_cells = 0;
    const double rvol0 = rvol;
    const auto tw0 = std::chrono::steady_clock::now();
    AMR_CUDA(cudaEventRecord(ev_run0, st));
    setbestsrc();
    int nextout = 0, iout = p.iout;
    if (iout == 0) { iout = 999999999; nextout = (p.nout > 0) ? 1 : 0; }
    if (tick_started) nextout = tk_nextout;
    double* tlevel = tk_tlevel;
    if (!tick_started) { tlevel[1] = time; for (int i = 2; i <= p.mxnest; ++i) tlevel[i] = tlevel[1]; }
    if (!tick_started || tk_nextchk == 0) {
      // tick.f:73-81: checkpoint times still to come
      tk_nextchk = 1;
      while (tk_nextchk <= (int)p.tchk.size() && p.tchk[tk_nextchk - 1] <= time) ++tk_nextchk;
    }
    tick_started = true;
    while (!finished()) {
      double outtime;
      if (p.nout > 0) outtime = (nextout <= p.nout) ? p.tout[nextout - 1] : RINF;
      else outtime = p.tfinal;
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
      ++cycles;
      if (max_cycles > 0 && cycles >= max_cycles) break;
    }
    tk_nextout = nextout;
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
    t_step += std::chrono::duration<double>(std::chrono::steady_clock::now() - tw0).count();
  }

  // ================================================================ results
  double mass() {
    ensure(1, NEED_STEP);  // the level's patch list on the device
    AMR_CUDA(cudaMemsetAsync(d_mass, 0, sizeof(double), st));
    launch_mass3(pool.d, d_patches.d, plan[1].d_plist.d, (int)plan[1].plist.size(), d_mass, st, f32);
    double m = 0;
    AMR_CUDA(cudaMemcpyAsync(&m, d_mass, sizeof(double), cudaMemcpyDeviceToHost, st));
    sync_stream();
    return m * hxposs[1] * hyposs[1] * hzposs[1];
  }
  // interior values of every grid in output order, [m][k][j][i] per grid: the solution, or
  // with aux set the aux arrays (naux components)
  long long count_values(bool aux = false) const {
    long long n = 0;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) n += (long long)node[m].nx() * node[m].ny() * node[m].nz();
    return n * (aux ? p.naux : nvar);
  }
  // gather_values into out (room for count_values(aux) doubles), copied there from the device
  void gather_into(double* out, bool aux = false) {
    const int nc = aux ? p.naux : nvar;
    std::vector<int> pl;
    std::vector<long long> c0(1, 0);
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) { pl.push_back(m); c0.push_back(c0.back() + (long long)node[m].nx() * node[m].ny() * node[m].nz()); }
    const long long total = c0.back() * nc;
    if (total == 0) return;
    DBuf<int> dp; dp.upload(pl, st, stg);
    DBuf<long long> dc; dc.upload(c0, st, stg);
    DBuf<double> dout; dout.ensure(total);
    launch_gather3(pool.d, d_patches.d, dp.d, dc.d, (int)pl.size(), nc, c0.back(), dout.d, st, f32, aux);
    AMR_CUDA(cudaMemcpyAsync(out, dout.d, sizeof(double) * total, cudaMemcpyDeviceToHost, st));
    sync_stream();
    dp.free(); dc.free(); dout.free();
  }
  std::vector<double> gather_values(bool aux = false) {
    std::vector<double> out((size_t)count_values(aux));
    if (!out.empty()) gather_into(out.data(), aux);
    return out;
  }
  // the rows of fort.q / fort.a (src/3d/valout.f90:140-160): per grid in output order, its
  // header, then k-planes of j-rows of i-cells, one line of nc e26.16 values per cell, a
  // blank line after every j-row, every k-plane and every grid
  void write_frame_file(FILE* f, const std::vector<double>& v, int nc) {
    size_t off = 0;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) {
        const HPatch3& g = node[m];
        const int n3[3] = {g.nx(), g.ny(), g.nz()};
        const double lo[3] = {g.xlo, g.ylo, g.zlo}, h[3] = {hxposs[lev], hyposs[lev], hzposs[lev]};
        write_grid_header(f, 3, m, lev, n3, lo, h);
        const size_t n = (size_t)g.nx() * g.ny() * g.nz();
        for (int k = 0; k < g.nz(); ++k) {
          for (int j = 0; j < g.ny(); ++j) {
            for (int i = 0; i < g.nx(); ++i) {
              for (int iv = 0; iv < nc; ++iv) std::fputs(fort_e(v[off + iv * n + ((size_t)k * g.ny() + j) * g.nx() + i], 26, 16).c_str(), f);
              std::fputc('\n', f);
            }
            std::fputs("  \n", f);
          }
          std::fputs("  \n", f);
        }
        std::fputs("  \n", f);
        off += n * nc;
      }
  }
  // valout.f90: |q| < 1e-90 (and |aux| < 1e-90 when aux is written) become 0 in place on the
  // interior cells, with or without files
  // whole arrays (ghost cells included) of every grid in output order, q(m,i,j,k) with m
  // fastest as raw doubles: binary output (valout.f90:161-172)
  std::vector<double> gather_enlarged(bool aux) {
    const int nc = aux ? p.naux : nvar;
    std::vector<int> pl;
    std::vector<long long> c0(1, 0);
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) { pl.push_back(m); c0.push_back(c0.back() + (long long)mitot(m) * mjtot(m) * mktot(m)); }
    std::vector<double> out((size_t)c0.back() * nc);
    if (out.empty()) return out;
    DBuf<int> dp; dp.upload(pl, st, stg);
    DBuf<long long> dc; dc.upload(c0, st, stg);
    DBuf<double> dout; dout.ensure(out.size());
    launch_gather_enlarged3(pool.d, d_patches.d, dp.d, dc.d, (int)pl.size(), nc, c0.back(), dout.d, aux, stepped ? p.dimsplit : 0, st, f32);
    AMR_CUDA(cudaMemcpyAsync(out.data(), dout.d, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, st));
    sync_stream();
    dp.free(); dc.free(); dout.free();
    return out;
  }
  bool stepped = false;  // a level substep has run (store2 then holds the last step's input)
  void output(double t) {
    const bool aux = p.out_aux(t);
    const bool binary = p.output_format == 3;
    for (int lev = 1; lev <= lfine; ++lev) {
      ensure(lev, NEED_STEP);
      if (binary) continue;  // the binary form zeroes nothing
      launch_zero_tiny3(pool.d, d_patches.d, plan[lev].d_plist.d, (int)plan[lev].plist.size(), nvar, st, f32);
      ++nkernels;
      if (aux) {
        launch_zero_tiny3(pool.d, d_patches.d, plan[lev].d_plist.d, (int)plan[lev].plist.size(), p.naux, st, f32, true);
        ++nkernels;
      }
    }
    if (!write_output) { ++frame; return; }
    int ngrids = 0;
    for (int lev = 1; lev <= lfine; ++lev) ngrids += (int)lgrids[lev].size();
    if (binary) {
      FILE* f = open_output(outdir, "fort.q", frame);
      for (int lev = 1; lev <= lfine; ++lev)
        for (int m : lgrids[lev]) {
          const HPatch3& g = node[m];
          const int n3[3] = {g.nx(), g.ny(), g.nz()};
          const double lo[3] = {g.xlo, g.ylo, g.zlo}, h[3] = {hxposs[lev], hyposs[lev], hzposs[lev]};
          write_grid_header(f, 3, m, lev, n3, lo, h);
        }
      if (std::fclose(f) != 0) throw std::runtime_error("cannot close fort.q in " + outdir);
      write_raw(open_output(outdir, "fort.b", frame, "wb"), gather_enlarged(false), outdir);
      if (aux) write_raw(open_output(outdir, "fort.a", frame, "wb"), gather_enlarged(true), outdir);
      write_fort_t(outdir, frame, t, nvar, ngrids, p.naux, 3, G3);
      ++frame;
      return;
    }
    FILE* f = open_output(outdir, "fort.q", frame);
    write_frame_file(f, gather_values(), nvar);
    if (std::fclose(f) != 0) throw std::runtime_error("cannot close fort.q in " + outdir);
    if (aux) {
      f = open_output(outdir, "fort.a", frame);
      write_frame_file(f, gather_values(true), p.naux);
      if (std::fclose(f) != 0) throw std::runtime_error("cannot close fort.a in " + outdir);
    }
    write_fort_t(outdir, frame, t, nvar, ngrids, p.naux, 3, G3);
    ++frame;
  }

  // amrgpu_set_solver: rpn3/rpt3/rptt3 plugin by name with its /cparam/ constants.
  //   euler_roe_efix  [gamma] or [gamma, efix]  (/cparam/ gamma,gamma1 of the 3D Euler examples)
  //   vc_advection    []  (face velocities come from aux 1..3; examples/advection_3d_swirl)
  // No constants keep the current ones. The run's equations and aux must match.
  void set_solver(const std::string& name, const std::vector<double>& v) override {
    if (name == "euler_roe_efix") {
      if (sp.solver != SOLVER3_EULER) throw std::invalid_argument("euler_roe_efix does not solve this run's equations");
      if (!v.empty() && v.size() != 1 && v.size() != 2) throw std::invalid_argument("euler_roe_efix: wrong number of constants");
      if (!v.empty()) {
        if (!(v[0] > 1.0)) throw std::invalid_argument("euler_roe_efix: gamma must exceed 1");
        sp.gamma = v[0]; sp.gamma1 = sp.gamma - 1.0;
        if (v.size() == 2) sp.efix = v[1] != 0.0 ? 1 : 0;
      }
    } else if (name == "vc_advection") {
      if (sp.solver != SOLVER3_SWIRL) throw std::invalid_argument("vc_advection does not solve this run's equations");
      if (!v.empty()) throw std::invalid_argument("vc_advection takes no constants (velocities are aux arrays)");
    } else {
      throw std::invalid_argument("unknown 3D Riemann solver '" + name + "' (euler_roe_efix, vc_advection)");
    }
    for (auto& G : lgraph) G.reset();  // captured launches hold the old constants
  }

  // ================================================================ AmrSolver
  int num_dim() const override { return 3; }
  cudaStream_t stream() const override { return st; }
  void set_batched(bool on) override { batched = on; }
  void set_profile(bool on) override { profile = on; }
  void set_graphs(bool on) override {
    use_graphs = on;
    if (!on) for (auto& G : lgraph) G.reset();
  }
  void set_schedule(int s) override {
    if (s < 0 || s > 2) throw std::runtime_error("amrgpu_set_schedule: 0 (autotune), 1 (per direction) or 2 (work queue)");
    schedule = s;
    for (auto& T : tune) T = Tune();
    for (auto& G : lgraph) G.reset();
  }
  void set_pool_limit(long long bytes) override { set_arena_limits(pool, regs, bytes); }
  void set_step_batching(int window_us) override {
    if (window_us != 0) throw std::invalid_argument("amrgpu_set_step_batching: cross-request batching is built for the 2D path");
  }
  void run(int mc) override { max_cycles = mc; tick(); }
  double level_advance(int level, double* cfl) override {
    if (level < 1 || level > lfine) throw std::runtime_error("level out of range");
    const double d = advanc(level);
    if (cfl) *cfl = cfl_level;
    return d;
  }
  void update_level(int level) override {
    if (level < 1 || level >= lfine) throw std::runtime_error("level out of range");
    update(level);
    sync_stream();
  }
  void regrid_from(int lbase) override {
    if (lbase < 1 || lbase > lfine || lbase >= p.mxnest) throw std::runtime_error("lbase out of range");
    regrid(lbase);
    setbestsrc();
  }
  void valout(const char* dir) override {
    const std::string keep = outdir;
    const bool kw = write_output;
    if (dir) { outdir = dir; write_output = true; }
    output(time);
    outdir = keep; write_output = kw;
  }
  double mass_() { return mass(); }
  std::vector<double> info() override {
    return {time, rvol, (double)ncycle, (double)lfine, t_step, t_regrid, tmass0, cflmax_run, (double)nkernels, (double)pool.peak * 8.0,
            (double)nsteps_launched, step_kernel_ms, step_kernel_cells, last_run_ms, run_cells, finished() ? 1.0 : 0.0, h2d_bytes,
            0, 0, 0, 0, 0, 0, 3.0, f32 ? 32.0 : 64.0, (double)graph_captures, (double)graph_replays,
            (double)tune_choices(1), (double)tune_choices(0), 8.0 * (double)(pool.cap + regs.cap)};
  }
  std::vector<int> grid_rows() override {
    std::vector<int> r;
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m : lgrids[lev]) {
        const HPatch3& g = node[m];
        r.insert(r.end(), {m, lev, g.ilo, g.ihi, g.jlo, g.jhi, g.klo, g.khi});
      }
    return r;
  }
  std::vector<double> values() override { return gather_values(); }
  long long value_count() override { return count_values(); }
  void values_into(double* out) override { gather_into(out); }
  std::vector<double> gauge_rows() override {
    std::vector<double> vals((size_t)gslots * nvar), out;
    if (gslots) AMR_CUDA(cudaMemcpy(vals.data(), d_gauge_out.d, sizeof(double) * vals.size(), cudaMemcpyDeviceToHost));
    for (const auto& G : p.gauges)
      for (const auto& r : grows) {
        if (r.gauge != G.num) continue;
        out.push_back(r.gauge); out.push_back(r.level); out.push_back(r.t);
        for (int k = 0; k < nvar; ++k) out.push_back(vals[(size_t)r.slot * nvar + k]);
      }
    return out;
  }
};

// quick_sort1.f (qsorti): non-stable index sort with the reference's comparison sequence (1-based views)
void Amr3Gpu::qsorti(std::vector<int>& ord, int n, const std::vector<long long>& a) {
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

AmrSolver* make_solver3(const std::string& rundir, const std::string& outdir, bool write_output, bool f32) {
  std::unique_ptr<Amr3Gpu> s(new Amr3Gpu());
  s->f32 = f32;
  s->outdir = outdir;
  s->write_output = write_output;
  s->init(rundir);
  return s.release();
}

}  // namespace amrb
