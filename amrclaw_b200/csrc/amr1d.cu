// The 1D AMR solve on the device: AMRClaw's src/1d path (amr1.f90, tick.f, advanc.f,
// stepgrid.f/step1.f90/flux1.f, bound.f90/filpatch.f90/intfil.f90/prefilp.f90,
// bc1amr.f90, saveqc.f/cstore.f, qad.f, fluxsv.f, fluxad.f, update.f/upbnd.f, the
// regridding routines and the gauges), with every grid's solution in a device pool.
//
// The grids of a 1D hierarchy are short (at most max1d = 500 cells with ghosts), so each
// array operation on grid data is a small kernel: the patch step is one block per grid
// (one thread per interface: Riemann solve, limiter on the unlimited neighbour waves,
// second-order correction, update, Courant number), ghost fills are copy, interpolation
// and boundary kernels scheduled by the host in the reference's recursive order, and the
// coarse/fine registers are filled and applied by kernels. The host keeps the grid table,
// clustering and scheduling (a few hundred cells per level), which run in microseconds.
//
// Layout: per grid two solution stores [nvar][mitot] (SoA, i fastest) in the pool; flux
// registers (svdflx(nvar,2) then qc1d(nvar,2)) in a register pool.
#include "common.cuh"
#include "hostutil.hpp"
#include "params.hpp"
#include "riemann1d.cuh"
#include "solver.hpp"
#include "valout.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace amrb {

namespace {

constexpr double UNSET1 = -1.0, DONTFLAG1 = 0.0, DOFLAG1 = 2.0, BADPRO1 = 3.0;
const double NEEDS_TO_BE_SET1 = (double)10.e33f;  // default-real literal of amr_module.f90
const double RINFINITY1 = (double)10.e32f;
constexpr int IINFINITY1 = 999999999;
constexpr int STEP1_THREADS = 512;  // one thread per interface; max1d = 500 cells with ghosts

// ------------------------------------------------------------------ kernels
// q(m, i) of a grid store at pool offset off with mitot cells: pool[off + m*mitot + i-1]
__device__ __forceinline__ double& QD(double* pool, long long off, int mitot, int m, int i) {
  return pool[off + (long long)m * mitot + (i - 1)];
}

// intfil.f90: cells [0, n) from a source grid's stores (1-based index si0 + k) into the
// destination (1-based index di0 + k): mode 1 store1, 2 store2, 3 alphai*new + alphac*old
__global__ void copy1_kernel(double* pool, long long dst, int dmitot, int di0, long long snew, long long sold, int smitot, int si0,
                             int n, int nvar, int mode, double ai, double ac) {
  const int k = threadIdx.x + blockIdx.x * blockDim.x;
  if (k >= n) return;
  for (int m = 0; m < nvar; ++m) {
    double v;
    if (mode == 1) v = QD(pool, snew, smitot, m, si0 + k);
    else if (mode == 2) v = QD(pool, sold, smitot, m, si0 + k);
    else v = QD(pool, snew, smitot, m, si0 + k) * ai + QD(pool, sold, smitot, m, si0 + k) * ac;
    QD(pool, dst, dmitot, m, di0 + k) = v;
  }
}

// filpatch.f90:154-190: limited interpolation of up to 8 unset fine cells from the coarse
// patch valcrse (ccells cells); cell k goes to row dst_i[k] from coarse cell ic[k] with eta[k]
struct Interp1 { int n; int dst_i[8]; int ic[8]; double eta[8]; };
__global__ void interp1_kernel(double* pool, long long dst, int dmitot, long long crse, int ccells, Interp1 op, int nvar) {
  const int k = threadIdx.x;
  if (k >= op.n) return;
  const int ic = op.ic[k];
  for (int m = 0; m < nvar; ++m) {
    const double valp = QD(pool, crse, ccells, m, ic + 1), valm = QD(pool, crse, ccells, m, ic - 1), valc = QD(pool, crse, ccells, m, ic);
    const double dupc = valp - valc, dumc = valc - valm, ducc = valp - valm;
    double du = (fabs(dumc) < fabs(dupc)) ? fabs(dumc) : fabs(dupc);  // std::min
    du = (0.5 * fabs(ducc) < 2.0 * du) ? 0.5 * fabs(ducc) : 2.0 * du;
    const double sgn = (dupc * dumc) >= 0.0 ? 1.0 : -1.0;
    const double fu = (0.0 < sgn) ? sgn : 0.0;
    const double uslope = du * ((ducc >= 0.0) ? 1.0 : -1.0) * fu;
    QD(pool, dst, dmitot, m, op.dst_i[k]) = valc + op.eta[k] * uslope;
  }
}

// bc1amr.f90: nxl ghost cells on the left, cells ibeg..nrow on the right (0: none);
// codes 1 extrapolation, 3 wall (negates component 2)
__global__ void bc1_kernel(double* pool, long long off, int nrow, int nvar, int nxl, int codel, int ibeg, int coder) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (nxl > 0 && (codel == 1 || codel == 3)) {
    for (int i = 1; i <= nxl; ++i)
      for (int m = 0; m < nvar; ++m) QD(pool, off, nrow, m, i) = QD(pool, off, nrow, m, codel == 1 ? nxl + 1 : 2 * nxl + 1 - i);
    if (codel == 3) for (int i = 1; i <= nxl; ++i) QD(pool, off, nrow, 1, i) = -QD(pool, off, nrow, 1, i);
  }
  if (ibeg > 0 && (coder == 1 || coder == 3)) {
    for (int i = ibeg; i <= nrow; ++i)
      for (int m = 0; m < nvar; ++m) QD(pool, off, nrow, m, i) = QD(pool, off, nrow, m, coder == 1 ? ibeg - 1 : 2 * ibeg - 1 - i);
    if (coder == 3) for (int i = ibeg; i <= nrow; ++i) QD(pool, off, nrow, 1, i) = -QD(pool, off, nrow, 1, i);
  }
}

// The patch step of one grid (stepgrid.f, step1.f90, flux1.f, inlinelimiter.f): thread t
// takes step1 interface i = t + 2 - mbc (cells i-1 | i); waves go to shared memory so the
// limiter reads the unlimited neighbour waves; fm/fp of interfaces 1..mx+1 are written to
// the grid's flux arrays (enlarged index i + mbc), the interior is updated in place and
// the Courant number goes to *cflmax
struct Step1Args {
  long long q, fm, fp;
  int mitot, nvar, mwaves, order;
  int mthlim[MAXW1];
  double dt, dx;
  Prob1 P;
};
__device__ __forceinline__ double philim1(double a, double b, int meth) {
  const double r = b / a;
  auto mx = [](double x, double y) { return (x < y) ? y : x; };
  auto mn = [](double x, double y) { return (y < x) ? y : x; };
  switch (meth) {
    case 2: return mx(0.0, mx(mn(1.0, 2.0 * r), mn(2.0, r)));
    case 3: return (r + fabs(r)) / (1.0 + fabs(r));
    case 4: { const double c = (1.0 + r) / 2.0; return mx(0.0, mn(c, mn(2.0, 2.0 * r))); }
    case 5: return r;
  }
  return mx(0.0, mn(1.0, r));
}
__global__ void __launch_bounds__(STEP1_THREADS) step1_kernel(double* pool, Step1Args a, unsigned long long* cflmax) {
  __shared__ double sw[STEP1_THREADS + 2][MAXW1][MAXW1];
  __shared__ double sred[STEP1_THREADS / 32];
  const int mbc = 2, mitot = a.mitot, mx = mitot - 2 * mbc, nvar = a.nvar, mwaves = a.mwaves;
  const int t = threadIdx.x;
  const int i = t + 2 - mbc;  // step1 interface index, 2-mbc .. mx+mbc
  const bool valid = i <= mx + mbc;
  double W[MAXW1][MAXW1], S[MAXW1], AM[MAXW1], AP[MAXW1];
  const double dtdx = a.dt / a.dx;
  if (valid) {
    double ql[MAXW1], qr[MAXW1];
    // step1 index i is enlarged index i + mbc; the interface sits between cells i-1 and i
    for (int m = 0; m < nvar; ++m) { ql[m] = QD(pool, a.q, mitot, m, i - 1 + mbc); qr[m] = QD(pool, a.q, mitot, m, i + mbc); }
    rp1_at(a.P, ql, qr, W, S, AM, AP);
    for (int mw = 0; mw < mwaves; ++mw)
      for (int m = 0; m < nvar; ++m) sw[t][mw][m] = W[mw][m];
  }
  __syncthreads();
  double cfl = 0.0;
  double fmv[MAXW1], fpv[MAXW1];
  const bool face = valid && i >= 1 && i <= mx + 1;
  if (face) {
    for (int m = 0; m < nvar; ++m) { fpv[m] = 0.0 - AP[m]; fmv[m] = 0.0 + AM[m]; }
    for (int mw = 0; mw < mwaves; ++mw) {
      const double x = dtdx * S[mw], y = -dtdx * S[mw];
      cfl = (cfl < x) ? x : cfl;
      cfl = (cfl < y) ? y : cfl;
    }
    if (a.order != 1) {
      for (int mw = 0; mw < mwaves; ++mw) {
        if (a.mthlim[mw] == 0) continue;
        double wnorm2 = 0.0, dotl = 0.0, dotr = 0.0;
        for (int m = 0; m < nvar; ++m) {
          wnorm2 = wnorm2 + W[mw][m] * W[mw][m];
          dotr = dotr + W[mw][m] * sw[t + 1][mw][m];
          dotl = dotl + sw[t - 1][mw][m] * W[mw][m];
        }
        if (wnorm2 == 0.0) continue;
        const double wl = (S[mw] > 0.0) ? philim1(wnorm2, dotl, a.mthlim[mw]) : philim1(wnorm2, dotr, a.mthlim[mw]);
        for (int m = 0; m < nvar; ++m) W[mw][m] = wl * W[mw][m];
      }
      const double dtdxave = 0.5 * (dtdx + dtdx);
      for (int m = 0; m < nvar; ++m) {
        double cq = 0.0;
        for (int mw = 0; mw < mwaves; ++mw) cq = cq + fabs(S[mw]) * (1.0 - fabs(S[mw]) * dtdxave) * W[mw][m];
        fmv[m] = fmv[m] + 0.5 * cq;
        fpv[m] = fpv[m] + 0.5 * cq;
      }
    }
    // step1.f90: fm = 0 + faddm (fm was zeroed)
    for (int m = 0; m < nvar; ++m) {
      QD(pool, a.fm, mitot, m, i + mbc) = 0.0 + fmv[m];
      QD(pool, a.fp, mitot, m, i + mbc) = 0.0 + fpv[m];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_xor_sync(0xffffffffu, cfl, o);
    cfl = (cfl < v) ? v : cfl;
  }
  if ((t & 31) == 0) sred[t >> 5] = cfl;
  __syncthreads();
  // stepgrid.f:89-99: q(i) -= dtdx*(fm(i+1) - fp(i)) over the interior (enlarged mbc+1 .. mitot-mbc)
  const int ic = t + mbc + 1;
  if (ic <= mitot - mbc)
    for (int m = 0; m < nvar; ++m)
      QD(pool, a.q, mitot, m, ic) = QD(pool, a.q, mitot, m, ic) - dtdx * (QD(pool, a.fm, mitot, m, ic + 1) - QD(pool, a.fp, mitot, m, ic));
  if (t == 0) {
    double c = 0.0;
    for (int k = 0; k < STEP1_THREADS / 32; ++k) c = (c < sred[k]) ? sred[k] : c;
    atomicMax(cflmax, (unsigned long long)__double_as_longlong(c));
  }
}

// qad.f: the coarse/fine Riemann problems at a fine grid's two ends into svdflx (regs:
// svdflx(nvar,2), qc1d(nvar,2)); the fine states are the ghost cells nghost and mitot-nghost+1
__global__ void qad1_kernel(double* pool, long long q, int mitot, double* regs, long long ffl, double delt, Prob1 P) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nvar = P.meqn;
  double l[MAXW1], r[MAXW1], W[MAXW1][MAXW1], S[MAXW1], AM[MAXW1], AP[MAXW1];
  double* svd = regs + ffl;
  const double* qc = regs + ffl + 2 * nvar;
  for (int m = 0; m < nvar; ++m) { l[m] = qc[m]; r[m] = QD(pool, q, mitot, m, 2); }
  rp1_at(P, l, r, W, S, AM, AP);
  for (int m = 0; m < nvar; ++m) svd[m] = svd[m] + AM[m] * delt + AP[m] * delt;
  for (int m = 0; m < nvar; ++m) { l[m] = QD(pool, q, mitot, m, mitot - 2 + 1); r[m] = qc[nvar + m]; }
  rp1_at(P, l, r, W, S, AM, AP);
  for (int m = 0; m < nvar; ++m) svd[nvar + m] = svd[nvar + m] - AM[m] * delt - AP[m] * delt;
}

// fluxsv.f: entry k: coarse face flux into a kid's register (side 1: -fp(i), 2: -fm(i+1))
struct Fsv1 { int i, side; long long dst; };
__global__ void fluxsv1_kernel(double* pool, long long fm, long long fp, int mitot, int nvar, double* regs, const Fsv1* e, int n,
                               double dtc) {
  const int k = threadIdx.x + blockIdx.x * blockDim.x;
  if (k >= n) return;
  const Fsv1 x = e[k];
  for (int m = 0; m < nvar; ++m)
    regs[x.dst + m] = x.side == 1 ? -QD(pool, fp, mitot, m, x.i) * dtc : -QD(pool, fm, mitot, m, x.i + 1) * dtc;
}
// fluxad.f: the fine grid's boundary fluxes fm(ng+1), fp(mitot-ng+1) into its own register
__global__ void fluxad1_kernel(double* pool, long long fm, long long fp, int mitot, int nvar, double* regs, long long ffl, double dtf) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int m = 0; m < nvar; ++m) regs[ffl + m] = regs[ffl + m] + QD(pool, fm, mitot, m, 3) * dtf;
  for (int m = 0; m < nvar; ++m) regs[ffl + nvar + m] = regs[ffl + nvar + m] + QD(pool, fp, mitot, m, mitot - 2 + 1) * dtf;
}
// upbnd.f: the register terms of a coarse grid in listbc order (sequential: a cell's
// terms add up in that order)
struct Upb1 { int icrse; double sgnm; long long reg; };
__global__ void upbnd1_kernel(double* pool, long long q, int mitot, int nvar, const double* regs, const Upb1* e, int n, double area) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < n; ++k)
    for (int m = 0; m < nvar; ++m)
      QD(pool, q, mitot, m, e[k].icrse) = QD(pool, q, mitot, m, e[k].icrse) + e[k].sgnm * regs[e[k].reg + m] / area;
}
// update.f: coarse cells ci0.. (n of them) = mean of the ratio fine cells from fi0
__global__ void average1_kernel(double* pool, long long cq, int cmitot, long long fq, int fmitot, int ci0, int fi0, int n, int ratio,
                                int nvar) {
  const int k = threadIdx.x + blockIdx.x * blockDim.x;
  if (k >= n) return;
  const int i = ci0 + k, iff = fi0 + k * ratio;
  const double totrat = ratio;
  for (int m = 0; m < nvar; ++m) QD(pool, cq, cmitot, m, i) = 0.0;
  for (int ico = 1; ico <= ratio; ++ico)
    for (int m = 0; m < nvar; ++m) QD(pool, cq, cmitot, m, i) = QD(pool, cq, cmitot, m, i) + QD(pool, fq, fmitot, m, iff + ico - 1);
  for (int m = 0; m < nvar; ++m) QD(pool, cq, cmitot, m, i) = QD(pool, cq, cmitot, m, i) / totrat;
}
// cstore.f: the first and last cell of a coarse ring row into qc1d
__global__ void cstore1_kernel(const double* pool, long long tmp, int nrow, int nvar, double* regs, long long ffl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int m = 0; m < nvar; ++m) {
    regs[ffl + 2 * nvar + m] = pool[tmp + (long long)m * nrow];
    regs[ffl + 3 * nvar + m] = pool[tmp + (long long)m * nrow + nrow - 1];
  }
}
// flag2refine1.f90's test: out[i-1] = 1 where some component differs by more than tol
// between cells i-1 and i+1 (interior i = 1..mx); density only for the blast
__global__ void grad1_kernel(const double* pool, long long q, int mitot, int nvar, int density_only, double tol, int8_t* out) {
  const int i = 1 + threadIdx.x + blockIdx.x * blockDim.x;
  const int mx = mitot - 4;
  if (i > mx) return;
  int8_t f = 0;
  const int mend = density_only ? 1 : nvar;
  for (int m = 0; m < mend; ++m) {
    const double d = fabs(QD((double*)pool, q, mitot, m, i + 1 + 2) - QD((double*)pool, q, mitot, m, i - 1 + 2));
    const double dq = (0.0 < d) ? d : 0.0;  // max(0, dq)
    if (dq > tol) { f = 1; break; }
  }
  out[i - 1] = f;
}
// filval.f90:150-185: interpolation into a new grid's cells still NEEDS_TO_BE_SET (their
// component 1 marks them), from the coarse values valc (mic cells)
__global__ void filval1_kernel(double* pool, long long val, int mitot, long long valc, int mic, int ratio, int nvar, double unset) {
  const int k = threadIdx.x + blockIdx.x * blockDim.x;
  const int i = 2 + k / ratio, ico = 1 + k % ratio;
  if (i > mic - 1) return;
  const int ifine = (i - 2) * ratio + 2 + ico;
  if (QD(pool, val, mitot, 0, ifine) != unset) return;
  const double xoff = ((double)ico - 0.5) / ratio - 0.5;
  for (int m = 0; m < nvar; ++m) {
    const double s1p = QD(pool, valc, mic, m, i + 1) - QD(pool, valc, mic, m, i), s1m = QD(pool, valc, mic, m, i) - QD(pool, valc, mic, m, i - 1);
    const double d = QD(pool, valc, mic, m, i + 1) - QD(pool, valc, mic, m, i - 1);
    const double a = fabs(s1p), b = fabs(s1m);
    double slopex = ((b < a) ? b : a) * ((d >= 0.0) ? 1.0 : -1.0);
    if (s1m * s1p <= 0.0) slopex = 0.0;
    QD(pool, val, mitot, m, ifine) = QD(pool, valc, mic, m, i) + xoff * slopex;
  }
}
__global__ void fill_value1_kernel(double* pool, long long off, int n, double v) {
  const int k = threadIdx.x + blockIdx.x * blockDim.x;
  if (k < n) pool[off + k] = v;
}
// gauges_module.f90 (update_gauges): (1-xoff) q(i) + xoff q(i+1), tiny values zeroed
__global__ void gauge1_kernel(const double* pool, long long q, int mitot, int nvar, int ii, double xoff, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int m = 0; m < nvar; ++m) {
    double v = (1. - xoff) * QD((double*)pool, q, mitot, m, ii) + xoff * QD((double*)pool, q, mitot, m, ii + 1);
    if (fabs(v) < 1e-90) v = 0.0;
    out[m] = v;
  }
}
// conck.f: the level's mass, grid after grid, cell after cell (the reference's order)
struct Mass1 { long long q; int mitot; };
__global__ void mass1_kernel(const double* pool, const Mass1* g, int n, double hx, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double tot = 0.0;
  for (int k = 0; k < n; ++k)
    for (int i = 3; i <= g[k].mitot - 2; ++i) tot = tot + pool[g[k].q + i - 1];
  *out = tot * hx;
}
// valout.f90 (ASCII): |q| < 1e-90 set to zero over the interior
__global__ void zero_tiny1_kernel(double* pool, long long q, int mitot, int nvar) {
  const int k = threadIdx.x + blockIdx.x * blockDim.x;
  if (k >= mitot * nvar) return;
  const int i = k % mitot + 1;
  if (i < 3 || i > mitot - 2) return;
  double& v = pool[q + k];
  if (fabs(v) < 1e-90) v = 0.0;
}

int grid_for(long long n, int b) { return (int)std::max<long long>(1, (n + b - 1) / b); }

}  // namespace

// ======================================================================= host driver
class Amr1Gpu {
 public:
  struct Node {
    int ilo = 0, ihi = 0, level = 0, levelptr = 0, nextfree = 0, numflags = 0;
    double xlo = 0, xhi = 0, time = 0;
    long long q1 = -1, q2 = -1;  // pool offsets of store1, store2
    long long ffl = -1;          // register offset: svdflx(nvar,2), qc1d(nvar,2)
    std::vector<int> listbc;     // (i, side, kid, register index) per entry
    bool has_cfl = false;
    std::vector<double> flags;
    std::vector<signed char> dom2;
    std::vector<int> bnd;
  };
  // ---------------- input
  RunParams p;
  Prob1 prob{};
  double beta = 0;
  bool density_flags = false;
  double xlower = 0, xupper = 1;
  int nx = 0, nvar = 1, mwaves = 1, nghost = 2, mxnest = 1, kcheck = 2, ibuff = 2, max1d = 500;
  double tolsp = 0.1, cut = 0.7, cfl = 0.9, dt_max = 1e99, tfinal = 0, t0 = 0;
  int method2 = 2, mthbc1 = 1, mthbc2 = 1;
  bool xperdom = false, vtime = true;
  int mthlim[MAXW1] = {0, 0, 0};
  int intratx[12] = {0}, kratio[12] = {0};
  std::vector<double> tout;
  int nout = 0, iout = 0, nstop = IINFINITY1, output_format = 1;
  bool output_t0 = true;
  struct Gauge { int num; double x, t1, t2; };
  std::vector<Gauge> gauges;
  struct Row { int gauge, level; double t; long long slot; };
  std::vector<Row> grows;
  struct Region { int minlevel, maxlevel; double tlow, thi, xlow, xhi; };
  std::vector<Region> regions;
  // ---------------- state
  std::vector<Node> node;
  int ndfree = 1, lfine = 1;
  int lstart[12] = {0}, newstl[12] = {0}, listsp[12] = {0}, icheck[12] = {0}, iregsz[12] = {0};
  double hxposs[12] = {0}, possk[12] = {0};
  std::vector<int> levelgrids[12];
  double cfl_level = 0, cflmax_run = 0, rvol = 0, tmass0 = 0, time = 0;
  int ncycle = 0, matlabu = 0;
  std::string outdir;
  bool write_output = false, record_gauges = true;
  std::vector<int> mbestsrc;
  // ---------------- device
  cudaStream_t st = nullptr;
  Arena pool, regs;
  Staging stg;
  unsigned long long* d_cfl = nullptr;
  unsigned long long* h_cfl = nullptr;
  double* d_mass = nullptr;
  DBuf<double> d_gauge;
  long long gslots = 0;
  DBuf<Fsv1> d_fsv;
  DBuf<Upb1> d_upb;
  DBuf<Mass1> d_massg;
  long long nkernels = 0;
  double t_step = 0, t_regrid = 0, last_run_ms = 0, run_cells = 0;
  int max_cycles = 0;
  bool tick_started = false;
  int tk_nextout = 0;
  double tk_tlevel[12] = {0};

  ~Amr1Gpu() {
    if (st) cudaStreamSynchronize(st);
    pool.destroy(); regs.destroy();
    stg.destroy();
    d_gauge.free(); d_fsv.free(); d_upb.free(); d_massg.free();
    if (d_cfl) cudaFree(d_cfl);
    if (h_cfl) cudaFreeHost(h_cfl);
    if (d_mass) cudaFree(d_mass);
    if (st) cudaStreamDestroy(st);
  }

  // ================================================================ input
  void read_input(const std::string& dir) {
    KeyFile c, a, g, r, s;
    if (!c.read(dir + "/claw.data")) throw std::runtime_error("cannot read claw.data");
    if (!a.read(dir + "/amr.data")) throw std::runtime_error("cannot read amr.data");
    if (c.n("num_dim") != 1) throw std::runtime_error("1D solver: num_dim must be 1");
    xlower = c.f("lower"); xupper = c.f("upper"); nx = c.n("num_cells");
    nvar = c.n("num_eqn"); mwaves = c.n("num_waves");
    if (c.n("num_aux") != 0) throw std::runtime_error("1D solver: no 1D problem carries aux arrays");
    if (c.n("capa_index") != 0) throw std::runtime_error("1D solver: capacity functions are not supported");
    if (c.b("use_fwaves")) throw std::runtime_error("1D solver: f-waves are not supported");
    t0 = c.f("t0");
    const int os = c.n("output_style");
    if (os == 1) {
      nout = c.n("num_output_times"); tfinal = c.f("tfinal"); output_t0 = c.b("output_t0");
      for (int k = 1; k <= nout; ++k) tout.push_back(t0 + k * (tfinal - t0) / (double)nout);
    } else if (os == 2) {
      for (auto& x : c.at("output_times")) tout.push_back(KeyFile::num(x));
      nout = (int)tout.size();
      output_t0 = tout[0] == t0;
      if (output_t0) { tout.erase(tout.begin()); nout -= 1; }
      tfinal = tout.back();
    } else {
      iout = c.n("output_step_interval"); nstop = c.n("total_steps"); output_t0 = c.b("output_t0"); tfinal = RINFINITY1;
    }
    output_format = c.n_or("output_format", 1);
    if (output_format != 1 && output_format != 3) throw std::runtime_error("output_format must be 1 (ASCII) or 3 (binary)");
    possk[1] = c.f("dt_initial"); dt_max = c.f("dt_max"); cfl = c.f("cfl_desired");
    vtime = c.b("dt_variable");
    method2 = c.n("order");
    if (c.n_or("source_split", 0) > 1) throw std::runtime_error("1D solver: source_split must be 0 or 1");
    for (int k = 0; k < mwaves && k < MAXW1; ++k) mthlim[k] = c.n("limiter", k);
    nghost = c.n("num_ghost");
    if (nghost != 2) throw std::runtime_error("1D solver: num_ghost must be 2");
    mthbc1 = c.n("bc_lower"); mthbc2 = c.n("bc_upper");
    if ((mthbc1 == 2) != (mthbc2 == 2)) throw std::runtime_error("periodic boundaries: both sides must be 2");
    for (int code : {mthbc1, mthbc2})
      if (code != 1 && code != 2 && code != 3) throw std::runtime_error("1D solver: boundaries must be extrapolation, periodic or wall");
    xperdom = mthbc1 == 2;
    mxnest = a.n("amr_levels_max");
    if (mxnest > 10) throw std::runtime_error("at most 10 levels");
    for (int k = 0; k < std::max(1, mxnest - 1); ++k) { intratx[k + 1] = a.n("refinement_ratios_x", k); kratio[k + 1] = a.n("refinement_ratios_t", k); }
    if (a.b("flag_richardson")) throw std::runtime_error("1D solver: Richardson estimation is not built for 1D");
    if (!a.b("flag2refine")) tolsp = 1e300; else tolsp = a.f("flag2refine_tol");
    kcheck = a.n("regrid_interval"); ibuff = a.n("regrid_buffer_width"); cut = a.f("clustering_cutoff");
    max1d = a.n_or("max1d", 500);
    if (max1d > STEP1_THREADS + 3) throw std::runtime_error("1D solver: max1d must be at most 515");
    if (r.read(dir + "/regions.data"))
      for (auto& row : r.rows)
        if (row.size() >= 6)
          regions.push_back(Region{(int)KeyFile::num(row[0]), (int)KeyFile::num(row[1]), KeyFile::num(row[2]), KeyFile::num(row[3]),
                                   KeyFile::num(row[4]), KeyFile::num(row[5])});
    if (g.read(dir + "/gauges.data"))
      for (auto& row : g.rows)
        if (row.size() >= 4) gauges.push_back(Gauge{(int)KeyFile::num(row[0]), KeyFile::num(row[1]), KeyFile::num(row[2]), KeyFile::num(row[3])});
    if (!s.read(dir + "/setprob.data")) throw std::runtime_error("cannot read setprob.data");
    const std::string pr = s.str("problem");
    prob.meqn = nvar; prob.mwaves = mwaves;
    if (pr == "advection_1d") {
      prob.solver = SOLVER1_ADVECTION; prob.u = s.f("u"); beta = s.f("beta");
      if (nvar != 1 || mwaves != 1) throw std::runtime_error("advection_1d needs num_eqn = num_waves = 1");
    } else if (pr == "acoustics_1d") {
      prob.solver = SOLVER1_ACOUSTICS; prob.rho = s.f("rho"); prob.bulk = s.f("bulk"); beta = s.f("beta");
      prob.cc = std::sqrt(prob.bulk / prob.rho); prob.zz = prob.cc * prob.rho;
      if (nvar != 2 || mwaves != 2) throw std::runtime_error("acoustics_1d needs num_eqn = num_waves = 2");
    } else if (pr == "euler_1d_wcblast") {
      prob.solver = SOLVER1_EULER; prob.gamma = s.f_or("gamma", 1.4); prob.gamma1 = prob.gamma - 1.0;
      density_flags = true;
      if (nvar != 3 || mwaves != 3) throw std::runtime_error("euler_1d_wcblast needs num_eqn = num_waves = 3");
    } else {
      throw std::runtime_error("1D solver: unknown problem '" + pr + "' (advection_1d, acoustics_1d, euler_1d_wcblast)");
    }
  }
  // qinit of the reference's 1D regression tests (the problem's user hook, run on the host)
  void qinit(int mx, double xl, double dx, std::vector<double>& q, int mitot) {
    for (int i = 1; i <= mx; ++i) {
      const double xcell = xl + (i - 0.5) * dx;
      auto Q = [&](int m) -> double& { return q[(size_t)m * mitot + (i + 2 - 1)]; };
      if (prob.solver == SOLVER1_ADVECTION) {
        Q(0) = std::exp(-beta * ((xcell - 0.75) * (xcell - 0.75)));
        if (xcell > 0.1 && xcell < 0.4) Q(0) = Q(0) + 1.0;
      } else if (prob.solver == SOLVER1_ACOUSTICS) {
        Q(0) = std::exp(-beta * ((xcell - 0.3) * (xcell - 0.3)));
        Q(1) = 0.0;
      } else {
        Q(0) = 1.0; Q(1) = 0.0;
        if (xcell < 0.1) Q(2) = 1.e3 / prob.gamma1;
        else if (xcell < 0.9) Q(2) = 1.e-2 / prob.gamma1;
        else Q(2) = 1.e2 / prob.gamma1;
      }
    }
  }

  // ================================================================ storage
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
    node[m] = Node();
    return m;
  }
  void putnod(int m) { node[m].nextfree = ndfree; ndfree = m; }
  int mitot_of(int m) const { return node[m].ihi - node[m].ilo + 1 + 2 * nghost; }
  long long qsize(int m) const { return (long long)nvar * mitot_of(m); }
  long long palloc(long long n) { return pool.alloc(n); }
  void pfree(long long off, long long n) { if (off >= 0) pool.release(off, n); }

  // ================================================================ ghost cells
  void launch_bc(long long off, int nrow, double hx, double xlo_p, double xhi_p) {
    if (xperdom) return;
    const double hxmarg = hx * .01;
    int nxl = 0, ibeg = 0;
    if (xlo_p < xlower - hxmarg) nxl = (int)((xlower + hxmarg - xlo_p) / hx);
    if (xhi_p > xupper + hxmarg) { const int nxr = (int)((xhi_p - xupper + hxmarg) / hx); ibeg = std::max(nrow - nxr + 1, 1); }
    if (nxl == 0 && ibeg == 0) return;
    // the cells the boundary conditions read must lie in the array
    if ((nxl > 0 && (mthbc1 == 3 ? 2 * nxl > nrow : nxl + 1 > nrow)) ||
        (ibeg > 0 && (mthbc2 == 3 ? 2 * ibeg - 1 - nrow < 1 : ibeg - 1 < 1)))
      throw std::runtime_error("bc1amr: ghost region wider than its array");
    bc1_kernel<<<1, 1, 0, st>>>(pool.d, off, nrow, nvar, nxl, mthbc1, ibeg, mthbc2);
    ++nkernels;
  }
  // intfil.f90 into the array at `dst` (dmitot cells) from row nrowst: flaguse of [ilo,ihi]
  void intfil(long long dst, int dmitot, double t, std::vector<signed char>& flaguse, int nrowst, int ilo, int ihi, int level, int msrc) {
    const double t_epsilon = 1.0e-4, dt = possk[level];
    std::fill(flaguse.begin(), flaguse.end(), 0);
    const std::vector<int>& srcs = msrc == -1 ? levelgrids[level] : node[msrc].bnd;
    for (int mptr : srcs) {
      Node& g = node[mptr];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi);
      if (ixlo > ixhi) continue;
      const double alphac = (g.time - t) / dt;
      const double alphai = 1.0 - alphac;
      if (alphai < -t_epsilon || alphai > 1.0 + t_epsilon) throw std::runtime_error("intfil: time wanted not available");
      int mode;
      if (std::fabs(alphai - 1.0) < t_epsilon) mode = 1;
      else if (std::fabs(alphai) < t_epsilon) mode = 2;
      else mode = 3;
      if (mode != 1 && level == mxnest) throw std::runtime_error("intfil: old values wanted at the finest level");
      const int n = ixhi - ixlo + 1;
      copy1_kernel<<<grid_for(n, 128), 128, 0, st>>>(pool.d, dst, dmitot, ixlo - ilo + nrowst, g.q1, g.q2, mitot_of(mptr),
                                                    ixlo - g.ilo + nghost + 1, n, nvar, mode, alphai, alphac);
      ++nkernels;
      for (int i = ixlo; i <= ixhi; ++i) flaguse[i - ilo] = 1;
    }
    if (ilo < 0) for (int i = ilo; i <= std::min(-1, nrowst + ihi - ilo); ++i) if (i <= ihi) flaguse[i - ilo] = 1;
    if (ihi >= iregsz[level]) for (int i = std::max(iregsz[level], ilo); i <= ihi; ++i) flaguse[i - ilo] = 1;
  }
  static double sgn1(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }
  // filpatch.f90 (filrecur) into the array at `dst` (dmitot cells)
  void filrecur(int level, long long dst, int dmitot, double t, int nrowst, int ilo, int ihi, bool patchOnly, int msrc) {
    const int mitot_patch = ihi - ilo + 1;
    const double dx_fine = hxposs[level], xlow_fine = xlower + ilo * dx_fine;
    std::vector<signed char> flaguse(mitot_patch);
    intfil(dst, dmitot, t, flaguse, nrowst, ilo, ihi, level, msrc);
    int first = -1, last = -1;
    for (int i = 1; i <= mitot_patch; ++i) if (!flaguse[i - 1]) { if (first < 0) first = i; last = i; }
    if (first > 0) {
      if (level == 1) throw std::runtime_error("filrecur: level 1 cells not covered");
      const double dx_coarse = hxposs[level - 1];
      const int u0 = first + ilo - 1, u1 = last + ilo - 1;
      const int r = intratx[level - 1];
      const int iplo = (u0 - r + nghost * r) / r - nghost, iphi = (u1 + r) / r;
      const double xlow_coarse = xlower + iplo * dx_coarse;
      const int mitot_coarse = iphi - iplo + 1;
      if (mitot_coarse > ihi - ilo + 3) throw std::runtime_error("filrecur: coarse patch too large");
      const long long crse = palloc((long long)nvar * mitot_coarse);
      fill_value1_kernel<<<grid_for((long long)nvar * mitot_coarse, 128), 128, 0, st>>>(pool.d, crse, nvar * mitot_coarse, 0.0);
      ++nkernels;
      if (xperdom && (iplo < 0 || iphi >= iregsz[level - 1])) prefilrecur(level - 1, crse, mitot_coarse, t, iplo, iphi, iplo);
      else filrecur(level - 1, crse, mitot_coarse, t, 1, iplo, iphi, true, -1);
      const double ratiox = (double)r;
      Interp1 op{};
      auto flush = [&] {
        if (op.n == 0) return;
        interp1_kernel<<<1, 32, 0, st>>>(pool.d, dst, dmitot, crse, mitot_coarse, op, nvar);
        ++nkernels;
        op.n = 0;
      };
      for (int i_fine = 1; i_fine <= mitot_patch; ++i_fine) {
        if (flaguse[i_fine - 1] != 0) continue;
        const int i_coarse = (int)std::floor((i_fine + ilo - 1) / ratiox) - iplo + 1;
        if (i_coarse < 2 || i_coarse > mitot_coarse - 1) throw std::runtime_error("filrecur: coarse stencil outside its patch");
        const double xcent_coarse = xlow_coarse + (i_coarse - .5) * dx_coarse;
        const double xcent_fine = xlower + (i_fine - 1 + ilo + .5) * dx_fine;
        op.dst_i[op.n] = i_fine + nrowst - 1;
        op.ic[op.n] = i_coarse;
        op.eta[op.n] = (xcent_fine - xcent_coarse) / dx_coarse;
        if (++op.n == 8) flush();
      }
      flush();
      pfree(crse, (long long)nvar * mitot_coarse);
    }
    if (patchOnly) launch_bc(dst, dmitot, dx_fine, xlow_fine, xlower + (ihi + 1) * dx_fine);
  }
  // prefilp.f90 (prefilrecur): the periodic pieces of [ilo,ihi], each into a scratch array
  // filled at its shifted place, then copied to the array at `dst` whose cell 1 is iglo
  void prefilrecur(int level, long long dst, int dmitot, double t, int ilo, int ihi, int iglo) {
    int ist[3] = {ilo, 0, iregsz[level]}, iend[3] = {-1, iregsz[level] - 1, ihi}, ish[3] = {iregsz[level], 0, -iregsz[level]};
    if (!xperdom) { ist[0] = iregsz[level]; ist[1] = ilo; ist[2] = iregsz[level]; iend[0] = -1; iend[1] = ihi; iend[2] = -1; ish[0] = ish[1] = ish[2] = 0; }
    for (int k = 0; k < 3; ++k) {
      const int i1 = std::max(ilo, ist[k]), i2 = std::min(ihi, iend[k]);
      if (i1 > i2) continue;
      const int mi = i2 - i1 + 1;
      const long long piece = palloc((long long)nvar * mi);
      fill_value1_kernel<<<grid_for((long long)nvar * mi, 128), 128, 0, st>>>(pool.d, piece, nvar * mi, 0.0);
      filrecur(level, piece, mi, t, 1, i1 + ish[k], i2 + ish[k], true, -1);
      copy1_kernel<<<grid_for(mi, 128), 128, 0, st>>>(pool.d, dst, dmitot, i1 - iglo + 1, piece, piece, mi, 1, mi, nvar, 1, 1.0, 0.0);
      nkernels += 2;
      pfree(piece, (long long)nvar * mi);
    }
  }
  // bound.f90
  void bound(double t, int mptr) {
    const Node& g = node[mptr];
    const int ng = nghost, lev = g.level, mitot = mitot_of(mptr);
    const double hx = hxposs[lev];
    const long long q = g.q1;
    if ((g.xlo - ng * hx < xlower) && xperdom) prefilrecur(lev, q, mitot, t, g.ilo - ng, g.ilo - 1, g.ilo - ng);
    else filrecur(lev, q, mitot, t, 1, g.ilo - ng, g.ilo - 1, false, mptr);
    if ((g.xhi + ng * hx > xupper) && xperdom) prefilrecur(lev, q, mitot, t, g.ihi + 1, g.ihi + ng, g.ilo - ng);
    else filrecur(lev, q, mitot, t, mitot - ng + 1, g.ihi + 1, g.ihi + ng, false, mptr);
    launch_bc(q, mitot, hx, g.xlo - ng * hx, g.xhi + ng * hx);
  }
  // icall.f: store1 of the grids of `level` over [ilo,ihi] into the array at dst from iputst
  void icall(long long dst, int dmitot, int ilo, int ihi, int level, int iputst) {
    for (int mptr = lstart[level]; mptr != 0; mptr = node[mptr].levelptr) {
      const Node& g = node[mptr];
      const int ixlo = std::max(g.ilo, ilo), ixhi = std::min(g.ihi, ihi);
      if (ixlo > ixhi) continue;
      const int n = ixhi - ixlo + 1;
      copy1_kernel<<<grid_for(n, 128), 128, 0, st>>>(pool.d, dst, dmitot, ixlo - ilo + iputst, g.q1, g.q1, mitot_of(mptr),
                                                    ixlo - g.ilo + nghost + 1, n, nvar, 1, 1.0, 0.0);
      ++nkernels;
    }
  }
  void preicall(long long dst, int dmitot, int ilo, int ihi, int level) {
    const int ist[3] = {ilo, 0, iregsz[level]}, iend[3] = {-1, iregsz[level] - 1, ihi}, ish[3] = {iregsz[level], 0, -iregsz[level]};
    for (int k = 0; k < 3; ++k) {
      const int i1 = std::max(ilo, ist[k]), i2 = std::min(ihi, iend[k]);
      if (i1 <= i2) icall(dst, dmitot, i1 + ish[k], i2 + ish[k], level, i1 - ilo + 1);
    }
  }

  // ================================================================ level substep
  void saveqc(int level) {
    const int levc = level - 1;
    const double hxc = hxposs[levc];
    for (int mkid = lstart[level]; mkid != 0; mkid = node[mkid].levelptr) {
      const Node& k = node[mkid];
      const int iclo = k.ilo / intratx[levc] - 1, ichi = (k.ihi + 1) / intratx[levc];
      const int nrow = ichi - iclo + 1;
      const long long tmp = palloc((long long)nvar * nrow);
      fill_value1_kernel<<<grid_for((long long)nvar * nrow, 128), 128, 0, st>>>(pool.d, tmp, nvar * nrow, 0.0);
      ++nkernels;
      if ((iclo < 0 || ichi == iregsz[levc]) && xperdom) preicall(tmp, nrow, iclo, ichi, levc);
      else icall(tmp, nrow, iclo, ichi, levc, 1);
      launch_bc(tmp, nrow, hxc, k.xlo - hxc, k.xhi + hxc);
      cstore1_kernel<<<1, 1, 0, st>>>(pool.d, tmp, nrow, nvar, regs.d, k.ffl);
      ++nkernels;
      pfree(tmp, (long long)nvar * nrow);
    }
  }
  void sample_gauges(int mptr) {
    if (!record_gauges || gauges.empty()) return;
    const Node& g = node[mptr];
    const double hx = hxposs[g.level], xlow = g.xlo - nghost * hx;
    for (size_t i = 0; i < gauges.size(); ++i) {
      if (mptr != mbestsrc[i]) continue;
      if (g.time < gauges[i].t1 || g.time > gauges[i].t2) continue;
      const int iindex = (int)(.5 + (gauges[i].x - xlow) / hx);
      const double xcent = xlow + (iindex - .5) * hx;
      const double xoff = (gauges[i].x - xcent) / hx;
      if ((long long)(gslots + 1) * nvar > (long long)d_gauge.cap) {
        std::vector<double> old((size_t)gslots * nvar);
        if (gslots) {
          AMR_CUDA(cudaMemcpyAsync(old.data(), d_gauge.d, sizeof(double) * old.size(), cudaMemcpyDeviceToHost, st));
          AMR_CUDA(cudaStreamSynchronize(st));
        }
        d_gauge.ensure(std::max<size_t>(1024, 2 * d_gauge.cap + nvar));
        if (gslots) AMR_CUDA(cudaMemcpyAsync(d_gauge.d, old.data(), sizeof(double) * old.size(), cudaMemcpyHostToDevice, st));
        AMR_CUDA(cudaStreamSynchronize(st));
      }
      gauge1_kernel<<<1, 1, 0, st>>>(pool.d, g.q1, mitot_of(mptr), nvar, iindex, xoff, d_gauge.d + gslots * nvar);
      ++nkernels;
      grows.push_back(Row{gauges[i].num, g.level, g.time, gslots});
      ++gslots;
    }
  }
  // advanc.f / par_advanc: ghost fill, saveqc, then per grid qad, gauges, step, registers
  double advanc(int level) {
    for (int mptr : levelgrids[level]) bound(node[mptr].time, mptr);
    if (level + 1 <= mxnest && lstart[level + 1] != 0) saveqc(level + 1);
    AMR_CUDA(cudaMemsetAsync(d_cfl, 0, sizeof(unsigned long long), st));
    const double hx = hxposs[level], delt = possk[level];
    double dtlevnew = RINFINITY1;
    for (int mptr : levelgrids[level]) {
      Node& g = node[mptr];
      const int mitot = mitot_of(mptr);
      if (level < mxnest) AMR_CUDA(cudaMemcpyAsync(pool.d + g.q2, pool.d + g.q1, sizeof(double) * qsize(mptr), cudaMemcpyDeviceToDevice, st));
      rvol = rvol + (g.ihi - g.ilo + 1);
      if (g.ffl >= 0) { qad1_kernel<<<1, 1, 0, st>>>(pool.d, g.q1, mitot, regs.d, g.ffl, delt, prob); ++nkernels; }
      sample_gauges(mptr);
      const long long fl = palloc(2LL * qsize(mptr));
      AMR_CUDA(cudaMemsetAsync(pool.d + fl, 0, sizeof(double) * 2 * qsize(mptr), st));
      Step1Args a{};
      a.q = g.q1; a.fm = fl; a.fp = fl + qsize(mptr); a.mitot = mitot; a.nvar = nvar; a.mwaves = mwaves; a.order = method2;
      for (int k = 0; k < MAXW1; ++k) a.mthlim[k] = mthlim[k];
      a.dt = delt; a.dx = hx; a.P = prob;
      // per-grid Courant numbers: each grid's step gets the level maximum so far reset
      // through its own dtnew below; the level maximum is the max of the grids'
      AMR_CUDA(cudaMemsetAsync(d_cfl + 1, 0, sizeof(unsigned long long), st));
      step1_kernel<<<1, STEP1_THREADS, 0, st>>>(pool.d, a, d_cfl + 1);
      ++nkernels;
      if (g.has_cfl) {
        std::vector<Fsv1> e;
        for (size_t k = 0; k + 3 < g.listbc.size(); k += 4) {
          if (g.listbc[k] == 0) break;
          e.push_back(Fsv1{g.listbc[k], g.listbc[k + 1], node[g.listbc[k + 2]].ffl + (long long)nvar * (g.listbc[k + 3] - 1)});
        }
        if (!e.empty()) {
          d_fsv.upload(e, st, stg);
          fluxsv1_kernel<<<grid_for((long long)e.size(), 64), 64, 0, st>>>(pool.d, a.fm, a.fp, mitot, nvar, regs.d, d_fsv.d, (int)e.size(), delt);
          ++nkernels;
        }
      }
      if (g.ffl >= 0) { fluxad1_kernel<<<1, 1, 0, st>>>(pool.d, a.fm, a.fp, mitot, nvar, regs.d, g.ffl, delt); ++nkernels; }
      AMR_CUDA(cudaMemcpyAsync(h_cfl, d_cfl + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
      AMR_CUDA(cudaStreamSynchronize(st));
      stg.reset();
      double cflgrid;
      std::memcpy(&cflgrid, h_cfl, sizeof(double));
      cfl_level = std::max(cfl_level, cflgrid);
      dtlevnew = std::min(dtlevnew, cflgrid > 0.0 ? delt * cfl / cflgrid : RINFINITY1);
      pfree(fl, 2LL * qsize(mptr));
      g.time = g.time + delt;
    }
    cflmax_run = std::max(cflmax_run, cfl_level);
    return dtlevnew;
  }

  // ================================================================ level sync
  void update(int level) {
    for (int mptr : levelgrids[level]) {
      Node& g = node[mptr];
      const int mitot = mitot_of(mptr);
      if (g.has_cfl) {
        std::vector<Upb1> e;
        std::vector<int> iused(mitot + 1, 0);
        for (size_t k = 0; k + 3 < g.listbc.size(); k += 4) {
          const int icrse = g.listbc[k];
          if (icrse == 0) break;
          const int iside = g.listbc[k + 1], norm = 1 << (iside - 1);
          if ((iused[icrse] / norm) % 2 == 1) continue;
          e.push_back(Upb1{icrse, iside == 2 ? -1.0 : 1.0, node[g.listbc[k + 2]].ffl + (long long)nvar * (g.listbc[k + 3] - 1)});
          iused[icrse] = iused[icrse] + norm;
        }
        if (!e.empty()) {
          d_upb.upload(e, st, stg);
          upbnd1_kernel<<<1, 1, 0, st>>>(pool.d, g.q1, mitot, nvar, regs.d, d_upb.d, (int)e.size(), hxposs[level]);
          ++nkernels;
        }
      }
      for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        const Node& k = node[mkid];
        const int iclo = k.ilo / intratx[level], ichi = k.ihi / intratx[level];
        const int iplo = std::max(g.ilo, iclo), iphi = std::min(g.ihi, ichi);
        if (iplo > iphi) continue;
        const int n = iphi - iplo + 1;
        average1_kernel<<<grid_for(n, 64), 64, 0, st>>>(pool.d, g.q1, mitot, k.q1, mitot_of(mkid), iplo - g.ilo + nghost + 1,
                                                       iplo * intratx[level] - k.ilo + nghost + 1, n, intratx[level], nvar);
        ++nkernels;
      }
    }
  }
  void prepf(int level) {
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
      node[m].ffl = regs.alloc(4LL * nvar);
      AMR_CUDA(cudaMemsetAsync(regs.d + node[m].ffl, 0, sizeof(double) * 4 * nvar, st));
    }
  }
  void setuse(std::vector<int>& lb, int mkid, int ilo, int ihi, int iclo, int ichi) {
    const int ist = iclo - 1, iend = ichi + 1;
    if (!(ist < ilo)) lb.insert(lb.end(), {ist - ilo + nghost + 1, 2, mkid, 1});
    if (!(iend > ihi)) lb.insert(lb.end(), {iend - ilo + nghost + 1, 1, mkid, 2});
  }
  // prepc.f (its first periodic branch adds nothing: it calls setuse with the 2D argument
  // list, so kflag is never 1)
  void prepc(int level) {
    int maxsp = 0;
    for (int m = lstart[level + 1]; m != 0; m = node[m].levelptr) maxsp += 2;
    listsp[level] = maxsp;
    if (maxsp == 0) return;
    const int imax = iregsz[level] - 1;
    for (int mpar = lstart[level]; mpar != 0; mpar = node[mpar].levelptr) {
      Node& p_ = node[mpar];
      p_.listbc.clear();
      p_.has_cfl = true;
      for (int mkid = lstart[level + 1]; mkid != 0; mkid = node[mkid].levelptr) {
        const int iclo = node[mkid].ilo / intratx[level], ichi = node[mkid].ihi / intratx[level];
        if (std::max(p_.ilo, iclo) <= std::min(p_.ihi, ichi) + 1) setuse(p_.listbc, mkid, p_.ilo, p_.ihi, iclo, ichi);
        if (xperdom && iclo == 0 && p_.ihi == imax) setuse(p_.listbc, mkid, p_.ilo, p_.ihi, iclo + iregsz[level], ichi + iregsz[level]);
      }
      p_.listbc.resize((size_t)4 * maxsp, 0);
    }
  }
  void putsp(int lbase, int level) {
    if (level != lfine)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { node[m].listbc.clear(); node[m].has_cfl = false; }
    if (level == lbase) return;
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
      if (node[m].ffl >= 0) regs.release(node[m].ffl, 4LL * nvar);
      node[m].ffl = -1;
    }
  }

  // ================================================================ grid lists
  void makeGridList(int lbase) {
    for (int lev = lbase + 1; lev <= lfine; ++lev) {
      levelgrids[lev].clear();
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) levelgrids[lev].push_back(m);
    }
  }
  void makeBndryList(int level) {
    const std::vector<int>& G = levelgrids[level];
    for (size_t n = 0; n < G.size(); ++n) {
      Node& g = node[G[n]];
      g.bnd.clear();
      const int imin = g.ilo - nghost, imax = g.ihi + nghost;
      for (size_t k = 0; k < G.size(); ++k) {
        if (k == n) continue;
        const Node& s = node[G[k]];
        if (std::max(s.ilo, imin) <= std::min(s.ihi, imax)) g.bnd.insert(g.bnd.begin(), G[k]);
      }
    }
  }
  // quick_sort1.f (qsorti), step by step: ties decide the grid order
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
  void arrangeGrids(int level, int numg) {
    std::vector<int> listgrids(numg + 1), index(numg + 1);
    std::vector<long long> cost(numg + 1);
    int mptr = lstart[level];
    for (int i = 1; i <= numg; ++i) { listgrids[i] = mptr; cost[i] = node[mptr].ihi - node[mptr].ilo + 1; mptr = node[mptr].levelptr; }
    qsorti(index, numg, cost);
    lstart[level] = listgrids[index[numg]];
    int prev = listgrids[index[numg]];
    for (int i = 1; i <= numg - 1; ++i) { node[prev].levelptr = listgrids[index[numg - i]]; prev = listgrids[index[numg - i]]; }
    node[prev].levelptr = 0;
  }
  void birect(int mptr1) {
    int mptr = mptr1;
    const int level = node[mptr].level;
    const double hx = hxposs[level];
    while (true) {
      const int nxg = node[mptr].ihi - node[mptr].ilo + 1;
      if (nxg + 2 * nghost > max1d) {
        int nxl = nxg / 2;
        const int lratio = level > 1 ? intratx[level - 1] : 2;
        nxl = (nxl / lratio) * lratio;
        const double cxmid = node[mptr].xlo + nxl * hx, cxhi = node[mptr].xhi;
        const int mnx = nodget();
        Node& a = node[mptr];
        Node& b = node[mnx];
        b.levelptr = a.levelptr; a.levelptr = mnx;
        a.xhi = cxmid;
        b.ihi = a.ihi; a.ihi = a.ilo + nxl - 1; b.ilo = a.ihi + 1;
        b.xlo = cxmid; b.xhi = cxhi; b.time = a.time; b.level = a.level;
        continue;
      }
      mptr = node[mptr].levelptr;
      if (mptr == 0) break;
    }
  }

  // ================================================================ flagging
  // flagger.f with flagregions1.f90 and flag2refine1.f90: the gradient test runs on the
  // device (grad1_kernel) over store1 after a ghost fill, or store2 at a run's first step
  void flagger(int lcheck, double start_time) {
    const int mbuff = std::max(nghost, ibuff + 1);
    for (int mptr : levelgrids[lcheck]) {
      Node& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1, mitot = nxg + 2 * nghost;
      g.flags.assign(nxg + 2 * mbuff, UNSET1);
      long long use;
      if (start_time + possk[lcheck] != g.time) { bound(g.time, mptr); use = g.q1; }
      else use = g.q2;
      // flagregions1.f90
      std::vector<int> minl(nxg + 1, 0), maxl(nxg + 1, 0);
      const double dx = hxposs[lcheck], xu = g.xlo + nxg * dx;
      for (const Region& R : regions) {
        if (g.time < R.tlow || g.time > R.thi) continue;
        if (g.xlo >= R.xhi || xu <= R.xlow) continue;
        const int i1 = std::max((int)std::floor((R.xlow - g.xlo) / dx) + 1, 1), i2 = std::min((int)std::floor((R.xhi - g.xlo) / dx) + 1, nxg);
        for (int i = i1; i <= i2; ++i) { minl[i] = std::max(minl[i], R.minlevel); maxl[i] = std::max(maxl[i], R.maxlevel); }
      }
      for (int i = 1; i <= nxg; ++i) {
        if (minl[i] > maxl[i]) throw std::runtime_error("flagregions1: minlevel > maxlevel");
        if (maxl[i] != 0) {
          if (lcheck < minl[i]) g.flags[i + mbuff - 1] = DOFLAG1;
          else if (lcheck >= maxl[i]) g.flags[i + mbuff - 1] = DONTFLAG1;
        }
      }
      if (tolsp > 1e299) continue;  // flag2refine = False
      std::vector<int8_t> grad(nxg);
      DBuf<int8_t> d_grad;
      d_grad.ensure(nxg);
      grad1_kernel<<<grid_for(nxg, 128), 128, 0, st>>>(pool.d, use, mitot, nvar, density_flags ? 1 : 0, tolsp, d_grad.d);
      ++nkernels;
      AMR_CUDA(cudaMemcpyAsync(grad.data(), d_grad.d, nxg, cudaMemcpyDeviceToHost, st));
      AMR_CUDA(cudaStreamSynchronize(st));
      d_grad.free();
      if (density_flags) {
        // tests/euler_1d_wcblast/flag2refine1.f90: every cell DONTFLAG, then the density test
        for (double& f : g.flags) f = DONTFLAG1;
        for (int i = 1; i <= nxg; ++i) if (grad[i - 1]) g.flags[i + mbuff - 1] = DOFLAG1;
      } else {
        bool keep = false;
        for (double f : g.flags) if (f == UNSET1) { keep = true; break; }
        if (keep)
          for (int i = 1; i <= nxg; ++i) if (g.flags[i + mbuff - 1] == UNSET1 && grad[i - 1]) g.flags[i + mbuff - 1] = DOFLAG1;
      }
    }
  }
  void projec1(int level, Node& g, int mbuff) {
    const int lrat2x = intratx[level] * intratx[level + 1];
    for (int mkid = newstl[level + 2]; mkid != 0; mkid = node[mkid].levelptr) {
      const Node& k = node[mkid];
      int ist = (int)std::floor((float)k.ilo / (float)lrat2x);
      int iend = (int)std::ceil((k.ihi + 1.0) / lrat2x) - 1;
      if (ibuff == 0) {
        if (ist * lrat2x == k.ilo) ist = ist - 1;
        if ((iend + 1) * lrat2x == k.ihi + 1) iend = iend + 1;
      }
      for (int i = std::max(ist, g.ilo - mbuff); i <= std::min(iend, g.ihi + mbuff); ++i) {
        double& f = g.flags[i - (g.ilo - mbuff)];
        if (f <= DONTFLAG1) f = BADPRO1;
      }
    }
  }
  void shiftset(Node& g, int mbuff) {
    const int lo = g.ilo - mbuff;
    std::vector<double> copy(g.flags.size(), 0.0);
    for (int i = g.ilo; i <= g.ihi; ++i) {
      const double r = g.flags[i - lo];
      if (r > 0) for (int m = i - ibuff; m <= i + ibuff; ++m) copy[m - lo] = r;
    }
    g.flags = copy;
  }
  void setPhysBndryFlags(std::vector<signed char>& f, int ilo, int ihi, int mbuff, int level) {
    const int lo = ilo - mbuff;
    if (ilo - mbuff < 0 && !xperdom) for (int i = ilo - mbuff; i <= -1; ++i) f[i - lo] = 1;
    if (ihi + mbuff >= iregsz[level] && !xperdom) for (int i = iregsz[level]; i <= ihi + mbuff; ++i) f[i - lo] = 1;
  }
  void griddomshrink(const std::vector<signed char>& in, int ilo, int ihi, int mbuff, std::vector<signed char>& out, int level) {
    const int lo = ilo - mbuff;
    out.assign(ihi - ilo + 1 + 2 * mbuff, 0);
    for (int i = ilo - mbuff + 1; i <= ihi + mbuff - 1; ++i) {
      out[i - lo] = in[i - lo];
      if (in[i - lo] <= 0 || in[i + 1 - lo] <= 0 || in[i - 1 - lo] <= 0) out[i - lo] = 0;
    }
    setPhysBndryFlags(out, ilo, ihi, mbuff, level);
  }
  void griddomup(const std::vector<signed char>& c, int ilo, int ihi, int mbuff, int lev, int ilofine, int ihifine, std::vector<signed char>& f) {
    const int lr = intratx[lev], clo = ilo - mbuff, flo = ilofine - mbuff;
    f.assign(ihifine - ilofine + 1 + 2 * mbuff, 0);
    auto C = [&](int i) -> signed char {
      if (i - clo < 0 || i - clo >= (int)c.size()) throw std::runtime_error("griddomup: coarse index out of range");
      return c[i - clo];
    };
    for (int i = ilo; i <= ihi; ++i) {
      const int ifine = i * lr - 1;
      for (int mi = 1; mi <= lr; ++mi) f[std::max(std::min(ifine + mi, ihifine + mbuff), ilofine - mbuff) - flo] = C(i);
    }
    for (int i = ihifine + 1; i <= ihifine + mbuff; ++i) f[i - flo] = C(i / lr);
    for (int i = ilofine - mbuff; i <= ilofine - 1; ++i) f[i - flo] = C(i / lr);
  }
  void setdomflags(Node& g, int mbuff, int lbase, int lcheck) {
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
    const int ist[3] = {ilo_c - mbuff, 0, iregsz[lbase]}, iend[3] = {-1, iregsz[lbase] - 1, ihi_c + mbuff};
    const int ish[3] = {iregsz[lbase], 0, -iregsz[lbase]};
    for (int mb = lstart[lbase]; mb != 0; mb = node[mb].levelptr) {
      const int iblo = node[mb].ilo, ibhi = node[mb].ihi;
      if (xperdom) {
        for (int k = 0; k < 3; ++k) {
          const int i1 = std::max(ilo_c - mbuff, ist[k]), i2 = std::min(ihi_c + mbuff, iend[k]);
          if (!(i1 <= i2)) continue;
          const int ixlo = std::max(iblo, i1 + ish[k]), ixhi = std::min(ibhi, i2 + ish[k]);
          for (int i = ixlo - ish[k]; i <= ixhi - ish[k]; ++i) flags[i - lo] = 1;
        }
      } else {
        for (int i = std::max(iblo, ilo_c - mbuff); i <= std::min(ibhi, ihi_c + mbuff); ++i) flags[i - lo] = 1;
      }
    }
    setPhysBndryFlags(flags, ilo_c, ihi_c, mbuff, lbase);
    std::vector<signed char> icopy = flags;
    griddomshrink(icopy, ilo_c, ihi_c, mbuff, g.dom2, lbase);
    for (int lev = lbase + 1; lev <= lcheck; ++lev) {
      griddomup(g.dom2, ilo_c, ihi_c, mbuff, lev - 1, igridst[lev], igridend[lev], icopy);
      griddomshrink(icopy, igridst[lev], igridend[lev], mbuff, g.dom2, lev);
      ilo_c = igridst[lev]; ihi_c = igridend[lev];
    }
  }
  int bufnst1(int lcheck, int lbase) {
    int numbad = 0;
    const int mbuff = std::max(nghost, ibuff + 1);
    for (int mptr : levelgrids[lcheck]) {
      Node& g = node[mptr];
      if (lcheck + 2 <= mxnest) projec1(lcheck, g, mbuff);
      shiftset(g, mbuff);
      int n = 0;
      for (double f : g.flags) if (f > DONTFLAG1) ++n;
      g.numflags = n;
      numbad += n;
      setdomflags(g, mbuff, lbase, lcheck);
    }
    return numbad;
  }
  void colate1(std::vector<double>& bp, int lcheck) {
    const int mbuff = std::max(nghost, ibuff + 1);
    bp.clear();
    for (int mptr : levelgrids[lcheck]) {
      Node& g = node[mptr];
      if (g.numflags != 0) {
        int imin = g.ilo - mbuff, imax = g.ihi + mbuff;
        if (!xperdom) { imin = std::max(imin, 0); imax = std::min(g.ihi + mbuff, iregsz[lcheck] - 1); }
        const int lo = g.ilo - mbuff;
        for (int i = imin; i <= imax; ++i) if (g.flags[i - lo] > DONTFLAG1 && g.dom2[i - lo] != 1) g.flags[i - lo] = 0.;
        for (int i = imin; i <= imax; ++i) {
          if (g.flags[i - lo] < 0 || g.flags[i - lo] <= DONTFLAG1) continue;
          int iwrap = i;
          if (xperdom) { if (i < 0) iwrap = i + iregsz[lcheck]; if (i >= iregsz[lcheck]) iwrap = i - iregsz[lcheck]; }
          bp.push_back((double)iwrap + .5);
        }
      }
      g.flags.clear(); g.dom2.clear();
    }
    if (lcheck >= 6) return;
    const int npts = (int)bp.size(), isize = iregsz[lcheck];
    std::vector<long long> iflags(npts + 1);
    std::vector<int> ix(npts + 1);
    for (int k = 1; k <= npts; ++k) iflags[k] = (int)(bp[k - 1] - .5) + mbuff;
    qsorti(ix, npts, iflags);
    std::vector<double> out;
    for (int k = 1; k <= npts;) {
      out.push_back((double)(iflags[ix[k]] % (isize + 2 * mbuff)) + .5 - mbuff);
      k = k + 1;
      while (k <= npts && iflags[ix[k]] == iflags[ix[k - 1]]) k = k + 1;
    }
    bp = out;
  }

  // ================================================================ clustering
  static void moment(int rect[2], const double* bp, int npt, double& usage) {
    double emx1 = bp[0], emn1 = emx1;
    for (int k = 0; k < npt; ++k) { if (bp[k] > emx1) emx1 = bp[k]; if (bp[k] < emn1) emn1 = bp[k]; }
    rect[0] = (int)std::lround(emn1 - .5);
    rect[1] = (int)std::lround(emx1 - .5);
    usage = (double)npt / (double)(rect[1] - rect[0] + 1);
  }
  // signs.f + findcut.f on the points [ist, iend)
  static int findcut(const double* bp, int ist, int iend, int idim) {
    std::vector<int> iscr(idim + 2, 0);
    int ilo = 1, ihi = idim;
    for (int k = ist; k < iend; ++k) iscr[(int)(bp[k] + 1.1)] += 1;
    for (int k = 1; k <= idim; ++k) if (iscr[k] != 0) { ilo = k; break; }
    for (int k = 1; k <= idim; ++k) if (iscr[idim + 1 - k] != 0) { ihi = idim + 1 - k; break; }
    for (int i = ilo; i <= ihi; ++i) if (iscr[i] == 0) return i;
    int ipre = iscr[ilo];
    for (int i = ilo + 1; i <= ihi - 1; ++i) { const int icur = iscr[i]; iscr[i] = iscr[i + 1] - 2 * icur + ipre; ipre = icur; }
    int locmaxi = 0, indexi = 0;
    const int imid = (ilo + ihi) / 2;
    for (int i = ilo + 2; i <= ihi - 1; ++i) {
      const int t1 = iscr[i - 1], t2 = iscr[i], d = std::abs(t1 - t2);
      if (t1 * t2 < 0) {
        if (d > locmaxi) { locmaxi = d; indexi = i; }
        else if (d == locmaxi && std::abs(i - imid) < std::abs(indexi - imid)) indexi = i;
      }
    }
    return locmaxi < 2 ? 0 : indexi;
  }
  void smartbis(std::vector<double>& bp, int npts, std::vector<int>& numptc, int& nclust, int idim) {
    nclust = 1;
    numptc.assign(1, npts);
    int icl = 0, ist = 0, iend = npts;
    while (true) {
      int rect[2]; double usenew;
      moment(rect, bp.data() + ist, numptc[icl], usenew);
      int index = usenew >= cut ? 0 : findcut(bp.data(), ist, iend, idim);
      if (usenew >= cut || index == 0) {
        if (++icl >= nclust) break;
        ist = iend; iend = ist + numptc[icl];
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
  bool baseCheck(int mnew, int lbase, int ilo, int ihi, int thisBuff) {
    const int levnew = node[mnew].level;
    const bool borderx = ilo == 0 || ihi == iregsz[levnew] - 1;
    int iclo = ilo, ichi = ihi;
    for (int lev = levnew - 1; lev >= lbase; --lev) { iclo = iclo / intratx[lev] - 1; ichi = ichi / intratx[lev] + 1; }
    if (!(xperdom && borderx)) { iclo = std::max(iclo, 0); ichi = std::min(ichi, iregsz[lbase] - 1); }
    std::vector<double> a(ichi - iclo + 1, 0.0);
    auto A = [&](int i) -> double& { return a[i - iclo]; };
    if (ilo == 0 && !xperdom) { A(iclo) = 1.; A(iclo + 1) = 1.; }
    if (ihi == iregsz[levnew] - 1 && !xperdom) { A(ichi) = 1.; A(ichi - 1) = 1.; }
    for (int mptr = lstart[lbase]; mptr != 0; mptr = node[mptr].levelptr) {
      const int iblo = node[mptr].ilo - thisBuff, ibhi = node[mptr].ihi + thisBuff;
      if (!(xperdom && borderx)) {
        for (int i = std::max(iclo, iblo); i <= std::min(ichi, ibhi); ++i) A(i) = 1.;
        continue;
      }
      const int ist[3] = {iclo, 0, iregsz[lbase]}, iend[3] = {-1, iregsz[lbase] - 1, ichi}, ish[3] = {iregsz[lbase], 0, -iregsz[lbase]};
      for (int k = 0; k < 3; ++k) {
        const int i1 = std::max(iclo, ist[k]), i2 = std::min(ichi, iend[k]);
        if (!(i1 <= i2)) continue;
        for (int i = std::max(i1 + ish[k], iblo); i <= std::min(i2 + ish[k], ibhi); ++i) A(i - ish[k]) = 1.;
      }
    }
    for (int i = iclo; i <= ichi; ++i) if (A(i) == 0) return false;
    return true;
  }
  bool nestck1(int mnew, int lbase, double* bp, int npts, std::vector<int>& numptc, int icl, int& nclust) {
    if (lbase == 1) return true;
    const int lratiox = intratx[node[mnew].level - 1];
    if (baseCheck(mnew, lbase, node[mnew].ilo, node[mnew].ihi, 0)) return true;
    if (npts <= 1) throw std::runtime_error("nestck1: a cluster of one point is not nested");
    const double rmid = ((node[mnew].ihi + node[mnew].ilo + 1) / 2.) / lratiox;
    int ipt = 0, ntop = npts - 1;
    while (true) {
      if (bp[ipt] < rmid) {
        if (++ipt <= ntop) continue;
        break;
      }
      std::swap(bp[ipt], bp[ntop]);
      if (ipt <= --ntop) continue;
      break;
    }
    numptc.insert(numptc.begin() + icl + 1, npts - (ntop + 1));
    numptc[icl] = ntop + 1;
    nclust = nclust + 1;
    return false;
  }
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
        Node& n = node[mnew];
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
  // filval.f90: old grids' values where they were, else interpolation from the coarse level
  void filval(int mptr, int level) {
    Node& g = node[mptr];
    const int r = intratx[level - 1];
    const double dx = hxposs[level], dxc = dx * r;
    const int iclo = g.ilo / r - 1, ichi = (g.ihi + 1) / r - 1 + 1;
    const int mic = (g.ihi - g.ilo + 1) / r + 2, mitot = mitot_of(mptr);
    const long long valc = palloc((long long)nvar * mic);
    fill_value1_kernel<<<grid_for((long long)nvar * mic, 128), 128, 0, st>>>(pool.d, valc, nvar * mic, 0.0);
    ++nkernels;
    if (xperdom && (iclo < 0 || ichi >= iregsz[level - 1])) preicall(valc, mic, iclo, ichi, level - 1);
    else icall(valc, mic, iclo, ichi, level - 1, 1);
    launch_bc(valc, mic, dxc, g.xlo - dxc, g.xhi + dxc);
    fill_value1_kernel<<<grid_for(mitot, 128), 128, 0, st>>>(pool.d, g.q1, mitot, NEEDS_TO_BE_SET1);
    ++nkernels;
    if (xperdom && (g.ilo < 0 || g.ihi >= iregsz[level])) preicall(g.q1, mitot, g.ilo - nghost, g.ihi + nghost, level);
    else icall(g.q1, mitot, g.ilo - nghost, g.ihi + nghost, level, 1);
    const int n = (mic - 2) * r;
    filval1_kernel<<<grid_for(n, 128), 128, 0, st>>>(pool.d, g.q1, mitot, valc, mic, r, nvar, NEEDS_TO_BE_SET1);
    ++nkernels;
    pfree(valc, (long long)nvar * mic);
  }
  void gfixup(int lbase, int lfnew) {
    putsp(lbase, lbase);
    for (int level = lbase + 1; level <= lfine; ++level) {
      putsp(lbase, level);
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) { if (node[m].q2 >= 0) pfree(node[m].q2, qsize(m)); node[m].q2 = -1; }
    }
    for (int lcheck = lbase + 1; lcheck <= mxnest; ++lcheck) {
      std::vector<int> nl;
      for (int m = newstl[lcheck]; m != 0; m = node[m].levelptr) nl.push_back(m);
      for (int m : nl) {
        node[m].q1 = palloc(qsize(m));
        AMR_CUDA(cudaMemsetAsync(pool.d + node[m].q1, 0, sizeof(double) * qsize(m), st));
      }
      for (int m : nl) filval(m, lcheck);
      int mptr = lstart[lcheck];
      while (mptr != 0) {
        const int mold = mptr;
        mptr = node[mptr].levelptr;
        pfree(node[mold].q1, qsize(mold));
        node[mold].q1 = -1;
        node[mold].bnd.clear();
        putnod(mold);
      }
      lstart[lcheck] = newstl[lcheck];
    }
    lfine = lfnew;
    for (int level = lbase + 1; level <= std::min(lfine, mxnest - 1); ++level)
      for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
        node[m].q2 = palloc(qsize(m));
        AMR_CUDA(cudaMemsetAsync(pool.d + node[m].q2, 0, sizeof(double) * qsize(m), st));
      }
  }
  void regrid(int lbase, double start_time) {
    int lcheck = std::min(lfine, mxnest - 1), lfnew = lbase;
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
      if (ng > 1) arrangeGrids(levnew, ng);
    }
    makeGridList(lbase);
    for (int levnew = lbase + 1; levnew <= lfine; ++levnew) makeBndryList(levnew);
  }

  // ================================================================ start-up
  void ginit(int msave, bool first, double start_time) {
    for (int mptr = msave; mptr != 0; mptr = node[mptr].levelptr) {
      Node& g = node[mptr];
      const int nxg = g.ihi - g.ilo + 1, mitot = nxg + 2 * nghost;
      if (first) {
        g.q1 = palloc(qsize(mptr));
        if (g.level < mxnest) g.q2 = palloc(qsize(mptr));
        g.time = start_time;
      }
      std::vector<double> q((size_t)qsize(mptr), 0.0);
      qinit(nxg, g.xlo, hxposs[g.level], q, mitot);
      AMR_CUDA(cudaMemcpyAsync(pool.d + (first ? g.q1 : g.q2), q.data(), sizeof(double) * q.size(), cudaMemcpyHostToDevice, st));
      if (first && g.q2 >= 0) AMR_CUDA(cudaMemsetAsync(pool.d + g.q2, 0, sizeof(double) * q.size(), st));
      AMR_CUDA(cudaStreamSynchronize(st));
    }
  }
  void domain(double start_time) {
    const int m0 = nodget();
    Node& g = node[m0];
    g.xlo = xlower; g.xhi = xupper; g.level = 1; g.ilo = 0; g.ihi = nx - 1;
    lstart[1] = m0;
    lfine = 1;
    birect(m0);
    ginit(m0, true, start_time);
    int ng = 0;
    for (int m = lstart[1]; m != 0; m = node[m].levelptr) ++ng;
    if (ng > 1) arrangeGrids(1, ng);
    makeGridList(0);
    makeBndryList(1);
    iregsz[1] = nx;
    for (int level = 2; level <= mxnest; ++level) {
      iregsz[level] = iregsz[level - 1] * intratx[level - 1];
      possk[level] = possk[level - 1] / (double)kratio[level - 1];
    }
  }
  void setgrd(double start_time) {
    if (mxnest == 1) return;
    for (int levnew = 2; levnew <= mxnest; ++levnew) {
      const int levold = levnew - 1;
      if (lstart[levold] == 0) break;
      int lfnew = levold;
      grdfit(levold, levold, start_time, start_time);
      if (newstl[levnew] != 0) lfnew = levnew;
      ginit(newstl[levnew], true, start_time);
      lstart[levnew] = newstl[levnew];
      lfine = lfnew;
      ginit(lstart[levold], false, start_time);
      int ng = 0;
      for (int m = lstart[levnew]; m != 0; m = node[m].levelptr) ++ng;
      if (ng > 1) arrangeGrids(levnew, ng);
      makeGridList(levold);
      makeBndryList(levnew);
    }
    for (int lev = 1; !(lev == mxnest || lev > lfine); ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr) { std::swap(node[m].q1, node[m].q2); node[m].time = start_time; }
    for (int level = 1; level <= lfine - 1; ++level) update(lfine - level);
    for (int level = 1; level <= lfine - 1; ++level) { prepf(level + 1); prepc(level); }
  }

  // ================================================================ gauges, mass, output
  void setbestsrc() {
    mbestsrc.assign(gauges.size(), 0);
    for (int lev = 1; lev <= lfine; ++lev)
      for (int m = lstart[lev]; m != 0; m = node[m].levelptr)
        for (size_t i = 0; i < gauges.size(); ++i)
          if (gauges[i].x >= node[m].xlo && gauges[i].x <= node[m].xhi) mbestsrc[i] = m;
  }
  double mass(int level = 1) {
    std::vector<Mass1> g;
    for (int m = lstart[level]; m != 0; m = node[m].levelptr) g.push_back(Mass1{node[m].q1, mitot_of(m)});
    d_massg.upload(g, st, stg);
    mass1_kernel<<<1, 1, 0, st>>>(pool.d, d_massg.d, (int)g.size(), hxposs[level], d_mass);
    ++nkernels;
    double v = 0;
    AMR_CUDA(cudaMemcpyAsync(&v, d_mass, sizeof(double), cudaMemcpyDeviceToHost, st));
    AMR_CUDA(cudaStreamSynchronize(st));
    stg.reset();
    return v;
  }
  std::vector<double> grid_values(int m) {
    std::vector<double> v((size_t)qsize(m));
    AMR_CUDA(cudaMemcpyAsync(v.data(), pool.d + node[m].q1, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, st));
    AMR_CUDA(cudaStreamSynchronize(st));
    return v;
  }
  void valout(double t) {
    const bool binary = output_format == 3;
    if (!binary)
      for (int level = 1; level <= lfine; ++level)
        for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
          zero_tiny1_kernel<<<grid_for(qsize(m), 128), 128, 0, st>>>(pool.d, node[m].q1, mitot_of(m), nvar);
          ++nkernels;
        }
    if (write_output) {
      FILE* f = open_output(outdir, "fort.q", matlabu);
      FILE* b = binary ? open_output(outdir, "fort.b", matlabu, "wb") : nullptr;
      std::vector<double> all;
      int ngrids = 0;
      for (int level = 1; level <= lfine; ++level)
        for (int m = lstart[level]; m != 0; m = node[m].levelptr) {
          ++ngrids;
          const int mx = node[m].ihi - node[m].ilo + 1, mitot = mitot_of(m);
          write_grid_header(f, 1, m, level, &mx, &node[m].xlo, &hxposs[level]);
          const std::vector<double> v = grid_values(m);
          if (binary) {
            for (int i = 1; i <= mitot; ++i) for (int iv = 0; iv < nvar; ++iv) all.push_back(v[(size_t)iv * mitot + i - 1]);
          } else {
            for (int i = nghost + 1; i <= mitot - nghost; ++i) {
              for (int iv = 0; iv < nvar; ++iv) std::fputs(fort_e(v[(size_t)iv * mitot + i - 1], 26, 16).c_str(), f);
              std::fputc('\n', f);
            }
            std::fputs("  \n", f);
          }
        }
      if (std::fclose(f) != 0) throw std::runtime_error("cannot write fort.q in " + outdir);
      if (b) write_raw(b, all, outdir);
      write_fort_t(outdir, matlabu, t, nvar, ngrids, 0, 1, nghost);
    }
    matlabu = matlabu + 1;
  }

  // ================================================================ tick.f
  bool finished() const { return ncycle >= nstop || time >= tfinal; }
  void tick(double start_time) {
    double dtnew[12];
    double* tlevel = tk_tlevel;
    int ntogo[12];
    int cycles = 0;
    setbestsrc();
    int nextout = 0;
    if (iout == 0) { iout = IINFINITY1; nextout = nout > 0 ? 1 : 0; }
    if (tick_started) nextout = tk_nextout;
    if (!tick_started) for (int i = 1; i <= mxnest; ++i) tlevel[i] = time;
    tick_started = true;
    const auto w0 = std::chrono::steady_clock::now();
    const double rv0 = rvol;
    while (!finished()) {
      const double outtime = nout > 0 ? ((nextout <= nout) ? tout[nextout - 1] : RINFINITY1) : tfinal;
      bool dumpout = false;
      if (time < outtime && time + (double)1.001f * possk[1] >= outtime) {
        possk[1] = outtime - time;
        for (int i = 2; i <= mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
        if (nout > 0) { nextout = nextout + 1; dumpout = true; }
      }
      int level = 1;
      ntogo[level] = 1;
      for (int i = 1; i <= 10; ++i) dtnew[i] = RINFINITY1;
      while (true) {
        int lbase = -1;
        if (icheck[level] >= kcheck) lbase = level;
        else if (level + 1 >= mxnest) lbase = -1;
        else if (icheck[level + 1] >= kcheck) lbase = level + 1;
        else if (level + 2 >= mxnest) lbase = -1;
        else if (icheck[level + 2] >= kcheck) lbase = level + 2;
        if (lbase > 0) {
          if (!(lbase == mxnest || lbase > lfine)) {
            const auto r0 = std::chrono::steady_clock::now();
            regrid(lbase, start_time);
            setbestsrc();
            t_regrid += std::chrono::duration<double>(std::chrono::steady_clock::now() - r0).count();
          }
          for (int i = lbase; i <= lfine; ++i) icheck[i] = 0;
          for (int i = lbase + 1; i <= lfine; ++i) tlevel[i] = tlevel[lbase];
        }
        cfl_level = 0.0;
        const double dtlevnew = advanc(level);
        ntogo[level] = ntogo[level] - 1;
        dtnew[level] = std::min(dtnew[level], dtlevnew);
        tlevel[level] = tlevel[level] + possk[level];
        icheck[level] = icheck[level] + 1;
        if (level < lfine) {
          level = level + 1;
          if (((possk[level - 1] - dtnew[level - 1]) / dtnew[level - 1]) > (double)0.05f)
            ntogo[level] = (int)((tlevel[level - 1] - tlevel[level]) / (dtnew[level - 1] / kratio[level - 1]) + (double)0.9f);
          else
            ntogo[level] = kratio[level - 1];
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
      if (vtime) {
        for (int i = 2; i <= lfine; ++i) { const int ii = lfine + 1 - i; dtnew[ii] = std::min(dtnew[ii], dtnew[ii + 1] * kratio[ii]); }
        dtnew[1] = std::min(dtnew[1], dt_max);
        possk[1] = dtnew[1];
        for (int i = 2; i <= mxnest; ++i) possk[i] = possk[i - 1] / kratio[i - 1];
      }
      if ((ncycle % iout == 0) || dumpout) valout(time);
      ++cycles;
      if (max_cycles > 0 && cycles >= max_cycles) break;
    }
    AMR_CUDA(cudaStreamSynchronize(st));
    tk_nextout = nextout;
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    t_step += sec;
    last_run_ms = 1e3 * sec;
    run_cells = rvol - rv0;
  }

  void init(const std::string& dir) {
    read_input(dir);
    AMR_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    AllocStreamScope alloc_scope(st);
    pool.init(1 << 20);
    regs.init(1 << 16);
    AMR_CUDA(cudaMalloc(&d_cfl, 2 * sizeof(unsigned long long)));
    AMR_CUDA(cudaMallocHost((void**)&h_cfl, sizeof(unsigned long long)));
    AMR_CUDA(cudaMalloc(&d_mass, sizeof(double)));
    hxposs[1] = (xupper - xlower) / nx;
    matlabu = output_t0 ? 0 : 1;
    node.assign(2, Node());
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
    tmass0 = mass(1);
    if (output_t0) valout(time);
    AMR_CUDA(cudaStreamSynchronize(st));
  }
};

// The 1D solver behind the C ABI's solver interface.
class Solver1 : public AmrSolver {
 public:
  Amr1Gpu g;
  int num_dim() const override { return 1; }
  cudaStream_t stream() const override { return g.st; }
  void set_batched(bool) override {}
  void set_profile(bool) override {}
  void set_graphs(bool on) override {
    if (on) throw std::invalid_argument("amrgpu_set_graphs: graph replay is built for the 3D path");
  }
  void set_schedule(int s) override {
    if (s != 0) throw std::invalid_argument("amrgpu_set_schedule: sweep schedules are built for the 3D path");
  }
  void set_solver(const std::string& name, const std::vector<double>& v) override {
    Prob1 P = g.prob;
    if (name == "advection") {
      if (v.size() != 1 || g.nvar != 1) throw std::invalid_argument("advection (1D) takes 1 constant (u) and num_eqn = 1");
      P.solver = SOLVER1_ADVECTION; P.u = v[0];
    } else if (name == "acoustics") {
      if (v.size() != 2 || g.nvar != 2) throw std::invalid_argument("acoustics (1D) takes 2 constants (rho, bulk) and num_eqn = 2");
      if (!(v[0] > 0) || !(v[1] > 0)) throw std::invalid_argument("acoustics: rho and bulk must be positive");
      P.solver = SOLVER1_ACOUSTICS; P.rho = v[0]; P.bulk = v[1]; P.cc = std::sqrt(P.bulk / P.rho); P.zz = P.cc * P.rho;
    } else if (name == "euler_roe_efix") {
      if (v.size() != 1 || g.nvar != 3) throw std::invalid_argument("euler_roe_efix (1D) takes 1 constant (gamma) and num_eqn = 3");
      if (!(v[0] > 1)) throw std::invalid_argument("euler_roe_efix: gamma must exceed 1");
      P.solver = SOLVER1_EULER; P.gamma = v[0]; P.gamma1 = v[0] - 1.0;
    } else {
      throw std::invalid_argument("unknown 1D Riemann solver '" + name + "' (advection, acoustics, euler_roe_efix)");
    }
    g.prob = P;
  }
  void set_pool_limit(long long bytes) override { set_arena_limits(g.pool, g.regs, bytes); }
  void set_step_batching(int window_us) override {
    if (window_us != 0) throw std::invalid_argument("amrgpu_set_step_batching: cross-request batching is built for the 2D path");
  }
  void run(int mc) override {
    AllocStreamScope alloc_scope(g.st);
    g.max_cycles = mc;
    g.tick(g.t0);
  }
  double level_advance(int level, double* cfl) override {
    if (level < 1 || level > g.lfine) throw std::invalid_argument("amrgpu_level_advance: no such level");
    AllocStreamScope alloc_scope(g.st);
    g.cfl_level = 0.0;
    const double dt = g.advanc(level);
    if (cfl) *cfl = g.cfl_level;
    return dt;
  }
  void update_level(int level) override {
    if (level < 1 || level >= g.lfine) throw std::invalid_argument("amrgpu_update: level must have a finer level");
    AllocStreamScope alloc_scope(g.st);
    g.update(level);
    AMR_CUDA(cudaStreamSynchronize(g.st));
  }
  void regrid_from(int lbase) override {
    if (lbase < 1 || lbase > g.lfine) throw std::invalid_argument("amrgpu_regrid: no such level");
    AllocStreamScope alloc_scope(g.st);
    g.regrid(lbase, g.t0);
    g.setbestsrc();
    AMR_CUDA(cudaStreamSynchronize(g.st));
  }
  void valout(const char* dir) override {
    const std::string keep = g.outdir;
    const bool kw = g.write_output;
    if (dir) { g.outdir = dir; g.write_output = true; }
    g.valout(g.time);
    g.outdir = keep; g.write_output = kw;
  }
  void write_checkpoint(const char*) override {
    throw std::invalid_argument("amrgpu_checkpoint: checkpoints are built for the 2D and 3D paths");
  }
  double mass() override { return g.mass(1); }
  std::vector<double> info() override {
    return {g.time, g.rvol, (double)g.ncycle, (double)g.lfine, g.t_step, g.t_regrid, g.tmass0, g.cflmax_run, (double)g.nkernels,
            (double)g.pool.peak * 8.0, 0.0, 0.0, 0.0, g.last_run_ms, g.run_cells, g.finished() ? 1.0 : 0.0, 0.0,
            0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 64.0, 0.0, 0.0, 0.0, 0.0, 8.0 * (double)(g.pool.cap + g.regs.cap)};
  }
  std::vector<int> grid_rows() override {
    std::vector<int> r;
    for (int lev = 1; lev <= g.lfine; ++lev)
      for (int m = g.lstart[lev]; m != 0; m = g.node[m].levelptr) r.insert(r.end(), {m, lev, g.node[m].ilo, g.node[m].ihi});
    return r;
  }
  long long value_count() override {
    long long n = 0;
    for (int lev = 1; lev <= g.lfine; ++lev)
      for (int m = g.lstart[lev]; m != 0; m = g.node[m].levelptr) n += (long long)g.nvar * (g.mitot_of(m) - 2 * g.nghost);
    return n;
  }
  std::vector<double> values() override {
    std::vector<double> out;
    for (int lev = 1; lev <= g.lfine; ++lev)
      for (int m = g.lstart[lev]; m != 0; m = g.node[m].levelptr) {
        const std::vector<double> v = g.grid_values(m);
        const int mitot = g.mitot_of(m);
        for (int iv = 0; iv < g.nvar; ++iv)
          for (int i = g.nghost + 1; i <= mitot - g.nghost; ++i) out.push_back(v[(size_t)iv * mitot + i - 1]);
      }
    return out;
  }
  std::vector<double> gauge_rows() override {
    const int nv = g.nvar;
    std::vector<double> vals((size_t)g.gslots * nv), out;
    if (g.gslots) {
      AMR_CUDA(cudaMemcpyAsync(vals.data(), g.d_gauge.d, sizeof(double) * vals.size(), cudaMemcpyDeviceToHost, g.st));
      AMR_CUDA(cudaStreamSynchronize(g.st));
    }
    for (const auto& G : g.gauges)
      for (const auto& r : g.grows) {
        if (r.gauge != G.num) continue;
        out.push_back(r.gauge); out.push_back(r.level); out.push_back(r.t);
        for (int k = 0; k < nv; ++k) out.push_back(vals[(size_t)r.slot * nv + k]);
      }
    return out;
  }
};

AmrSolver* make_solver1(const std::string& rundir, const std::string& outdir, bool write_output) {
  std::unique_ptr<Solver1> s(new Solver1());
  s->g.outdir = outdir;
  s->g.write_output = write_output;
  s->g.init(rundir);
  return s.release();
}

}  // namespace amrb
