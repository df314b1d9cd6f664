// Device Riemann solvers for the 2D patch step, one interface per call.
//
// These replace the reference's rpn2/rpt2 plugin interface
// (calls at src/2d/flux2.f:125-126, 202-204, 219-221 and src/2d/qad.f:129-130)
// with per-interface device functions that take the state left of the
// interface (cell i-1, the reference's qr(:,i-1)) and right of it (cell i, the
// reference's ql(:,i)). The solvers themselves are not in the reference (they
// come from the un-vendored clawpack/riemann); they are written from the
// published mathematics:
//   advection   constant-velocity upwinding (LeVeque, FVMHP 2002, ch. 20.5)
//   acoustics   constant-coefficient characteristic decomposition (FVMHP 3.8, 21.5)
//   euler       Roe solver, 4 waves, Harten-Hyman entropy fix (FVMHP 15.3);
//               transverse Roe splitting (FVMHP 21.6)
//   vc_advection  advection in a face-centred velocity field: aux(1) = u at the left
//               face, aux(2) = v at the bottom face of each cell (FVMHP 9.5, 20.8)
// Arithmetic is written in a fixed evaluation order so that, built without
// FMA contraction, results are bit-identical to the CPU oracle.
#pragma once
#include "common.cuh"
#include "../../include/amrgpu_riemann.cuh"

namespace amrb {

enum SolverKind { SOLVER_ADVECTION = 1, SOLVER_ACOUSTICS = 2, SOLVER_EULER = 3, SOLVER_VC_ADVECTION = 4 };

constexpr int MAXAUX2 = 3;  // aux components a 2D run may carry (the staged aux tile)
enum AuxType { AUX_CENTER = 0, AUX_XLEFT = 1, AUX_YLEFT = 2, AUX_CAPACITY = 3 };

struct ProbDev {
  int solver;
  int efix;
  double ubar, vbar, wbar;
  double rho, bulk, cc, zz;
  double gamma, gamma1;
  int naux;                 // aux components of the run (0..MAXAUX2)
  int auxtype[MAXAUX2];     // amr.data aux_type codes (qad.f picks face values by them)
};

// std::min / std::max semantics (first argument on ties), including signed zeros.
template <class R> __host__ __device__ __forceinline__ R dmin(R a, R b) { return (b < a) ? b : a; }
template <class R> __host__ __device__ __forceinline__ R dmax(R a, R b) { return (a < b) ? b : a; }
template <class R> __host__ __device__ __forceinline__ R dsign(R a, R b) { return b >= R(0) ? fabs(a) : -fabs(a); }

// ---------------------------------------------------------------- advection
struct Advection2 {
  static constexpr int MEQN = 1, MWAVES = 1, NAUX = 0;
  template <class R>
  __device__ static void rpn(const ProbDev& P, int ixy, const R* qL, const R* qR, const R*, const R*,
                             R (&wave)[MWAVES][MEQN], R (&s)[MWAVES], R (&amdq)[MEQN], R (&apdq)[MEQN]) {
    wave[0][0] = qR[0] - qL[0];
    s[0] = (ixy == 1) ? R(P.ubar) : R(P.vbar);
    amdq[0] = dmin(s[0], R(0)) * wave[0][0];
    apdq[0] = dmax(s[0], R(0)) * wave[0][0];
  }
  template <class R>
  __device__ static void rpt(const ProbDev& P, int ixy, int imp, const R* qL, const R* qR, const R*, const R*,
                             const R*, const R* asdq, R (&bm)[MEQN], R (&bp)[MEQN]) {
    const R st = (ixy == 1) ? R(P.vbar) : R(P.ubar);
    bm[0] = dmin(st, R(0)) * asdq[0];
    bp[0] = dmax(st, R(0)) * asdq[0];
  }
};

// ---------------------------------------------------------------- acoustics
struct Acoustics2 {
  static constexpr int MEQN = 3, MWAVES = 2, NAUX = 0;
  template <class R>
  __device__ static void rpn(const ProbDev& P, int ixy, const R* qL, const R* qR, const R*, const R*,
                             R (&wave)[MWAVES][MEQN], R (&s)[MWAVES], R (&amdq)[MEQN], R (&apdq)[MEQN]) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    const R zz = R(P.zz), cc = R(P.cc);
    const R d1 = qR[0] - qL[0];
    const R d2 = qR[mu] - qL[mu];
    const R a1 = (-d1 + zz * d2) / (R(2) * zz);
    const R a2 = (d1 + zz * d2) / (R(2) * zz);
    wave[0][0] = -a1 * zz; wave[0][mu] = a1; wave[0][mv] = R(0); s[0] = -cc;
    wave[1][0] = a2 * zz; wave[1][mu] = a2; wave[1][mv] = R(0); s[1] = cc;
#pragma unroll
    for (int m = 0; m < MEQN; ++m) {
      R am = R(0), ap = R(0);
#pragma unroll
      for (int mw = 0; mw < MWAVES; ++mw) {
        if (s[mw] < R(0)) am = am + s[mw] * wave[mw][m];
        else ap = ap + s[mw] * wave[mw][m];
      }
      amdq[m] = am; apdq[m] = ap;
    }
  }
  template <class R>
  __device__ static void rpt(const ProbDev& P, int ixy, int imp, const R* qL, const R* qR, const R*, const R*,
                             const R*, const R* asdq, R (&bm)[MEQN], R (&bp)[MEQN]) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    const R zz = R(P.zz), cc = R(P.cc);
    const R a1 = (-asdq[0] + zz * asdq[mv]) / (R(2) * zz);
    const R a2 = (asdq[0] + zz * asdq[mv]) / (R(2) * zz);
    bm[0] = cc * a1 * zz; bm[mu] = R(0); bm[mv] = -cc * a1;
    bp[0] = cc * a2 * zz; bp[mu] = R(0); bp[mv] = cc * a2;
  }
};

// ---------------------------------------------------------------- euler (Roe)
struct Euler2 {
  static constexpr int MEQN = 4, MWAVES = 4, NAUX = 0;
  template <class R>
  __device__ static void rpn(const ProbDev& P, int ixy, const R* qL, const R* qR, const R*, const R*,
                             R (&wave)[MWAVES][MEQN], R (&s)[MWAVES], R (&amdq)[MEQN], R (&apdq)[MEQN]) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    const R g1 = R(P.gamma1), gam = R(P.gamma);
    const R rl = qL[0], rr = qR[0];
    const R sql = sqrt(rl), sqr = sqrt(rr);
    const R pl = g1 * (qL[3] - R(0.5) * (qL[mu] * qL[mu] + qL[mv] * qL[mv]) / rl);
    const R pr = g1 * (qR[3] - R(0.5) * (qR[mu] * qR[mu] + qR[mv] * qR[mv]) / rr);
    const R rsum = sql + sqr;
    const R u = (qL[mu] / sql + qR[mu] / sqr) / rsum;
    const R v = (qL[mv] / sql + qR[mv] / sqr) / rsum;
    const R enth = ((qL[3] + pl) / sql + (qR[3] + pr) / sqr) / rsum;
    const R u2v2 = u * u + v * v;
    const R a2 = g1 * (enth - R(0.5) * u2v2);
    const R a = sqrt(a2);
    const R g1a2 = g1 / a2;
    const R euv = enth - u2v2;
    const R d1 = qR[0] - qL[0];
    const R d2 = qR[mu] - qL[mu];
    const R d3 = qR[mv] - qL[mv];
    const R d4 = qR[3] - qL[3];
    const R ae = g1a2 * (euv * d1 + u * d2 + v * d3 - d4);
    const R as = d3 - v * d1;
    const R a4 = (d2 + (a - u) * d1 - a * ae) / (R(2) * a);
    const R a1 = d1 - ae - a4;
    wave[0][0] = a1; wave[0][mu] = a1 * (u - a); wave[0][mv] = a1 * v; wave[0][3] = a1 * (enth - u * a); s[0] = u - a;
    wave[1][0] = ae; wave[1][mu] = ae * u; wave[1][mv] = ae * v; wave[1][3] = ae * R(0.5) * u2v2; s[1] = u;
    wave[2][0] = R(0); wave[2][mu] = R(0); wave[2][mv] = as; wave[2][3] = as * v; s[2] = u;
    wave[3][0] = a4; wave[3][mu] = a4 * (u + a); wave[3][mv] = a4 * v; wave[3][3] = a4 * (enth + u * a); s[3] = u + a;
    R df[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      R t = R(0);
#pragma unroll
      for (int mw = 0; mw < 4; ++mw) t = t + s[mw] * wave[mw][m];
      df[m] = t;
    }
    bool fixed = false;
    if (P.efix) {
      const R cl = sqrt(gam * pl / rl);
      const R sl = qL[mu] / rl - cl;
      if (sl < R(0) && s[0] > R(0)) {
        const R r1 = qL[0] + wave[0][0];
        const R ru1 = qL[mu] + wave[0][mu];
        const R rv1 = qL[mv] + wave[0][mv];
        const R e1 = qL[3] + wave[0][3];
        const R p1 = g1 * (e1 - R(0.5) * (ru1 * ru1 + rv1 * rv1) / r1);
        const R c1 = sqrt(gam * p1 / r1);
        const R sr = ru1 / r1 - c1;
        if (sr > R(0)) {
          const R sfract = sl * (sr - s[0]) / (sr - sl);
#pragma unroll
          for (int m = 0; m < 4; ++m) { amdq[m] = sfract * wave[0][m]; apdq[m] = df[m] - amdq[m]; }
          fixed = true;
        }
      }
      if (!fixed) {
        const R cr = sqrt(gam * pr / rr);
        const R sr = qR[mu] / rr + cr;
        if (s[3] < R(0) && sr > R(0)) {
          const R r3 = qR[0] - wave[3][0];
          const R ru3 = qR[mu] - wave[3][mu];
          const R rv3 = qR[mv] - wave[3][mv];
          const R e3 = qR[3] - wave[3][3];
          const R p3 = g1 * (e3 - R(0.5) * (ru3 * ru3 + rv3 * rv3) / r3);
          const R c3 = sqrt(gam * p3 / r3);
          const R sl3 = ru3 / r3 + c3;
          if (sl3 < R(0)) {
            const R sfract = sr * (s[3] - sl3) / (sr - sl3);
#pragma unroll
            for (int m = 0; m < 4; ++m) { apdq[m] = sfract * wave[3][m]; amdq[m] = df[m] - apdq[m]; }
            fixed = true;
          }
        }
      }
    }
    if (!fixed) {
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        R am = R(0);
#pragma unroll
        for (int mw = 0; mw < 4; ++mw)
          if (s[mw] < R(0)) am = am + s[mw] * wave[mw][m];
        amdq[m] = am;
        apdq[m] = df[m] - am;
      }
    }
  }
  template <class R>
  __device__ static void rpt(const ProbDev& P, int ixy, int imp, const R* qL, const R* qR, const R*, const R*,
                             const R*, const R* asdq, R (&bm)[MEQN], R (&bp)[MEQN]) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    const R g1 = R(P.gamma1);
    const R rl = qL[0], rr = qR[0];
    const R sql = sqrt(rl), sqr = sqrt(rr);
    const R pl = g1 * (qL[3] - R(0.5) * (qL[mu] * qL[mu] + qL[mv] * qL[mv]) / rl);
    const R pr = g1 * (qR[3] - R(0.5) * (qR[mu] * qR[mu] + qR[mv] * qR[mv]) / rr);
    const R rsum = sql + sqr;
    const R u = (qL[mu] / sql + qR[mu] / sqr) / rsum;
    const R v = (qL[mv] / sql + qR[mv] / sqr) / rsum;
    const R enth = ((qL[3] + pl) / sql + (qR[3] + pr) / sqr) / rsum;
    const R u2v2 = u * u + v * v;
    const R a2 = g1 * (enth - R(0.5) * u2v2);
    const R a = sqrt(a2);
    const R g1a2 = g1 / a2;
    const R euv = enth - u2v2;
    const R d1 = asdq[0], dmu = asdq[mu], dmv = asdq[mv], d4 = asdq[3];
    const R ae = g1a2 * (euv * d1 + u * dmu + v * dmv - d4);
    const R as = dmu - u * d1;
    const R a4 = (dmv + (a - v) * d1 - a * ae) / (R(2) * a);
    const R a1 = d1 - ae - a4;
    R w[4][4], sp[4];
    w[0][0] = a1; w[0][mu] = a1 * u; w[0][mv] = a1 * (v - a); w[0][3] = a1 * (enth - v * a); sp[0] = v - a;
    w[1][0] = ae; w[1][mu] = ae * u; w[1][mv] = ae * v; w[1][3] = ae * R(0.5) * u2v2; sp[1] = v;
    w[2][0] = R(0); w[2][mu] = as; w[2][mv] = R(0); w[2][3] = as * u; sp[2] = v;
    w[3][0] = a4; w[3][mu] = a4 * u; w[3][mv] = a4 * (v + a); w[3][3] = a4 * (enth + v * a); sp[3] = v + a;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      R b_m = R(0), b_p = R(0);
#pragma unroll
      for (int mw = 0; mw < 4; ++mw) {
        b_m = b_m + dmin(sp[mw], R(0)) * w[mw][m];
        b_p = b_p + dmax(sp[mw], R(0)) * w[mw][m];
      }
      bm[m] = b_m; bp[m] = b_p;
    }
  }
};

// ---------------------------------------------------------------- vc_advection
// auxL / auxR: aux of the cells left and right of the interface (the reference's auxr(:,i-1)
// and auxl(:,i)); the normal speed is the right cell's own face velocity. rpt: aux1/aux2/aux3
// are the aux of the cell asdq belongs to in the rows below, at and above the sweep's row;
// the split moves asdq with that cell's transverse face velocities on its lower face
// (aux2) and on its upper face (aux3, the lower face of the cell above).
struct VcAdvection2 {
  static constexpr int MEQN = 1, MWAVES = 1, NAUX = 2;
  template <class R>
  __device__ static void rpn(const ProbDev&, int ixy, const R* qL, const R* qR, const R*, const R* auxR,
                             R (&wave)[MWAVES][MEQN], R (&s)[MWAVES], R (&amdq)[MEQN], R (&apdq)[MEQN]) {
    const R u = auxR[ixy - 1];
    wave[0][0] = qR[0] - qL[0];
    s[0] = u;
    amdq[0] = dmin(u, R(0)) * wave[0][0];
    apdq[0] = dmax(u, R(0)) * wave[0][0];
  }
  template <class R>
  __device__ static void rpt(const ProbDev&, int ixy, int, const R*, const R*, const R*, const R* aux2,
                             const R* aux3, const R* asdq, R (&bm)[MEQN], R (&bp)[MEQN]) {
    const int kv = 3 - ixy;
    bm[0] = dmin(aux2[kv - 1], R(0)) * asdq[0];
    bp[0] = dmax(aux3[kv - 1], R(0)) * asdq[0];
  }
};

// the registered 2D plugins satisfy the device plugin contract (include/amrgpu_riemann.cuh)
static_assert(amrgpu_plugin::Check2D<Advection2, ProbDev, double>::value, "advection: rpn2/rpt2 contract");
static_assert(amrgpu_plugin::Check2D<Acoustics2, ProbDev, double>::value, "acoustics: rpn2/rpt2 contract");
static_assert(amrgpu_plugin::Check2D<Euler2, ProbDev, double>::value, "euler_roe_efix: rpn2/rpt2 contract");
static_assert(amrgpu_plugin::Check2D<Euler2, ProbDev, float>::value, "euler_roe_efix (FP32): rpn2/rpt2 contract");
static_assert(amrgpu_plugin::Check2D<VcAdvection2, ProbDev, double>::value, "vc_advection: rpn2/rpt2 contract");

}  // namespace amrb
