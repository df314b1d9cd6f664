// Oracle (test infrastructure only): CPU Riemann solvers for the 2D oracle.
//
// The reference does not ship its Riemann solvers: every application Makefile
// pulls rpn2_*/rpt2_* from the separate clawpack/riemann repository
// (tests/advection_2d_square/Makefile:56-57, examples/euler_2d_quadrants/Makefile:55-56),
// which is not vendored and not version-pinned. These are restated from the
// published mathematics with the reference's calling convention:
//   rpn2(ixy,...,ql,qr,...)  the interface i sits between qr(:,i-1) and ql(:,i)
//                            (call site src/2d/flux2.f:125-126, qad.f:129-130)
//   rpt2(ixy,imp,...,asdq)   splits asdq into down/up-going parts
//                            (call sites src/2d/flux2.f:202-204, 219-221)
// Loops run over i = 2-mbc .. mx+mbc like the clawpack solvers.
//
//  * advection: constant velocity upwinding (LeVeque, FVMHP 2002, ch. 4 and 20.5).
//  * acoustics: characteristic decomposition of the constant-coefficient
//    acoustics system (FVMHP 2002, sections 3.8, 21.3 and 21.5).
//  * euler: Roe solver, 4 waves (two acoustic, entropy, shear), Harten-Hyman
//    entropy fix for transonic rarefactions; Roe-linearised transverse solver
//    (FVMHP 2002, sections 15.3.3-15.3.5, 19.3.3 and 21.6).
//  * vc_advection: advection in a face-centred velocity field, aux(1) = u at the
//    left face and aux(2) = v at the bottom face of each cell (the rpn2/rpt2 pair
//    tests/advection_2d_annulus/Makefile names); the normal speed is the interface's
//    own face velocity, a transverse split moves asdq with the transverse face
//    velocities of the cell it came from (FVMHP 2002, sections 9.5 and 20.8).
#pragma once
#include <cmath>
#include <algorithm>

namespace orc {

enum SolverKind { SOLVER_ADVECTION = 1, SOLVER_ACOUSTICS = 2, SOLVER_EULER = 3, SOLVER_VC_ADVECTION = 4 };

struct ProbParams {
  int solver = SOLVER_ADVECTION;
  double ubar = 0, vbar = 0, wbar = 0;       // advection
  double rho = 1, bulk = 1, cc = 1, zz = 1;  // acoustics
  double gamma = 1.4, gamma1 = 0.4;          // euler
  bool efix = true;
};

// Fortran-style 1-D slice accessor: a(m, i) with m = 1..meqn, i from 1-mbc.
struct Slice {
  double* p; int ld; int base;  // base = 1-mbc
  double& operator()(int m, int i) const { return p[(m - 1) + ld * (i - base)]; }
};
struct Waves {  // wave(m, mw, i)
  double* p; int meqn; int mwaves; int base;
  double& operator()(int m, int mw, int i) const {
    return p[(m - 1) + meqn * ((mw - 1) + mwaves * (i - base))];
  }
};

inline double dsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }

// ---------------------------------------------------------------- rpn2
inline void rpn2(const ProbParams& P, int ixy, int meqn, int mwaves, int mbc, int mx,
                 Slice ql, Slice qr, Slice auxl, Slice auxr, Waves wave, Slice s,
                 Slice amdq, Slice apdq) {
  (void)auxr;
  if (P.solver == SOLVER_VC_ADVECTION) {
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      wave(1, 1, i) = ql(1, i) - qr(1, i - 1);
      s(1, i) = auxl(ixy, i);
      amdq(1, i) = std::min(auxl(ixy, i), 0.0) * wave(1, 1, i);
      apdq(1, i) = std::max(auxl(ixy, i), 0.0) * wave(1, 1, i);
    }
    return;
  }
  if (P.solver == SOLVER_ADVECTION) {
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      wave(1, 1, i) = ql(1, i) - qr(1, i - 1);
      s(1, i) = (ixy == 1) ? P.ubar : P.vbar;
      amdq(1, i) = std::min(s(1, i), 0.0) * wave(1, 1, i);
      apdq(1, i) = std::max(s(1, i), 0.0) * wave(1, 1, i);
    }
    return;
  }
  if (P.solver == SOLVER_ACOUSTICS) {
    const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      const double d1 = ql(1, i) - qr(1, i - 1);
      const double d2 = ql(mu, i) - qr(mu, i - 1);
      const double a1 = (-d1 + P.zz * d2) / (2.0 * P.zz);
      const double a2 = (d1 + P.zz * d2) / (2.0 * P.zz);
      wave(1, 1, i) = -a1 * P.zz; wave(mu, 1, i) = a1; wave(mv, 1, i) = 0.0;
      s(1, i) = -P.cc;
      wave(1, 2, i) = a2 * P.zz; wave(mu, 2, i) = a2; wave(mv, 2, i) = 0.0;
      s(2, i) = P.cc;
    }
    for (int i = 2 - mbc; i <= mx + mbc; ++i)
      for (int m = 1; m <= meqn; ++m) {
        double am = 0.0, ap = 0.0;
        for (int mw = 1; mw <= mwaves; ++mw) {
          if (s(mw, i) < 0.0) am = am + s(mw, i) * wave(m, mw, i);
          else ap = ap + s(mw, i) * wave(m, mw, i);
        }
        amdq(m, i) = am; apdq(m, i) = ap;
      }
    return;
  }
  if (P.solver == SOLVER_EULER) {
    const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
    const double g1 = P.gamma1, gam = P.gamma;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      // Roe averages of the left state qr(:,i-1) and the right state ql(:,i)
      const double rl = qr(1, i - 1), rr = ql(1, i);
      const double sql = std::sqrt(rl), sqr = std::sqrt(rr);
      const double pl = g1 * (qr(4, i - 1) - 0.5 * (qr(mu, i - 1) * qr(mu, i - 1) + qr(mv, i - 1) * qr(mv, i - 1)) / rl);
      const double pr = g1 * (ql(4, i) - 0.5 * (ql(mu, i) * ql(mu, i) + ql(mv, i) * ql(mv, i)) / rr);
      const double rsum = sql + sqr;
      const double u = (qr(mu, i - 1) / sql + ql(mu, i) / sqr) / rsum;
      const double v = (qr(mv, i - 1) / sql + ql(mv, i) / sqr) / rsum;
      const double enth = ((qr(4, i - 1) + pl) / sql + (ql(4, i) + pr) / sqr) / rsum;
      const double u2v2 = u * u + v * v;
      const double a2 = g1 * (enth - 0.5 * u2v2);
      const double a = std::sqrt(a2);
      const double g1a2 = g1 / a2;
      const double euv = enth - u2v2;
      const double d1 = ql(1, i) - qr(1, i - 1);
      const double d2 = ql(mu, i) - qr(mu, i - 1);
      const double d3 = ql(mv, i) - qr(mv, i - 1);
      const double d4 = ql(4, i) - qr(4, i - 1);
      const double ae = g1a2 * (euv * d1 + u * d2 + v * d3 - d4);   // entropy wave strength
      const double as = d3 - v * d1;                                // shear wave strength
      const double a4 = (d2 + (a - u) * d1 - a * ae) / (2.0 * a);
      const double a1 = d1 - ae - a4;
      wave(1, 1, i) = a1; wave(mu, 1, i) = a1 * (u - a); wave(mv, 1, i) = a1 * v; wave(4, 1, i) = a1 * (enth - u * a);
      s(1, i) = u - a;
      wave(1, 2, i) = ae; wave(mu, 2, i) = ae * u; wave(mv, 2, i) = ae * v; wave(4, 2, i) = ae * 0.5 * u2v2;
      s(2, i) = u;
      wave(1, 3, i) = 0.0; wave(mu, 3, i) = 0.0; wave(mv, 3, i) = as; wave(4, 3, i) = as * v;
      s(3, i) = u;
      wave(1, 4, i) = a4; wave(mu, 4, i) = a4 * (u + a); wave(mv, 4, i) = a4 * v; wave(4, 4, i) = a4 * (enth + u * a);
      s(4, i) = u + a;
    }
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      // total flux difference and Godunov splitting, with the Harten-Hyman fix
      // for a transonic rarefaction in the 1-wave or in the 4-wave.
      double df[4];
      for (int m = 1; m <= 4; ++m) {
        double t = 0.0;
        for (int mw = 1; mw <= 4; ++mw) t = t + s(mw, i) * wave(m, mw, i);
        df[m - 1] = t;
      }
      bool fixed = false;
      if (P.efix) {
        // 1-wave: characteristic speed u-c left of and right of the wave
        const double rl = qr(1, i - 1);
        const double pl = g1 * (qr(4, i - 1) - 0.5 * (qr(mu, i - 1) * qr(mu, i - 1) + qr(mv, i - 1) * qr(mv, i - 1)) / rl);
        const double cl = std::sqrt(gam * pl / rl);
        const double sl = qr(mu, i - 1) / rl - cl;
        if (sl < 0.0 && s(1, i) > 0.0) {
          const double r1 = qr(1, i - 1) + wave(1, 1, i);
          const double ru1 = qr(mu, i - 1) + wave(mu, 1, i);
          const double rv1 = qr(mv, i - 1) + wave(mv, 1, i);
          const double e1 = qr(4, i - 1) + wave(4, 1, i);
          const double p1 = g1 * (e1 - 0.5 * (ru1 * ru1 + rv1 * rv1) / r1);
          const double c1 = std::sqrt(gam * p1 / r1);
          const double sr = ru1 / r1 - c1;
          if (sr > 0.0) {
            const double sfract = sl * (sr - s(1, i)) / (sr - sl);
            for (int m = 1; m <= 4; ++m) {
              amdq(m, i) = sfract * wave(m, 1, i);
              apdq(m, i) = df[m - 1] - amdq(m, i);
            }
            fixed = true;
          }
        }
        if (!fixed) {
          // 4-wave: speed u+c left of and right of the wave
          const double rr = ql(1, i);
          const double pr = g1 * (ql(4, i) - 0.5 * (ql(mu, i) * ql(mu, i) + ql(mv, i) * ql(mv, i)) / rr);
          const double cr = std::sqrt(gam * pr / rr);
          const double sr = ql(mu, i) / rr + cr;
          if (s(4, i) < 0.0 && sr > 0.0) {
            const double r3 = ql(1, i) - wave(1, 4, i);
            const double ru3 = ql(mu, i) - wave(mu, 4, i);
            const double rv3 = ql(mv, i) - wave(mv, 4, i);
            const double e3 = ql(4, i) - wave(4, 4, i);
            const double p3 = g1 * (e3 - 0.5 * (ru3 * ru3 + rv3 * rv3) / r3);
            const double c3 = std::sqrt(gam * p3 / r3);
            const double sl3 = ru3 / r3 + c3;
            if (sl3 < 0.0) {
              const double sfract = sr * (s(4, i) - sl3) / (sr - sl3);
              for (int m = 1; m <= 4; ++m) {
                apdq(m, i) = sfract * wave(m, 4, i);
                amdq(m, i) = df[m - 1] - apdq(m, i);
              }
              fixed = true;
            }
          }
        }
      }
      if (!fixed) {
        for (int m = 1; m <= 4; ++m) {
          double am = 0.0;
          for (int mw = 1; mw <= 4; ++mw)
            if (s(mw, i) < 0.0) am = am + s(mw, i) * wave(m, mw, i);
          amdq(m, i) = am;
          apdq(m, i) = df[m - 1] - am;
        }
      }
    }
    return;
  }
}

// ---------------------------------------------------------------- rpt2
inline void rpt2(const ProbParams& P, int ixy, int imp, int meqn, int mbc, int mx,
                 Slice ql, Slice qr, Slice aux1, Slice aux2, Slice aux3,
                 Slice asdq, Slice bmasdq, Slice bpasdq) {
  (void)aux1;
  if (P.solver == SOLVER_VC_ADVECTION) {
    // kv: the transverse velocity component; i1: the cell asdq belongs to (i-1 for the
    // amdq side, i for apdq); aux2 holds its row, aux3 the row above
    const int kv = 3 - ixy;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      const int i1 = i - 2 + imp;
      bmasdq(1, i) = std::min(aux2(kv, i1), 0.0) * asdq(1, i);
      bpasdq(1, i) = std::max(aux3(kv, i1), 0.0) * asdq(1, i);
    }
    return;
  }
  if (P.solver == SOLVER_ADVECTION) {
    const double st = (ixy == 1) ? P.vbar : P.ubar;
    const double stm = std::min(st, 0.0), stp = std::max(st, 0.0);
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      bmasdq(1, i) = stm * asdq(1, i);
      bpasdq(1, i) = stp * asdq(1, i);
    }
    return;
  }
  if (P.solver == SOLVER_ACOUSTICS) {
    const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      const double a1 = (-asdq(1, i) + P.zz * asdq(mv, i)) / (2.0 * P.zz);
      const double a2 = (asdq(1, i) + P.zz * asdq(mv, i)) / (2.0 * P.zz);
      bmasdq(1, i) = P.cc * a1 * P.zz; bmasdq(mu, i) = 0.0; bmasdq(mv, i) = -P.cc * a1;
      bpasdq(1, i) = P.cc * a2 * P.zz; bpasdq(mu, i) = 0.0; bpasdq(mv, i) = P.cc * a2;
    }
    return;
  }
  if (P.solver == SOLVER_EULER) {
    // Eigen-decomposition of the Jacobian in the transverse direction, at the
    // Roe average of the two states of interface i.
    const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
    const double g1 = P.gamma1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      const double rl = qr(1, i - 1), rr = ql(1, i);
      const double sql = std::sqrt(rl), sqr = std::sqrt(rr);
      const double pl = g1 * (qr(4, i - 1) - 0.5 * (qr(mu, i - 1) * qr(mu, i - 1) + qr(mv, i - 1) * qr(mv, i - 1)) / rl);
      const double pr = g1 * (ql(4, i) - 0.5 * (ql(mu, i) * ql(mu, i) + ql(mv, i) * ql(mv, i)) / rr);
      const double rsum = sql + sqr;
      const double u = (qr(mu, i - 1) / sql + ql(mu, i) / sqr) / rsum;
      const double v = (qr(mv, i - 1) / sql + ql(mv, i) / sqr) / rsum;
      const double enth = ((qr(4, i - 1) + pl) / sql + (ql(4, i) + pr) / sqr) / rsum;
      const double u2v2 = u * u + v * v;
      const double a2 = g1 * (enth - 0.5 * u2v2);
      const double a = std::sqrt(a2);
      const double g1a2 = g1 / a2;
      const double euv = enth - u2v2;
      const double d1 = asdq(1, i), dmu = asdq(mu, i), dmv = asdq(mv, i), d4 = asdq(4, i);
      const double ae = g1a2 * (euv * d1 + u * dmu + v * dmv - d4);
      const double as = dmu - u * d1;
      const double a4 = (dmv + (a - v) * d1 - a * ae) / (2.0 * a);
      const double a1 = d1 - ae - a4;
      // waves in the transverse direction: speeds v-a, v, v, v+a
      double w[4][4], sp[4];
      w[0][0] = a1; w[0][mu - 1] = a1 * u; w[0][mv - 1] = a1 * (v - a); w[0][3] = a1 * (enth - v * a); sp[0] = v - a;
      w[1][0] = ae; w[1][mu - 1] = ae * u; w[1][mv - 1] = ae * v; w[1][3] = ae * 0.5 * u2v2; sp[1] = v;
      w[2][0] = 0.0; w[2][mu - 1] = as; w[2][mv - 1] = 0.0; w[2][3] = as * u; sp[2] = v;
      w[3][0] = a4; w[3][mu - 1] = a4 * u; w[3][mv - 1] = a4 * (v + a); w[3][3] = a4 * (enth + v * a); sp[3] = v + a;
      for (int m = 0; m < 4; ++m) {
        double bm = 0.0, bp = 0.0;
        for (int mw = 0; mw < 4; ++mw) {
          bm = bm + std::min(sp[mw], 0.0) * w[mw][m];
          bp = bp + std::max(sp[mw], 0.0) * w[mw][m];
        }
        bmasdq(m + 1, i) = bm; bpasdq(m + 1, i) = bp;
      }
    }
    return;
  }
}

}  // namespace orc
