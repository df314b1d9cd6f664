// Oracle (test infrastructure only): CPU Riemann solvers for the 1D oracle.
//
// The reference does not ship its Riemann solvers: the 1D regression tests pull
// rp1_acoustics, rp1_advection and rp1_euler_with_efix from the separate clawpack/riemann
// repository (tests/acoustics_1d_homogeneous/Makefile, tests/advection_1d_example1/Makefile,
// tests/euler_1d_wcblast/Makefile), which is not vendored and not version-pinned. These
// are restated from the published mathematics with the reference's calling convention:
//   rp1(...,ql,qr,...)  the interface i sits between qr(:,i-1) and ql(:,i)
//                       (call sites src/1d/flux1.f:68-69, qad.f:113-114, 173-174)
// Loops run over i = 2-mbc .. mx+mbc like the clawpack solvers.
//
//  * advection: constant velocity upwinding (LeVeque, FVMHP 2002, ch. 4).
//  * acoustics: characteristic decomposition of constant-coefficient acoustics
//    (FVMHP 2002, section 3.8).
//  * euler: Roe solver with 3 waves and the Harten-Hyman entropy fix for transonic
//    rarefactions, the fluctuations gathered wave by wave from the left as the
//    clawpack rp1_euler_with_efix solver does (FVMHP 2002, sections 15.3.3-15.3.5).
#pragma once
#include <algorithm>
#include <cmath>

namespace orc1 {

enum SolverKind1 { SOLVER1_ADVECTION = 1, SOLVER1_ACOUSTICS = 2, SOLVER1_EULER = 3 };

struct ProbParams1 {
  int solver = SOLVER1_ADVECTION;
  double u = 1.0;                            // advection
  double rho = 1, bulk = 1, cc = 1, zz = 1;  // acoustics
  double gamma = 1.4, gamma1 = 0.4;          // euler
  bool efix = true;
};

// Fortran-style accessors: a(m, i) with i from base = 1-mbc; wave(m, mw, i)
struct Slice1 {
  double* p; int ld; int base;
  double& operator()(int m, int i) const { return p[(m - 1) + ld * (i - base)]; }
};
struct Waves1 {
  double* p; int meqn; int mwaves; int base;
  double& operator()(int m, int mw, int i) const { return p[(m - 1) + meqn * ((mw - 1) + mwaves * (i - base))]; }
};

inline void rp1(const ProbParams1& P, int meqn, int mwaves, int mbc, int mx, Slice1 ql, Slice1 qr, Waves1 wave, Slice1 s,
                Slice1 amdq, Slice1 apdq) {
  if (P.solver == SOLVER1_ADVECTION) {
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      wave(1, 1, i) = ql(1, i) - qr(1, i - 1);
      s(1, i) = P.u;
      amdq(1, i) = std::min(P.u, 0.0) * wave(1, 1, i);
      apdq(1, i) = std::max(P.u, 0.0) * wave(1, 1, i);
    }
    return;
  }
  if (P.solver == SOLVER1_ACOUSTICS) {
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      const double d1 = ql(1, i) - qr(1, i - 1);
      const double d2 = ql(2, i) - qr(2, i - 1);
      const double a1 = (-d1 + P.zz * d2) / (2.0 * P.zz);
      const double a2 = (d1 + P.zz * d2) / (2.0 * P.zz);
      wave(1, 1, i) = -a1 * P.zz; wave(2, 1, i) = a1; s(1, i) = -P.cc;
      wave(1, 2, i) = a2 * P.zz; wave(2, 2, i) = a2; s(2, i) = P.cc;
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
  // Euler: Roe averages of the left state qr(:,i-1) and the right state ql(:,i)
  const double g1 = P.gamma1, gam = P.gamma;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    const double rl = qr(1, i - 1), rr = ql(1, i);
    const double sql = std::sqrt(rl), sqr = std::sqrt(rr);
    const double pl = g1 * (qr(3, i - 1) - 0.5 * (qr(2, i - 1) * qr(2, i - 1)) / rl);
    const double pr = g1 * (ql(3, i) - 0.5 * (ql(2, i) * ql(2, i)) / rr);
    const double rsum = sql + sqr;
    const double u = (qr(2, i - 1) / sql + ql(2, i) / sqr) / rsum;
    const double enth = ((qr(3, i - 1) + pl) / sql + (ql(3, i) + pr) / sqr) / rsum;
    const double a2 = g1 * (enth - 0.5 * u * u);
    const double a = std::sqrt(a2);
    const double d1 = ql(1, i) - qr(1, i - 1);
    const double d2 = ql(2, i) - qr(2, i - 1);
    const double d3 = ql(3, i) - qr(3, i - 1);
    const double ae = (g1 / a2) * ((enth - u * u) * d1 + u * d2 - d3);  // entropy wave strength
    const double a3 = (d2 + (a - u) * d1 - a * ae) / (2.0 * a);
    const double a1 = d1 - ae - a3;
    wave(1, 1, i) = a1; wave(2, 1, i) = a1 * (u - a); wave(3, 1, i) = a1 * (enth - u * a); s(1, i) = u - a;
    wave(1, 2, i) = ae; wave(2, 2, i) = ae * u; wave(3, 2, i) = ae * 0.5 * u * u; s(2, i) = u;
    wave(1, 3, i) = a3; wave(2, 3, i) = a3 * (u + a); wave(3, 3, i) = a3 * (enth + u * a); s(3, i) = u + a;
  }
  // Harten-Hyman entropy fix, wave by wave from the left: amdq gathers the left-going part
  // of the 1-wave (all of it, or the fraction of a transonic rarefaction), the 2-wave if it
  // goes left, and the left-going part of the 3-wave; apdq = sum s*wave - amdq
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    const double rhoim1 = qr(1, i - 1);
    const double pim1 = g1 * (qr(3, i - 1) - 0.5 * (qr(2, i - 1) * qr(2, i - 1)) / rhoim1);
    const double cim1 = std::sqrt(gam * pim1 / rhoim1);
    const double s0 = qr(2, i - 1) / rhoim1 - cim1;  // u-c in the left state
    if (s0 >= 0.0 && s(1, i) > 0.0) {
      for (int m = 1; m <= 3; ++m) amdq(m, i) = 0.0;  // everything goes right
      continue;
    }
    const double rho1 = qr(1, i - 1) + wave(1, 1, i);
    const double rhou1 = qr(2, i - 1) + wave(2, 1, i);
    const double en1 = qr(3, i - 1) + wave(3, 1, i);
    const double p1 = g1 * (en1 - 0.5 * (rhou1 * rhou1) / rho1);
    const double c1 = std::sqrt(gam * p1 / rho1);
    const double s1 = rhou1 / rho1 - c1;  // u-c right of the 1-wave
    double sfract;
    if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s(1, i)) / (s1 - s0);
    else if (s(1, i) < 0.0) sfract = s(1, i);
    else sfract = 0.0;
    for (int m = 1; m <= 3; ++m) amdq(m, i) = sfract * wave(m, 1, i);
    if (s(2, i) >= 0.0) continue;
    for (int m = 1; m <= 3; ++m) amdq(m, i) = amdq(m, i) + s(2, i) * wave(m, 2, i);
    const double rhoi = ql(1, i);
    const double pi = g1 * (ql(3, i) - 0.5 * (ql(2, i) * ql(2, i)) / rhoi);
    const double ci = std::sqrt(gam * pi / rhoi);
    const double s3 = ql(2, i) / rhoi + ci;  // u+c in the right state
    const double rho2 = ql(1, i) - wave(1, 3, i);
    const double rhou2 = ql(2, i) - wave(2, 3, i);
    const double en2 = ql(3, i) - wave(3, 3, i);
    const double p2 = g1 * (en2 - 0.5 * (rhou2 * rhou2) / rho2);
    const double c2 = std::sqrt(gam * p2 / rho2);
    const double s2 = rhou2 / rho2 + c2;  // u+c left of the 3-wave
    if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s(3, i)) / (s3 - s2);
    else if (s(3, i) < 0.0) sfract = s(3, i);
    else continue;
    for (int m = 1; m <= 3; ++m) amdq(m, i) = amdq(m, i) + sfract * wave(m, 3, i);
  }
  for (int m = 1; m <= 3; ++m)
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      double df = 0.0;
      for (int mw = 1; mw <= mwaves; ++mw) df = df + s(mw, i) * wave(m, mw, i);
      apdq(m, i) = df - amdq(m, i);
    }
}

}  // namespace orc1
