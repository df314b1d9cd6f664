// 1D Riemann solvers of the patch step (the reference's rp1 plugins) as host/device
// functions at one interface: ql is the state left of the interface (cell i-1, the
// reference's qr(:,i-1)) and qr the state right of it (cell i, its ql(:,i)). Each
// expression is evaluated in the order of the CPU restatement so FP64 results are
// bit-identical (the library is built without FMA contraction).
//  * advection: constant-velocity upwinding (LeVeque, FVMHP 2002, ch. 4)
//  * acoustics: characteristic decomposition of constant-coefficient acoustics (FVMHP 3.8)
//  * euler: Roe solver, 3 waves, Harten-Hyman entropy fix, fluctuations gathered wave by
//    wave from the left (FVMHP 15.3.3-15.3.5)
#pragma once
#include <cmath>

namespace amrb {

enum Plugin1 { SOLVER1_ADVECTION = 1, SOLVER1_ACOUSTICS = 2, SOLVER1_EULER = 3 };
constexpr int MAXW1 = 3;  // waves and equations of the 1D plugins

struct Prob1 {
  int solver;
  int meqn, mwaves;
  double u;                  // advection
  double rho, bulk, cc, zz;  // acoustics
  double gamma, gamma1;      // euler
};

__host__ __device__ inline void rp1_at(const Prob1& P, const double* ql, const double* qr, double (&wave)[MAXW1][MAXW1],
                                       double (&s)[MAXW1], double (&amdq)[MAXW1], double (&apdq)[MAXW1]) {
  if (P.solver == SOLVER1_ADVECTION) {
    wave[0][0] = qr[0] - ql[0];
    s[0] = P.u;
    amdq[0] = (0.0 < P.u ? 0.0 : P.u) * wave[0][0];  // std::min(u, 0.0)
    apdq[0] = (P.u < 0.0 ? 0.0 : P.u) * wave[0][0];  // std::max(u, 0.0)
    return;
  }
  if (P.solver == SOLVER1_ACOUSTICS) {
    const double d1 = qr[0] - ql[0], d2 = qr[1] - ql[1];
    const double a1 = (-d1 + P.zz * d2) / (2.0 * P.zz);
    const double a2 = (d1 + P.zz * d2) / (2.0 * P.zz);
    wave[0][0] = -a1 * P.zz; wave[0][1] = a1; s[0] = -P.cc;
    wave[1][0] = a2 * P.zz; wave[1][1] = a2; s[1] = P.cc;
    for (int m = 0; m < 2; ++m) {
      double am = 0.0, ap = 0.0;
      for (int mw = 0; mw < 2; ++mw) {
        if (s[mw] < 0.0) am = am + s[mw] * wave[mw][m];
        else ap = ap + s[mw] * wave[mw][m];
      }
      amdq[m] = am; apdq[m] = ap;
    }
    return;
  }
  const double g1 = P.gamma1, gam = P.gamma;
  const double rl = ql[0], rr = qr[0];
  const double sql = sqrt(rl), sqr = sqrt(rr);
  const double pl = g1 * (ql[2] - 0.5 * (ql[1] * ql[1]) / rl);
  const double pr = g1 * (qr[2] - 0.5 * (qr[1] * qr[1]) / rr);
  const double rsum = sql + sqr;
  const double u = (ql[1] / sql + qr[1] / sqr) / rsum;
  const double enth = ((ql[2] + pl) / sql + (qr[2] + pr) / sqr) / rsum;
  const double a2 = g1 * (enth - 0.5 * u * u);
  const double a = sqrt(a2);
  const double d1 = qr[0] - ql[0], d2 = qr[1] - ql[1], d3 = qr[2] - ql[2];
  const double ae = (g1 / a2) * ((enth - u * u) * d1 + u * d2 - d3);
  const double a3 = (d2 + (a - u) * d1 - a * ae) / (2.0 * a);
  const double a1 = d1 - ae - a3;
  wave[0][0] = a1; wave[0][1] = a1 * (u - a); wave[0][2] = a1 * (enth - u * a); s[0] = u - a;
  wave[1][0] = ae; wave[1][1] = ae * u; wave[1][2] = ae * 0.5 * u * u; s[1] = u;
  wave[2][0] = a3; wave[2][1] = a3 * (u + a); wave[2][2] = a3 * (enth + u * a); s[2] = u + a;
  // entropy fix: amdq from the left-going parts, wave by wave
  [&] {
    const double rhoim1 = ql[0];
    const double pim1 = g1 * (ql[2] - 0.5 * (ql[1] * ql[1]) / rhoim1);
    const double cim1 = sqrt(gam * pim1 / rhoim1);
    const double s0 = ql[1] / rhoim1 - cim1;
    if (s0 >= 0.0 && s[0] > 0.0) {
      for (int m = 0; m < 3; ++m) amdq[m] = 0.0;
      return;
    }
    const double rho1 = ql[0] + wave[0][0], rhou1 = ql[1] + wave[0][1], en1 = ql[2] + wave[0][2];
    const double p1 = g1 * (en1 - 0.5 * (rhou1 * rhou1) / rho1);
    const double c1 = sqrt(gam * p1 / rho1);
    const double s1 = rhou1 / rho1 - c1;
    double sfract;
    if (s0 < 0.0 && s1 > 0.0) sfract = s0 * (s1 - s[0]) / (s1 - s0);
    else if (s[0] < 0.0) sfract = s[0];
    else sfract = 0.0;
    for (int m = 0; m < 3; ++m) amdq[m] = sfract * wave[0][m];
    if (s[1] >= 0.0) return;
    for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + s[1] * wave[1][m];
    const double rhoi = qr[0];
    const double pi = g1 * (qr[2] - 0.5 * (qr[1] * qr[1]) / rhoi);
    const double ci = sqrt(gam * pi / rhoi);
    const double s3 = qr[1] / rhoi + ci;
    const double rho2 = qr[0] - wave[2][0], rhou2 = qr[1] - wave[2][1], en2 = qr[2] - wave[2][2];
    const double p2 = g1 * (en2 - 0.5 * (rhou2 * rhou2) / rho2);
    const double c2 = sqrt(gam * p2 / rho2);
    const double s2 = rhou2 / rho2 + c2;
    if (s2 < 0.0 && s3 > 0.0) sfract = s2 * (s3 - s[2]) / (s3 - s2);
    else if (s[2] < 0.0) sfract = s[2];
    else return;
    for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + sfract * wave[2][m];
  }();
  for (int m = 0; m < 3; ++m) {
    double df = 0.0;
    for (int mw = 0; mw < 3; ++mw) df = df + s[mw] * wave[mw][m];
    apdq[m] = df - amdq[m];
  }
}

}  // namespace amrb
