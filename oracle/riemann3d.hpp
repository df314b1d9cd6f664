// Oracle (test infrastructure only): CPU Riemann solvers for the 3D oracle.
//
// As in 2D the reference takes rpn3/rpt3/rptt3 from the un-vendored
// clawpack/riemann repository (tests/advection_3d_swirl/Makefile pulls
// rpn3_vc_advection / rpt3_vc_advection / rptt3_vc_advection). These are
// restated from the published mathematics with the reference's calling
// convention (call sites src/3d/flux3.f:220-226, 302-365, 411-422, 538-545;
// qad.f:125-126):
//   rpn3(ixyz,...,ql,qr,auxl,auxr)   interface i sits between qr(:,i-1) and ql(:,i)
//   rpt3(ixyz,icoor,imp,...,asdq)    splits asdq in the transverse direction
//                                    icoor (2: "y-like", 3: "z-like")
//   rptt3(ixyz,icoor,imp,impt,...)   splits a quantity already split in the
//                                    other transverse direction (side impt)
// The transverse directions of a sweep are cyclic: ixyz=1 -> (y, z), ixyz=2 ->
// (z, x), ixyz=3 -> (x, y). aux1/aux2/aux3 hold the -1/0/+1 neighbours in the
// y-like direction and their third index the -1/0/+1 neighbours in the z-like
// direction (src/3d/step3.f:167-180, 275-288, 391-404).
//
//  * euler: Roe solver with 3 waves (u-a; entropy + two shear waves at u; u+a)
//    and the Harten-Hyman fix for transonic rarefactions in the acoustic waves;
//    the transverse and doubly transverse splits decompose the vector in the
//    eigenvectors of the flux Jacobian of the transverse direction at the Roe
//    average of the normal interface (LeVeque, FVMHP 2002, 15.3, 19.3.3, 21.6;
//    Langseth & LeVeque, J. Comput. Phys. 165 (2000) 126-166).
//  * vc_advection: upwinding with face-centred velocities (aux 1..3 = u, v, w
//    at the left x-, y- and z-face of the cell); the transverse splits move a
//    fluctuation with the transverse face velocity of the cell it sits in
//    (Langseth & LeVeque 2000, section 3).
#pragma once
#include "riemann2d.hpp"

namespace orc {

// aux slices of a pencil: a(ma, i, kk), kk = 1..3 (z-like offset -1/0/+1)
struct AuxSlice3 {
  double* p; int maux; int base; int len;
  double& operator()(int ma, int i, int kk) const {
    return p[(ma - 1) + maux * ((i - base) + (size_t)len * (kk - 1))];
  }
};

// Momentum components in the frame of sweep ixyz: normal, y-like, z-like.
inline void frame3(int ixyz, int& mu, int& mv, int& mw) {
  if (ixyz == 1) { mu = 2; mv = 3; mw = 4; }
  else if (ixyz == 2) { mu = 3; mv = 4; mw = 2; }
  else { mu = 4; mv = 2; mw = 3; }
}

struct Roe3 { double u[5], enth, u2, a, g1a2, euv; };

// Roe average of the states qr(:,i-1) and ql(:,i); u[m] is the velocity of momentum component m (2..4).
inline Roe3 roe3(const ProbParams& P, Slice ql, Slice qr, int i) {
  const double g1 = P.gamma1;
  const double rl = qr(1, i - 1), rr = ql(1, i);
  const double sql = std::sqrt(rl), sqr = std::sqrt(rr);
  const double pl = g1 * (qr(5, i - 1) - 0.5 * (qr(2, i - 1) * qr(2, i - 1) + qr(3, i - 1) * qr(3, i - 1) + qr(4, i - 1) * qr(4, i - 1)) / rl);
  const double pr = g1 * (ql(5, i) - 0.5 * (ql(2, i) * ql(2, i) + ql(3, i) * ql(3, i) + ql(4, i) * ql(4, i)) / rr);
  const double rsum = sql + sqr;
  Roe3 R;
  R.u[0] = R.u[1] = 0.0;
  for (int m = 2; m <= 4; ++m) R.u[m] = (qr(m, i - 1) / sql + ql(m, i) / sqr) / rsum;
  R.enth = ((qr(5, i - 1) + pl) / sql + (ql(5, i) + pr) / sqr) / rsum;
  R.u2 = R.u[2] * R.u[2] + R.u[3] * R.u[3] + R.u[4] * R.u[4];
  const double a2 = g1 * (R.enth - 0.5 * R.u2);
  R.a = std::sqrt(a2);
  R.g1a2 = g1 / a2;
  R.euv = R.enth - R.u2;
  return R;
}

// Eigen-decomposition of d in direction mn (momentum index of the direction;
// mt1, mt2 the other two): 3 waves, speeds un-a, un, un+a, summed into the
// left- and right-going parts.
inline void euler3_split(const Roe3& R, int mn, int mt1, int mt2, const double d[5], double bm[5], double bp[5]) {
  const double un = R.u[mn], a = R.a;
  const double a3 = R.g1a2 * (R.euv * d[0] + un * d[mn - 1] + R.u[mt1] * d[mt1 - 1] + R.u[mt2] * d[mt2 - 1] - d[4]);
  const double a2 = d[mt1 - 1] - R.u[mt1] * d[0];
  const double a4 = d[mt2 - 1] - R.u[mt2] * d[0];
  const double a5 = (d[mn - 1] + (a - un) * d[0] - a * a3) / (2.0 * a);
  const double a1 = d[0] - a3 - a5;
  double w[3][5], sp[3];
  w[0][0] = a1; w[0][mn - 1] = a1 * (un - a); w[0][mt1 - 1] = a1 * R.u[mt1]; w[0][mt2 - 1] = a1 * R.u[mt2];
  w[0][4] = a1 * (R.enth - un * a); sp[0] = un - a;
  w[1][0] = a3; w[1][mn - 1] = a3 * un; w[1][mt1 - 1] = a3 * R.u[mt1] + a2; w[1][mt2 - 1] = a3 * R.u[mt2] + a4;
  w[1][4] = a3 * 0.5 * R.u2 + a2 * R.u[mt1] + a4 * R.u[mt2]; sp[1] = un;
  w[2][0] = a5; w[2][mn - 1] = a5 * (un + a); w[2][mt1 - 1] = a5 * R.u[mt1]; w[2][mt2 - 1] = a5 * R.u[mt2];
  w[2][4] = a5 * (R.enth + un * a); sp[2] = un + a;
  for (int m = 0; m < 5; ++m) {
    double am = 0.0, ap = 0.0;
    for (int k = 0; k < 3; ++k) {
      am = am + std::min(sp[k], 0.0) * w[k][m];
      ap = ap + std::max(sp[k], 0.0) * w[k][m];
    }
    bm[m] = am; bp[m] = ap;
  }
}

// ---------------------------------------------------------------- rpn3
inline void rpn3(const ProbParams& P, int ixyz, int meqn, int mwaves, int mbc, int mx,
                 Slice ql, Slice qr, Slice auxl, Slice auxr, Waves wave, Slice s,
                 Slice amdq, Slice apdq) {
  (void)auxr;
  if (P.solver == SOLVER_VC_ADVECTION) {
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      wave(1, 1, i) = ql(1, i) - qr(1, i - 1);
      s(1, i) = auxl(ixyz, i);
      amdq(1, i) = std::min(auxl(ixyz, i), 0.0) * wave(1, 1, i);
      apdq(1, i) = std::max(auxl(ixyz, i), 0.0) * wave(1, 1, i);
    }
    return;
  }
  if (P.solver == SOLVER_ADVECTION) {
    const double vel = (ixyz == 1) ? P.ubar : (ixyz == 2) ? P.vbar : P.wbar;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      wave(1, 1, i) = ql(1, i) - qr(1, i - 1);
      s(1, i) = vel;
      amdq(1, i) = std::min(vel, 0.0) * wave(1, 1, i);
      apdq(1, i) = std::max(vel, 0.0) * wave(1, 1, i);
    }
    return;
  }
  // Euler
  int mu, mv, mw;
  frame3(ixyz, mu, mv, mw);
  const double g1 = P.gamma1, gam = P.gamma;
  (void)meqn; (void)mwaves;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    const Roe3 R = roe3(P, ql, qr, i);
    const double u = R.u[mu], v = R.u[mv], w = R.u[mw], a = R.a;
    const double d1 = ql(1, i) - qr(1, i - 1);
    const double du = ql(mu, i) - qr(mu, i - 1);
    const double dv = ql(mv, i) - qr(mv, i - 1);
    const double dw = ql(mw, i) - qr(mw, i - 1);
    const double d5 = ql(5, i) - qr(5, i - 1);
    const double a3 = R.g1a2 * (R.euv * d1 + u * du + v * dv + w * dw - d5);
    const double a2 = dv - v * d1;
    const double a4 = dw - w * d1;
    const double a5 = (du + (a - u) * d1 - a * a3) / (2.0 * a);
    const double a1 = d1 - a3 - a5;
    wave(1, 1, i) = a1; wave(mu, 1, i) = a1 * (u - a); wave(mv, 1, i) = a1 * v; wave(mw, 1, i) = a1 * w;
    wave(5, 1, i) = a1 * (R.enth - u * a);
    s(1, i) = u - a;
    wave(1, 2, i) = a3; wave(mu, 2, i) = a3 * u; wave(mv, 2, i) = a3 * v + a2; wave(mw, 2, i) = a3 * w + a4;
    wave(5, 2, i) = a3 * 0.5 * R.u2 + a2 * v + a4 * w;
    s(2, i) = u;
    wave(1, 3, i) = a5; wave(mu, 3, i) = a5 * (u + a); wave(mv, 3, i) = a5 * v; wave(mw, 3, i) = a5 * w;
    wave(5, 3, i) = a5 * (R.enth + u * a);
    s(3, i) = u + a;
  }
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double df[5];
    for (int m = 1; m <= 5; ++m) {
      double t = 0.0;
      for (int k = 1; k <= 3; ++k) t = t + s(k, i) * wave(m, k, i);
      df[m - 1] = t;
    }
    bool fixed = false;
    if (P.efix) {
      // 1-wave: u-c left of and right of the wave
      const double rl = qr(1, i - 1);
      const double pl = g1 * (qr(5, i - 1) - 0.5 * (qr(2, i - 1) * qr(2, i - 1) + qr(3, i - 1) * qr(3, i - 1) + qr(4, i - 1) * qr(4, i - 1)) / rl);
      const double cl = std::sqrt(gam * pl / rl);
      const double sl = qr(mu, i - 1) / rl - cl;
      if (sl < 0.0 && s(1, i) > 0.0) {
        double q1[5];
        for (int m = 1; m <= 5; ++m) q1[m - 1] = qr(m, i - 1) + wave(m, 1, i);
        const double p1 = g1 * (q1[4] - 0.5 * (q1[1] * q1[1] + q1[2] * q1[2] + q1[3] * q1[3]) / q1[0]);
        const double c1 = std::sqrt(gam * p1 / q1[0]);
        const double sr = q1[mu - 1] / q1[0] - c1;
        if (sr > 0.0) {
          const double sfract = sl * (sr - s(1, i)) / (sr - sl);
          for (int m = 1; m <= 5; ++m) {
            amdq(m, i) = sfract * wave(m, 1, i);
            apdq(m, i) = df[m - 1] - amdq(m, i);
          }
          fixed = true;
        }
      }
      if (!fixed) {
        // 3-wave: u+c left of and right of the wave
        const double rr = ql(1, i);
        const double pr = g1 * (ql(5, i) - 0.5 * (ql(2, i) * ql(2, i) + ql(3, i) * ql(3, i) + ql(4, i) * ql(4, i)) / rr);
        const double cr = std::sqrt(gam * pr / rr);
        const double sr = ql(mu, i) / rr + cr;
        if (s(3, i) < 0.0 && sr > 0.0) {
          double q3[5];
          for (int m = 1; m <= 5; ++m) q3[m - 1] = ql(m, i) - wave(m, 3, i);
          const double p3 = g1 * (q3[4] - 0.5 * (q3[1] * q3[1] + q3[2] * q3[2] + q3[3] * q3[3]) / q3[0]);
          const double c3 = std::sqrt(gam * p3 / q3[0]);
          const double sl3 = q3[mu - 1] / q3[0] + c3;
          if (sl3 < 0.0) {
            const double sfract = sr * (s(3, i) - sl3) / (sr - sl3);
            for (int m = 1; m <= 5; ++m) {
              apdq(m, i) = sfract * wave(m, 3, i);
              amdq(m, i) = df[m - 1] - apdq(m, i);
            }
            fixed = true;
          }
        }
      }
    }
    if (!fixed) {
      for (int m = 1; m <= 5; ++m) {
        double am = 0.0;
        for (int k = 1; k <= 3; ++k)
          if (s(k, i) < 0.0) am = am + s(k, i) * wave(m, k, i);
        amdq(m, i) = am;
        apdq(m, i) = df[m - 1] - am;
      }
    }
  }
}

// ---------------------------------------------------------------- rpt3
inline void rpt3(const ProbParams& P, int ixyz, int icoor, int imp, int meqn, int mbc, int mx,
                 Slice ql, Slice qr, AuxSlice3 aux1, AuxSlice3 aux2, AuxSlice3 aux3,
                 Slice asdq, Slice bmasdq, Slice bpasdq) {
  (void)meqn;
  if (P.solver == SOLVER_VC_ADVECTION) {
    int mu, mv, mw;
    frame3(ixyz, mu, mv, mw);
    const int comp = (icoor == 2) ? mv - 1 : mw - 1;  // aux index of the transverse face velocity
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      const int i1 = i - 2 + imp;
      if (icoor == 2) {
        bmasdq(1, i) = std::min(aux2(comp, i1, 2), 0.0) * asdq(1, i);
        bpasdq(1, i) = std::max(aux3(comp, i1, 2), 0.0) * asdq(1, i);
      } else {
        bmasdq(1, i) = std::min(aux2(comp, i1, 2), 0.0) * asdq(1, i);
        bpasdq(1, i) = std::max(aux2(comp, i1, 3), 0.0) * asdq(1, i);
      }
    }
    return;
  }
  if (P.solver == SOLVER_ADVECTION) {
    int mu, mv, mw;
    frame3(ixyz, mu, mv, mw);
    const int comp = (icoor == 2) ? mv - 1 : mw - 1;
    const double vel = (comp == 1) ? P.ubar : (comp == 2) ? P.vbar : P.wbar;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      bmasdq(1, i) = std::min(vel, 0.0) * asdq(1, i);
      bpasdq(1, i) = std::max(vel, 0.0) * asdq(1, i);
    }
    return;
  }
  (void)aux1; (void)aux2; (void)aux3; (void)imp;
  int mu, mv, mw;
  frame3(ixyz, mu, mv, mw);
  const int mn = (icoor == 2) ? mv : mw;
  const int mt1 = (icoor == 2) ? mw : mu;
  const int mt2 = (icoor == 2) ? mu : mv;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    const Roe3 R = roe3(P, ql, qr, i);
    double d[5], bm[5], bp[5];
    for (int m = 0; m < 5; ++m) d[m] = asdq(m + 1, i);
    euler3_split(R, mn, mt1, mt2, d, bm, bp);
    for (int m = 0; m < 5; ++m) { bmasdq(m + 1, i) = bm[m]; bpasdq(m + 1, i) = bp[m]; }
  }
}

// ---------------------------------------------------------------- rptt3
inline void rptt3(const ProbParams& P, int ixyz, int icoor, int imp, int impt, int meqn, int mbc, int mx,
                  Slice ql, Slice qr, AuxSlice3 aux1, AuxSlice3 aux2, AuxSlice3 aux3,
                  Slice bsasdq, Slice cmbsasdq, Slice cpbsasdq) {
  if (P.solver == SOLVER_VC_ADVECTION) {
    int mu, mv, mw;
    frame3(ixyz, mu, mv, mw);
    const int comp = (icoor == 2) ? mv - 1 : mw - 1;
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      const int i1 = i - 2 + imp;
      if (icoor == 2) {
        // moved in the z-like direction to the neighbour impt (1: -1, 2: +1)
        const int kz = (impt == 1) ? 1 : 3;
        cmbsasdq(1, i) = std::min(aux2(comp, i1, kz), 0.0) * bsasdq(1, i);
        cpbsasdq(1, i) = std::max(aux3(comp, i1, kz), 0.0) * bsasdq(1, i);
      } else {
        // moved in the y-like direction to the neighbour impt
        const AuxSlice3& A = (impt == 1) ? aux1 : aux3;
        cmbsasdq(1, i) = std::min(A(comp, i1, 2), 0.0) * bsasdq(1, i);
        cpbsasdq(1, i) = std::max(A(comp, i1, 3), 0.0) * bsasdq(1, i);
      }
    }
    return;
  }
  // constant advection and Euler: the same split as rpt3 in direction icoor
  rpt3(P, ixyz, icoor, imp, meqn, mbc, mx, ql, qr, aux1, aux2, aux3, bsasdq, cmbsasdq, cpbsasdq);
}

}  // namespace orc
