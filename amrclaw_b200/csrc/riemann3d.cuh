// 3D Euler Riemann solver of the patch step as device functions, one interface
// at a time: rpn3 (Roe, 3 waves, Harten-Hyman entropy fix) and the transverse /
// doubly transverse split used by rpt3 and rptt3 (which coincide for Euler: both
// decompose a fluctuation in the eigenvectors of the transverse flux Jacobian at
// the Roe average of the normal interface). Every expression is evaluated in the
// order of the CPU restatement so FP64 results are bit-identical (the library is
// built without FMA contraction).
#pragma once
#include "riemann2d.cuh"

namespace amrb {

template <class R> struct Roe3T { R u[5], enth, u2, a, g1a2, euv; };
using Roe3D = Roe3T<double>;

// Momentum components of sweep ixyz: normal, y-like, z-like (cyclic).
__host__ __device__ __forceinline__ void frame3d(int ixyz, int& mu, int& mv, int& mw) {
  if (ixyz == 1) { mu = 2; mv = 3; mw = 4; }
  else if (ixyz == 2) { mu = 3; mv = 4; mw = 2; }
  else { mu = 4; mv = 2; mw = 3; }
}

// Roe average of the left state L (cell i-1) and the right state R (cell i); arrays are 1-based.
template <class T>
__device__ __forceinline__ Roe3T<T> roe3d(T g1, const T* L, const T* R) {
  const T rl = L[1], rr = R[1];
  const T sql = sqrt(rl), sqr = sqrt(rr);
  const T pl = g1 * (L[5] - T(0.5) * (L[2] * L[2] + L[3] * L[3] + L[4] * L[4]) / rl);
  const T pr = g1 * (R[5] - T(0.5) * (R[2] * R[2] + R[3] * R[3] + R[4] * R[4]) / rr);
  const T rsum = sql + sqr;
  Roe3T<T> o;
  o.u[0] = o.u[1] = T(0);
#pragma unroll
  for (int m = 2; m <= 4; ++m) o.u[m] = (L[m] / sql + R[m] / sqr) / rsum;
  o.enth = ((L[5] + pl) / sql + (R[5] + pr) / sqr) / rsum;
  o.u2 = o.u[2] * o.u[2] + o.u[3] * o.u[3] + o.u[4] * o.u[4];
  const T a2 = g1 * (o.enth - T(0.5) * o.u2);
  o.a = sqrt(a2);
  o.g1a2 = g1 / a2;
  o.euv = o.enth - o.u2;
  return o;
}

// Split d (0-based, 5 components) in direction mn (momentum index 2..4; mt1, mt2 the others).
template <class T>
__device__ __forceinline__ void euler3d_split(const Roe3T<T>& R, int mn, int mt1, int mt2, const T* d, T* bm, T* bp) {
  const T un = R.u[mn], a = R.a;
  const T a3 = R.g1a2 * (R.euv * d[0] + un * d[mn - 1] + R.u[mt1] * d[mt1 - 1] + R.u[mt2] * d[mt2 - 1] - d[4]);
  const T a2 = d[mt1 - 1] - R.u[mt1] * d[0];
  const T a4 = d[mt2 - 1] - R.u[mt2] * d[0];
  const T a5 = (d[mn - 1] + (a - un) * d[0] - a * a3) / (T(2) * a);
  const T a1 = d[0] - a3 - a5;
  T w[3][5], sp[3];
  w[0][0] = a1; w[0][mn - 1] = a1 * (un - a); w[0][mt1 - 1] = a1 * R.u[mt1]; w[0][mt2 - 1] = a1 * R.u[mt2];
  w[0][4] = a1 * (R.enth - un * a); sp[0] = un - a;
  w[1][0] = a3; w[1][mn - 1] = a3 * un; w[1][mt1 - 1] = a3 * R.u[mt1] + a2; w[1][mt2 - 1] = a3 * R.u[mt2] + a4;
  w[1][4] = a3 * T(0.5) * R.u2 + a2 * R.u[mt1] + a4 * R.u[mt2]; sp[1] = un;
  w[2][0] = a5; w[2][mn - 1] = a5 * (un + a); w[2][mt1 - 1] = a5 * R.u[mt1]; w[2][mt2 - 1] = a5 * R.u[mt2];
  w[2][4] = a5 * (R.enth + un * a); sp[2] = un + a;
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    T am = T(0), ap = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      am = am + dmin(sp[k], T(0)) * w[k][m];
      ap = ap + dmax(sp[k], T(0)) * w[k][m];
    }
    bm[m] = am; bp[m] = ap;
  }
}

// Transverse split (rpt3 / rptt3) of d in direction icoor (2: y-like, 3: z-like) of sweep ixyz.
template <class T>
__device__ __forceinline__ void euler3d_trans(const Roe3T<T>& R, int ixyz, int icoor, const T* d, T* bm, T* bp) {
  int mu, mv, mw;
  frame3d(ixyz, mu, mv, mw);
  const int mn = (icoor == 2) ? mv : mw;
  const int mt1 = (icoor == 2) ? mw : mu;
  const int mt2 = (icoor == 2) ? mu : mv;
  euler3d_split(R, mn, mt1, mt2, d, bm, bp);
}

// rpn3 at one interface: L = q(i-1), R = q(i) (1-based arrays of 5) with their Roe
// average o = roe3d(g1, L, R). Returns the waves (3 x 5, 0-based components), speeds,
// and the fluctuations.
template <class T>
__device__ __forceinline__ void euler3d_rpn_roe(T gam, T g1, bool efix, int ixyz, const T* L, const T* R,
                                                const Roe3T<T>& o, T wave[3][5], T s[3], T* amdq, T* apdq) {
  int mu, mv, mw;
  frame3d(ixyz, mu, mv, mw);
  const T u = o.u[mu], v = o.u[mv], w = o.u[mw], a = o.a;
  const T d1 = R[1] - L[1], du = R[mu] - L[mu], dv = R[mv] - L[mv], dw = R[mw] - L[mw], d5 = R[5] - L[5];
  const T a3 = o.g1a2 * (o.euv * d1 + u * du + v * dv + w * dw - d5);
  const T a2 = dv - v * d1;
  const T a4 = dw - w * d1;
  const T a5 = (du + (a - u) * d1 - a * a3) / (T(2) * a);
  const T a1 = d1 - a3 - a5;
  wave[0][0] = a1; wave[0][mu - 1] = a1 * (u - a); wave[0][mv - 1] = a1 * v; wave[0][mw - 1] = a1 * w;
  wave[0][4] = a1 * (o.enth - u * a);
  s[0] = u - a;
  wave[1][0] = a3; wave[1][mu - 1] = a3 * u; wave[1][mv - 1] = a3 * v + a2; wave[1][mw - 1] = a3 * w + a4;
  wave[1][4] = a3 * T(0.5) * o.u2 + a2 * v + a4 * w;
  s[1] = u;
  wave[2][0] = a5; wave[2][mu - 1] = a5 * (u + a); wave[2][mv - 1] = a5 * v; wave[2][mw - 1] = a5 * w;
  wave[2][4] = a5 * (o.enth + u * a);
  s[2] = u + a;
  T df[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    T t = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) t = t + s[k] * wave[k][m];
    df[m] = t;
  }
  bool fixed = false;
  if (efix) {
    const T rl = L[1];
    const T pl = g1 * (L[5] - T(0.5) * (L[2] * L[2] + L[3] * L[3] + L[4] * L[4]) / rl);
    const T cl = sqrt(gam * pl / rl);
    const T sl = L[mu] / rl - cl;
    if (sl < T(0) && s[0] > T(0)) {
      T q1[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) q1[m] = L[m + 1] + wave[0][m];
      const T p1 = g1 * (q1[4] - T(0.5) * (q1[1] * q1[1] + q1[2] * q1[2] + q1[3] * q1[3]) / q1[0]);
      const T c1 = sqrt(gam * p1 / q1[0]);
      const T sr = q1[mu - 1] / q1[0] - c1;
      if (sr > T(0)) {
        const T sfract = sl * (sr - s[0]) / (sr - sl);
#pragma unroll
        for (int m = 0; m < 5; ++m) { amdq[m] = sfract * wave[0][m]; apdq[m] = df[m] - amdq[m]; }
        fixed = true;
      }
    }
    if (!fixed) {
      const T rr = R[1];
      const T pr = g1 * (R[5] - T(0.5) * (R[2] * R[2] + R[3] * R[3] + R[4] * R[4]) / rr);
      const T cr = sqrt(gam * pr / rr);
      const T sr = R[mu] / rr + cr;
      if (s[2] < T(0) && sr > T(0)) {
        T q3[5];
#pragma unroll
        for (int m = 0; m < 5; ++m) q3[m] = R[m + 1] - wave[2][m];
        const T p3 = g1 * (q3[4] - T(0.5) * (q3[1] * q3[1] + q3[2] * q3[2] + q3[3] * q3[3]) / q3[0]);
        const T c3 = sqrt(gam * p3 / q3[0]);
        const T sl3 = q3[mu - 1] / q3[0] + c3;
        if (sl3 < T(0)) {
          const T sfract = sr * (s[2] - sl3) / (sr - sl3);
#pragma unroll
          for (int m = 0; m < 5; ++m) { apdq[m] = sfract * wave[2][m]; amdq[m] = df[m] - apdq[m]; }
          fixed = true;
        }
      }
    }
  }
  if (!fixed) {
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      T am = T(0);
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (s[k] < T(0)) am = am + s[k] * wave[k][m];
      amdq[m] = am;
      apdq[m] = df[m] - am;
    }
  }
}

template <class T>
__device__ __forceinline__ void euler3d_rpn(T gam, T g1, bool efix, int ixyz, const T* L, const T* R,
                                            T wave[3][5], T s[3], T* amdq, T* apdq) {
  const Roe3T<T> o = roe3d(g1, L, R);
  euler3d_rpn_roe(gam, g1, efix, ixyz, L, R, o, wave, s, amdq, apdq);
}

}  // namespace amrb
