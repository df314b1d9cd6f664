// 3D kernels of the patch-advance path (sm_100a, FP64, built without FMA contraction).
//
//   sweep3_kernel<DIR>  one thread per cell of every pencil of a sweep direction of
//                       every patch of a level (flux3.f:4-633 over step3.f's pencils):
//                       Roe solves of the cell's own interface and of the next one,
//                       wave limiter, second-order correction, and the transverse and
//                       doubly transverse splits. The cell's transverse increments
//                       (gadd, hadd) are accumulated in the reference's statement
//                       order (terms of interface c, then of interface c+1) and left
//                       in a per-level staging buffer together with faddm/faddp.
//   face3_kernel        every face flux of the level, summing the staged increments
//                       in the order step3.f adds them (x-, y-, then z-sweeps; pencils
//                       in loop order).
//   update3_kernel      conservative update (stepgrid.f:142-153) into the other buffer.
//   fsv3 / fad3         flux registers from the face fluxes (fluxsv.f, fluxad.f).
//   qad3_kernel         coarse/fine Riemann problems into the registers (qad.f:4-534).
//   fill3 / bc3         ghost-fill programs (intfil.f, filpatch.f, filval.f, cstore.f)
//                       and bc3amr.f90 extrapolation / wall boundaries.
//   upbnd3 / average3   level sync (upbnd.f, update.f).
//   gauges3, mass3, gather3: gauge sampling (gauges_module.f90:302-460), conck.f,
//                       output gather. (Flagging kernels: flags3d.cu.)
#include "kernels3d.cuh"
#include <algorithm>

namespace amrb {

namespace {

constexpr int NG3 = 2;  // num_ghost (the host rejects other values)

__device__ __forceinline__ int floordiv3(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

__device__ __forceinline__ int find_patch(const long long* pre, int np, long long t) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
  atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

template <class T>
__device__ __forceinline__ T philim3(int meth, T r) {
  switch (meth) {
    case 1: return dmax(T(0), dmin(T(1), r));
    case 2: return dmax(dmax(T(0), dmin(T(1), T(2) * r)), dmin(T(2), r));
    case 3: return (r + fabs(r)) / (T(1) + fabs(r));
    case 4: { const T c = (T(1) + r) / T(2); return dmax(T(0), dmin(dmin(c, T(2)), T(2) * r)); }
    case 5: return r;
  }
  return T(0);
}

// ------------------------------------------------------------------- sweeps
// One thread per interface of a pencil. A tile of SW_T consecutive interfaces (of the
// level's pencils of one direction, pencils of n1+3 interfaces 0..n1+2 each) makes
// its Riemann solves once and shares the waves in shared memory; tiles overlap by
// three interfaces so that every cell's two interfaces (c and c+1) and their
// neighbours (for the limiters) fall in the tile that owns the cell.
//   phase A  rpn3 at the thread's interface (waves to shared memory)
//   phase B1 limiter and second-order correction of interface e; faddm/faddp of e;
//            transverse terms of the apdq side (flux3.f: to cell i = e), stored
//   phase B2 transverse terms of the amdq side (to cell i-1 = e-1), added to what B1
//            stored for that cell, term by term in flux3.f's statement order
#ifndef SW_TILE
#define SW_TILE 128  // interfaces per sweep tile (threads per block)
#endif
constexpr int SW_T = SW_TILE;
constexpr int SW_OWN = SW_T - 3;
#ifndef SW_MINB
#define SW_MINB 3  // resident tiles per SM the register budget is sized for (FP64)
#endif
#ifndef SW_MINB_F32
#define SW_MINB_F32 5  // the same for the FP32 form: half the shared buffer, 96 registers, no spills
#endif
template <class T>
constexpr int sweep_min_blocks() { return sizeof(T) == 4 ? SW_MINB_F32 : SW_MINB; }

// (a - 3*b) (m4 = 2) or a: the doubly transverse inputs of flux3.f:429-507
template <int NV, class T>
__device__ __forceinline__ void dt_input(int m4, T sgn3, const T* a, const T* b, T* o) {
#pragma unroll
  for (int m = 0; m < NV; ++m) o[m] = (m4 == 2) ? a[m] + sgn3 * b[m] : a[m];
}

// ---- physics policies of the sweep: the problem's rpn3 / rpt3 / rptt3 at one interface.
// imp: 1 splits the amdq side (cell e-1), 2 the apdq side (cell e); icoor: 2 the y-like,
// 3 the z-like transverse direction; impt: the side (1 minus, 2 plus) of the first split.

// Euler (Roe, entropy fix): every split uses the Roe average of the interface.
template <class T>
struct Euler3Phys {
  static constexpr int NV = 5, NW = 3;
  Roe3T<T> R;
  template <int DIR>
  __device__ __forceinline__ void load(const T*, const PatchDev&, long long, long long, long long, int) {}
  template <int DIR>
  __device__ __forceinline__ void load_normal(const T*, const PatchDev&, long long, long long, long long, int) {}
  template <int DIR>
  __device__ __forceinline__ void rpn(const Step3Params& sp, const T* QL, const T* QR, T (&W)[NW][NV], T* S, T* AM, T* AP) {
    R = roe3d((T)sp.gamma1, QL, QR);
    euler3d_rpn_roe((T)sp.gamma, (T)sp.gamma1, sp.efix != 0, DIR, QL, QR, R, W, S, AM, AP);
  }
  template <int DIR>
  __device__ __forceinline__ void rpt(int, int icoor, const T* in, T* m, T* p) const { euler3d_trans(R, DIR, icoor, in, m, p); }
  template <int DIR>
  __device__ __forceinline__ void rptt(int, int icoor, int, const T* in, T* m, T* p) const { euler3d_trans(R, DIR, icoor, in, m, p); }
};

// Advection in a face-centred velocity field (aux 1..3 = u, v, w at the left x-, y- and
// z-face of each cell): the normal speed is the interface's own face velocity; a split
// moves a fluctuation with the transverse face velocities of the cell it belongs to, on
// its lower and upper face, in the pencil row it has already been moved to (impt).
// The y-like / z-like axes of the sweeps are (j, k), (k, i), (i, j) (step3.f's aux1..3
// and their third index).
template <class T>
struct Swirl3Phys {
  static constexpr int NV = 1, NW = 1;
  T un;
  // [0]: cell e-1, [1]: cell e. vy: y-like face velocity at (dy, dz) = (0,0), (+1,0),
  // (0,-1), (+1,-1), (0,+1), (+1,+1); vz: z-like one at (0,0), (0,+1), (-1,0), (-1,+1),
  // (+1,0), (+1,+1)
  T vy[2][6], vz[2][6];
  template <int DIR>
  __device__ __forceinline__ void load(const T* pool, const PatchDev& P, long long base, long long step, long long plane, int e) {
    const T* a = pool + P.aux;
    const long long mi = P.mitot, mij = (long long)P.mitot * P.mjtot;
    const long long sy = DIR == 1 ? mi : DIR == 2 ? mij : 1;
    const long long sz = DIR == 1 ? mij : DIR == 2 ? 1 : mi;
    const int cy = DIR == 1 ? 1 : DIR == 2 ? 2 : 0, cz = DIR == 1 ? 2 : DIR == 2 ? 0 : 1;
    un = a[(long long)(DIR - 1) * plane + base + (long long)e * step];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const long long at = base + (long long)(e - 1 + c) * step;
      const T* ay = a + cy * plane + at;
      const T* az = a + cz * plane + at;
      vy[c][0] = ay[0]; vy[c][1] = ay[sy]; vy[c][2] = ay[-sz]; vy[c][3] = ay[sy - sz]; vy[c][4] = ay[sz]; vy[c][5] = ay[sy + sz];
      vz[c][0] = az[0]; vz[c][1] = az[sz]; vz[c][2] = az[-sy]; vz[c][3] = az[sz - sy]; vz[c][4] = az[sy]; vz[c][5] = az[sy + sz];
    }
  }
  // the split step's rpn3 needs only the interface's own face velocity (no transverse rows)
  template <int DIR>
  __device__ __forceinline__ void load_normal(const T* pool, const PatchDev& P, long long base, long long step, long long plane, int e) {
    un = pool[P.aux + (long long)(DIR - 1) * plane + base + (long long)e * step];
  }
  template <int DIR>
  __device__ __forceinline__ void rpn(const Step3Params&, const T* QL, const T* QR, T (&W)[NW][NV], T* S, T* AM, T* AP) {
    W[0][0] = QR[1] - QL[1];
    S[0] = un;
    AM[0] = dmin(un, T(0)) * W[0][0];
    AP[0] = dmax(un, T(0)) * W[0][0];
  }
  template <int DIR>
  __device__ __forceinline__ void rpt(int imp, int icoor, const T* in, T* m, T* p) const {
    const int c = imp - 1;
    if (icoor == 2) { m[0] = dmin(vy[c][0], T(0)) * in[0]; p[0] = dmax(vy[c][1], T(0)) * in[0]; }
    else { m[0] = dmin(vz[c][0], T(0)) * in[0]; p[0] = dmax(vz[c][1], T(0)) * in[0]; }
  }
  template <int DIR>
  __device__ __forceinline__ void rptt(int imp, int icoor, int impt, const T* in, T* m, T* p) const {
    const int c = imp - 1, o = impt == 1 ? 2 : 4;
    if (icoor == 2) { m[0] = dmin(vy[c][o], T(0)) * in[0]; p[0] = dmax(vy[c][o + 1], T(0)) * in[0]; }
    else { m[0] = dmin(vz[c][o], T(0)) * in[0]; p[0] = dmax(vz[c][o + 1], T(0)) * in[0]; }
  }
};

// the registered 3D plugins satisfy the device plugin contract (include/amrgpu_riemann.cuh)
static_assert(amrgpu_plugin::Check3D<Euler3Phys<double>, Step3Params, double>::value, "euler_roe_efix: rpn3/rpt3/rptt3 contract");
static_assert(amrgpu_plugin::Check3D<Swirl3Phys<double>, Step3Params, double>::value, "vc_advection: rpn3/rpt3/rptt3 contract");
static_assert(amrgpu_plugin::Check3D<Euler3Phys<float>, Step3Params, float>::value, "euler_roe_efix (FP32): contract");

// The transverse and doubly transverse terms of one side of interface e (flux3.f:429-507
// for gadd, 552-630 for hadd): imp 2 splits apdq into the terms of cell e, imp 1 splits
// amdq into the terms of cell e-1. g points at the cell's column of the shared terms
// (row x at g[x * SW_T]): gadd (side, offset d) in rows ((side-1)*3 + d+1)*NV + m, hadd in
// rows (6 + (side-1)*3 + d+1)*NV + m. imp 2 starts every term from zero, imp 1 adds to what
// imp 2 left. Each term gets its summands in flux3.f's statement order: the transverse
// split, the doubly transverse parts, then the second-order part (m3 = 2). The splits are
// made in an order that keeps few of them live at once: the z-like ones first (their
// doubly transverse parts feed gadd), then the y-like ones; the hadd terms wait in shared
// memory between their first summand and the rest.
template <int DIR, class T, class PH>
__device__ __forceinline__ void trans_side(const PH& ph, int imp, const T* F, const T* CQ, int m3, int m4, T dtdx, T dtdy,
                                           T dtdz, T* g) {
  constexpr int NV = PH::NV;
  auto G = [&](int x) -> T& { return g[x * SW_T]; };
  const T c6 = (T)(1.0 / 6.0);
  const T sgn3 = imp == 2 ? T(-3) : T(3);
  const bool first = imp == 2;
  // z-like split of the fluctuation and of the second-order part
  T cm[NV], cp[NV], cmq[NV], cpq[NV];
  ph.template rpt<DIR>(imp, 3, F, cm, cp);
  if (m3 == 2) ph.template rpt<DIR>(imp, 3, CQ, cmq, cpq);
  else {
#pragma unroll
    for (int m = 0; m < NV; ++m) cmq[m] = cpq[m] = T(0);
  }
  // hadd: the first summand of the (0, 1, 1) and (1, 1, 1) terms
#pragma unroll
  for (int m = 0; m < NV; ++m) {
    const T b01 = first ? T(0) : G(7 * NV + m), b11 = first ? T(0) : G(10 * NV + m);
    G(7 * NV + m) = b01 - T(0.5) * dtdx * cm[m];
    G(10 * NV + m) = b11 - T(0.5) * dtdx * cp[m];
  }
  // gadd: the y-like split, the doubly transverse parts of the z-like split, the second order
  {
    T P1[NV], P2[NV], M1[NV], M2[NV];
    if (m4 > 0) {
      T t[NV];
      dt_input<NV>(m4, sgn3, cp, cpq, t);
      ph.template rptt<DIR>(imp, 2, 2, t, P1, P2);
      dt_input<NV>(m4, sgn3, cm, cmq, t);
      ph.template rptt<DIR>(imp, 2, 1, t, M1, M2);
    }
    T bm[NV], bp[NV];
    ph.template rpt<DIR>(imp, 2, F, bm, bp);
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      T g01 = (first ? T(0) : G(1 * NV + m)) - T(0.5) * dtdx * bm[m];
      T g11 = (first ? T(0) : G(4 * NV + m)) - T(0.5) * dtdx * bp[m];
      if (m4 > 0) {
        T g00 = first ? T(0) : G(0 * NV + m), g02 = first ? T(0) : G(2 * NV + m);
        T g10 = first ? T(0) : G(3 * NV + m), g12 = first ? T(0) : G(5 * NV + m);
        g11 = g11 + c6 * dtdx * dtdz * (P2[m] - M2[m]);
        g01 = g01 + c6 * dtdx * dtdz * (P1[m] - M1[m]);
        g12 = g12 - c6 * dtdx * dtdz * P2[m];
        g02 = g02 - c6 * dtdx * dtdz * P1[m];
        g10 = g10 + c6 * dtdx * dtdz * M2[m];
        g00 = g00 + c6 * dtdx * dtdz * M1[m];
        G(0 * NV + m) = g00;
        G(2 * NV + m) = g02;
        G(3 * NV + m) = g10;
        G(5 * NV + m) = g12;
      } else if (first) {
        G(0 * NV + m) = T(0);
        G(2 * NV + m) = T(0);
        G(3 * NV + m) = T(0);
        G(5 * NV + m) = T(0);
      }
      G(1 * NV + m) = g01;
      G(4 * NV + m) = g11;
    }
    T bmq[NV], bpq[NV];
    if (m3 == 2) {
      ph.template rpt<DIR>(imp, 2, CQ, bmq, bpq);
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        G(4 * NV + m) = first ? G(4 * NV + m) + dtdx * bpq[m] : G(4 * NV + m) - dtdx * bpq[m];
        G(1 * NV + m) = first ? G(1 * NV + m) + dtdx * bmq[m] : G(1 * NV + m) - dtdx * bmq[m];
      }
    } else {
#pragma unroll
      for (int m = 0; m < NV; ++m) bmq[m] = bpq[m] = T(0);
    }
    // hadd: the doubly transverse parts of the y-like split, then the second order
    T X1[NV], X2[NV], Y1[NV], Y2[NV];
    if (m4 > 0) {
      T t[NV];
      dt_input<NV>(m4, sgn3, bp, bpq, t);
      ph.template rptt<DIR>(imp, 3, 2, t, X1, X2);
      dt_input<NV>(m4, sgn3, bm, bmq, t);
      ph.template rptt<DIR>(imp, 3, 1, t, Y1, Y2);
    }
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      T h01 = G(7 * NV + m), h11 = G(10 * NV + m);
      if (m4 > 0) {
        T h00 = first ? T(0) : G(6 * NV + m), h02 = first ? T(0) : G(8 * NV + m);
        T h10 = first ? T(0) : G(9 * NV + m), h12 = first ? T(0) : G(11 * NV + m);
        h11 = h11 + c6 * dtdx * dtdy * (X2[m] - Y2[m]);
        h01 = h01 + c6 * dtdx * dtdy * (X1[m] - Y1[m]);
        h12 = h12 - c6 * dtdx * dtdy * X2[m];
        h02 = h02 - c6 * dtdx * dtdy * X1[m];
        h10 = h10 + c6 * dtdx * dtdy * Y2[m];
        h00 = h00 + c6 * dtdx * dtdy * Y1[m];
        G(6 * NV + m) = h00;
        G(8 * NV + m) = h02;
        G(9 * NV + m) = h10;
        G(11 * NV + m) = h12;
      } else if (first) {
        G(6 * NV + m) = T(0);
        G(8 * NV + m) = T(0);
        G(9 * NV + m) = T(0);
        G(11 * NV + m) = T(0);
      }
      if (m3 == 2) {
        h11 = first ? h11 + dtdx * cpq[m] : h11 - dtdx * cpq[m];
        h01 = first ? h01 + dtdx * cmq[m] : h01 - dtdx * cmq[m];
      }
      G(7 * NV + m) = h01;
      G(10 * NV + m) = h11;
    }
  }
}

// one tile of sweep direction DIR. sW: the block's shared buffer, first the waves
// [NW*NV][SW_T], then (after they are read) the transverse terms [12*NV][SW_T] of the
// tile's cells: the apdq side writes them, the amdq side of the next interface adds to
// them there, and each cell's terms then go to the stash in one coalesced write
template <int DIR, class T, class PH>
__device__ __forceinline__ void sweep3_tile(const Step3Args& A, long long tile, T (*sW)[SW_T]) {
  constexpr int NV = PH::NV, NW = PH::NW;
  T* const sG = &sW[0][0];
  auto G = [&](int x, int col) -> T& { return sG[x * SW_T + col]; };
  const long long* c0 = A.comp0 + (long long)(DIR - 1) * (A.np + 1);
  const long long* s0 = A.sweep0 + (long long)(DIR - 1) * (A.np + 1);
  const long long first = c0[0], last = c0[A.np];
  const int l = threadIdx.x;
  const long long g = first + tile * SW_OWN - 1 + l;
  const bool valid = g >= first && g < last;
  const Step3Params sp = A.sp;
  const double dn = DIR == 1 ? A.dx : DIR == 2 ? A.dy : A.dz;
  const double dt = A.dt_dev ? *A.dt_dev : A.dt;
  const T dtdx = (T)(dt / dn);
  // transverse steps of flux3's dtdy / dtdz arguments for this sweep (step3.f:192, 300, 416)
  const T dtdy = (T)(DIR == 1 ? dt / A.dy : DIR == 2 ? dt / A.dz : dt / A.dx);
  const T dtdz = (T)(DIR == 1 ? dt / A.dz : DIR == 2 ? dt / A.dx : dt / A.dy);
  int e = -1, n1 = 0;
  long long slot = 0;  // stash slot of pencil cell e (meaningful for e in 1..n1+1)
  PH ph;
  T W[NW][NV], S[NW], AM[NV], AP[NV];
  if (valid) {
    const int pi = find_patch(c0, A.np, g);
    const PatchDev& P = A.patches[A.plist[pi]];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
    n1 = DIR == 1 ? mx : DIR == 2 ? my : mz;
    const int n2 = DIR == 1 ? my : mx;
    const long long loc = g - c0[pi];
    e = (int)(loc % (n1 + 3));
    const long long pen = loc / (n1 + 3);
    const int a = (int)(pen % (n2 + 2)), b = (int)(pen / (n2 + 2));
    slot = s0[pi] + pen * (n1 + 1) + (e - 1);
    const long long mi = P.mitot, mj = P.mjtot;
    long long base, step;  // enlarged-array index of pencil cell x is base + x*step (cell 0: enlarged index 1)
    if (DIR == 1) { base = ((long long)(b - 1 + NG3) * mj + (a - 1 + NG3)) * mi + (NG3 - 1); step = 1; }
    else if (DIR == 2) { base = ((long long)(b - 1 + NG3) * mj + (NG3 - 1)) * mi + (a - 1 + NG3); step = mi; }
    else { base = ((long long)(NG3 - 1) * mj + (b - 1 + NG3)) * mi + (a - 1 + NG3); step = mi * mj; }
    const long long plane = mi * mj * P.mktot;
    const T* q = static_cast<const T*>(A.pool) + P.q[P.cur];
    T QL[NV + 1], QR[NV + 1];
    const long long atl = base + (long long)(e - 1) * step, atr = atl + step;
#pragma unroll
    for (int m = 1; m <= NV; ++m) { QL[m] = q[(m - 1) * plane + atl]; QR[m] = q[(m - 1) * plane + atr]; }
    QL[0] = QR[0] = T(0);
    ph.template load<DIR>(static_cast<const T*>(A.pool), P, base, step, plane, e);
    ph.template rpn<DIR>(sp, QL, QR, W, S, AM, AP);
#pragma unroll
    for (int k = 0; k < NW; ++k)
#pragma unroll
      for (int m = 0; m < NV; ++m) sW[k * NV + m][l] = W[k][m];
  }
  __syncthreads();
  // interfaces 1..n1+1 carry fluxes; the tile edges only serve their neighbours
  const bool live = valid && e >= 1 && e <= n1 + 1 && l >= 1 && l <= SW_T - 2;
  const bool owned = live && l <= SW_T - 3;
  T cfl = T(0);
  T CQ[NV];
#pragma unroll
  for (int m = 0; m < NV; ++m) CQ[m] = T(0);
  T* st = static_cast<T*>(A.stash) + slot;
  const long long ss = A.stash_stride;
  const T c6 = (T)(1.0 / 6.0);
  const int m3 = sp.m3, m4 = sp.m4, order = sp.order;
  if (live) {
    // Courant number of interface e (flux3.f:237-246)
#pragma unroll
    for (int k = 0; k < NW; ++k) cfl = dmax(cfl, dmax(dtdx * S[k], -dtdx * S[k]));
    if (order != 1) {
      // limiter.f: r from the unlimited neighbour waves, upwind side by the speed's sign
      const T dtdxave = T(0.5) * (dtdx + dtdx);
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        if (sp.mthlim[k] == 0) continue;
        T dl = T(0), dr = T(0), wn = T(0);
#pragma unroll
        for (int m = 0; m < NV; ++m) dl = dl + sW[k * NV + m][l - 1] * W[k][m];
#pragma unroll
        for (int m = 0; m < NV; ++m) dr = dr + W[k][m] * sW[k * NV + m][l + 1];
#pragma unroll
        for (int m = 0; m < NV; ++m) wn = wn + W[k][m] * W[k][m];
        if (wn != T(0)) {
          const T r = (S[k] > T(0)) ? dl / wn : dr / wn;
          const T phi = philim3(sp.mthlim[k], r);
#pragma unroll
          for (int m = 0; m < NV; ++m) W[k][m] = phi * W[k][m];
        }
      }
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        T x = T(0);
#pragma unroll
        for (int k = 0; k < NW; ++k) x = x + T(0.5) * fabs(S[k]) * (T(1) - fabs(S[k]) * dtdxave) * W[k][m];
        CQ[m] = x;
      }
    }
    if (owned) {
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        T fm = T(0) + AM[m], fp = T(0) - AP[m];
        if (order != 1) { fm = fm + CQ[m]; fp = fp + CQ[m]; }
        st[(long long)m * ss] = fm;
        st[(long long)(NV + m) * ss] = fp;
      }
      if (e <= n1 && m3 <= 0)
        for (int x = 2 * NV; x < stash_values(NV); ++x) st[(long long)x * ss] = T(0);
    }
  }
  __syncthreads();  // the waves in sW are read: the buffer takes the transverse terms now
  // apdq side of interface e: the terms of cell e (flux3.f:429-505, 552-628 with i = e)
  if (owned && e <= n1 && m3 > 0) trans_side<DIR, T, PH>(ph, 2, AP, CQ, m3, m4, dtdx, dtdy, dtdz, sG + l);
  __syncthreads();
  // amdq side of interface e: the terms of cell e-1, owned by thread l-1 of this tile
  if (live && m3 > 0 && e >= 2 && l >= 2) trans_side<DIR, T, PH>(ph, 1, AM, CQ, m3, m4, dtdx, dtdy, dtdz, sG + (l - 1));
  __syncthreads();
  // the cell's transverse terms to the stash
  if (owned && e <= n1 && m3 > 0)
    for (int x = 0; x < 12 * NV; ++x) st[(long long)(2 * NV + x) * ss] = G(x, l);
  // block-wide max of the Courant number, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) cfl = dmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, o));
  if ((threadIdx.x & 31) == 0 && cfl > T(0)) atomic_max_nonneg(A.cflmax, (double)cfl);
}

// one launch per direction: a block per tile
// shared memory of a sweep block: the larger of the wave buffer and the transverse terms
template <class T, class PH>
constexpr int sweep3_smem_bytes() {
  return (PH::NW > 12 ? PH::NW : 12) * PH::NV * SW_T * (int)sizeof(T);
}
template <int DIR, class T, class PH>
__global__ void __launch_bounds__(SW_T, sweep_min_blocks<T>()) sweep3_kernel(Step3Args A) {
  extern __shared__ __align__(16) unsigned char sweep_smem[];
  sweep3_tile<DIR, T, PH>(A, blockIdx.x, reinterpret_cast<T (*)[SW_T]>(sweep_smem));
}

// persistent work queue over the tiles of all three directions of the level (x tiles,
// then y, then z): resident blocks take the next tile from an atomic counter until none
// is left. The tiles are independent (each writes its own stash slots), so no block
// waits on another.
template <class T, class PH>
__global__ void __launch_bounds__(SW_T, sweep_min_blocks<T>()) sweep3_queue_kernel(Step3Args A, unsigned int nx, unsigned int nxy, unsigned int ntot) {
  extern __shared__ __align__(16) unsigned char sweep_smem[];
  T (*sW)[SW_T] = reinterpret_cast<T (*)[SW_T]>(sweep_smem);
  __shared__ unsigned int item;
  for (;;) {
    __syncthreads();  // the previous tile is done with sW and item
    if (threadIdx.x == 0) item = atomicAdd(A.queue, 1u);
    __syncthreads();
    const unsigned int it = item;
    if (it >= ntot) return;
    if (it < nx) sweep3_tile<1, T, PH>(A, it, sW);
    else if (it < nxy) sweep3_tile<2, T, PH>(A, it - nx, sW);
    else sweep3_tile<3, T, PH>(A, it - nxy, sW);
  }
}

// ------------------------------------------------------------------- dimensional splitting
// stepgrid_dimSplit.f:4-264 (step3x.f, step3y.f, step3z.f, flux3_dimSplit.f) as one launch
// per direction. Pencils (split_pencils): x along every (j, k) row of the enlarged patch,
// y along the interior i and every k, z along the interior (i, j); each of n1+3 interfaces
// 0..n1+2 (cells e-1 | e), in tiles of SW_T consecutive interfaces overlapping by three like
// the unsplit sweeps. A thread solves its interface (waves shared for the limiter), forms
// fm = 0 + (amdq + cqxx) and fp = 0 + (-apdq + cqxx) (flux3_dimSplit.f's faddm = amdq,
// faddp = -apdq, + cqxx, added to zeroed arrays), and updates the cell it owns:
//   x: q[cur] -> q[1-cur] (every row; only interior i are written or read later)
//   y: q[1-cur] -> the level's split scratch (interior i and j, every k)
//   z: split scratch -> q[1-cur] (interior cells)
// Faces of interior pencils go to the flux array for fluxsv / fluxad.
template <int DIR, class T, class PH>
__global__ void __launch_bounds__(SW_T) split3_kernel(Step3Args A) {
  constexpr int NV = PH::NV, NW = PH::NW;
  __shared__ T sW[NW * NV][SW_T];
  __shared__ T sF[2 * NV][SW_T];
  const long long* c0 = A.scomp0 + (long long)(DIR - 1) * (A.np + 1);
  const long long first = c0[0], last = c0[A.np];
  const int l = threadIdx.x;
  const long long g = first + (long long)blockIdx.x * SW_OWN - 1 + l;
  const bool valid = g >= first && g < last;
  const Step3Params sp = A.sp;
  const double dn = DIR == 1 ? A.dx : DIR == 2 ? A.dy : A.dz;
  const double dt = A.dt_dev ? *A.dt_dev : A.dt;
  const T dtdx = (T)(dt / dn);
  int e = -1, n1 = 0, pi = 0;
  bool interior_pencil = false;
  long long base = 0, step = 0, plane = 0, fidx0 = 0, fstep = 0;
  const T* qi = nullptr;
  T* qo = nullptr;
  PH ph;
  T W[NW][NV], S[NW], AM[NV], AP[NV];
  if (valid) {
    pi = find_patch(c0, A.np, g);
    const PatchDev& P = A.patches[A.plist[pi]];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
    n1 = DIR == 1 ? mx : DIR == 2 ? my : mz;
    const int na = DIR == 1 ? my + 4 : mx;  // pencils: a fastest, then b
    const long long loc = g - c0[pi];
    e = (int)(loc % (n1 + 3));
    const long long pen = loc / (n1 + 3);
    const int a = (int)(pen % na), b = (int)(pen / na);
    const long long mi = P.mitot, mj = P.mjtot;
    // enlarged 0-based index of pencil cell x (1-based along the pencil) is base + (x + 1) * step
    long long ie = 0, je = 0, ke = 0;
    if (DIR == 1) { je = a; ke = b; step = 1; interior_pencil = a >= 2 && a < my + 2 && b >= 2 && b < mz + 2; }
    else if (DIR == 2) { ie = a + 2; ke = b; step = mi; interior_pencil = b >= 2 && b < mz + 2; }
    else { ie = a + 2; je = b + 2; step = mi * mj; interior_pencil = true; }
    base = (ke * mj + je) * mi + ie;
    plane = mi * mj * P.mktot;
    const T* pool = static_cast<const T*>(A.pool);
    T* scratch = static_cast<T*>(A.split) + (long long)NV * A.ecell0[pi];
    qi = DIR == 1 ? pool + P.q[P.cur] : DIR == 2 ? pool + P.q[1 - P.cur] : scratch;
    qo = DIR == 1 ? const_cast<T*>(pool) + P.q[1 - P.cur] : DIR == 2 ? scratch : const_cast<T*>(pool) + P.q[1 - P.cur];
    // face (e) of this pencil in the patch's face block: x-faces i = e, y-faces j = e, z-faces k = e
    // (face cell (i, j, k) is ((k-1)*NJ + (j-1))*NI + (i-1) of the block, as face3_kernel)
    const long long NI = mx + 1, NJ = my + 1;
    if (DIR == 1) { fidx0 = ((long long)(b - 2) * NJ + (a - 2)) * NI - 1; fstep = 1; }              // j = a-1, k = b-1
    else if (DIR == 2) { fidx0 = ((long long)(b - 2) * NJ - 1) * NI + a; fstep = NI; }              // i = a+1, k = b-1
    else { fidx0 = (long long)b * NI + a - NJ * NI; fstep = NJ * NI; }                              // i = a+1, j = b+1
    fidx0 += A.face0[pi];
    T QL[NV + 1], QR[NV + 1];
    const long long atl = base + (long long)e * step, atr = atl + step;  // cells e-1 and e
#pragma unroll
    for (int m = 1; m <= NV; ++m) { QL[m] = qi[(m - 1) * plane + atl]; QR[m] = qi[(m - 1) * plane + atr]; }
    QL[0] = QR[0] = T(0);
    ph.template load_normal<DIR>(pool, P, base, step, plane, e + 1);
    ph.template rpn<DIR>(sp, QL, QR, W, S, AM, AP);
#pragma unroll
    for (int k = 0; k < NW; ++k)
#pragma unroll
      for (int m = 0; m < NV; ++m) sW[k * NV + m][l] = W[k][m];
  }
  __syncthreads();
  const bool live = valid && e >= 1 && e <= n1 + 1 && l >= 1 && l <= SW_T - 2;
  const bool owned = live && l <= SW_T - 3;
  T cfl = T(0);
  if (live) {
#pragma unroll
    for (int k = 0; k < NW; ++k) cfl = dmax(cfl, dmax(dtdx * S[k], -dtdx * S[k]));
    T CQ[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) CQ[m] = T(0);
    if (sp.order != 1) {
      const T dtdxave = T(0.5) * (dtdx + dtdx);
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        if (sp.mthlim[k] == 0) continue;
        T dl = T(0), dr = T(0), wn = T(0);
#pragma unroll
        for (int m = 0; m < NV; ++m) dl = dl + sW[k * NV + m][l - 1] * W[k][m];
#pragma unroll
        for (int m = 0; m < NV; ++m) dr = dr + W[k][m] * sW[k * NV + m][l + 1];
#pragma unroll
        for (int m = 0; m < NV; ++m) wn = wn + W[k][m] * W[k][m];
        if (wn != T(0)) {
          const T r = (S[k] > T(0)) ? dl / wn : dr / wn;
          const T phi = philim3(sp.mthlim[k], r);
#pragma unroll
          for (int m = 0; m < NV; ++m) W[k][m] = phi * W[k][m];
        }
      }
#pragma unroll
      for (int m = 0; m < NV; ++m) {
        T x = T(0);
#pragma unroll
        for (int k = 0; k < NW; ++k) x = x + T(0.5) * fabs(S[k]) * (T(1) - fabs(S[k]) * dtdxave) * W[k][m];
        CQ[m] = x;
      }
    }
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      const T fm = sp.order != 1 ? T(0) + (AM[m] + CQ[m]) : T(0) + AM[m];
      const T fp = sp.order != 1 ? T(0) + (-AP[m] + CQ[m]) : T(0) + (-AP[m]);
      sF[m][l] = fm;
      sF[NV + m][l] = fp;
      if (owned && interior_pencil) {
        T* F = static_cast<T*>(A.flux) + fidx0 + (long long)e * fstep;
        const long long fs = A.flux_stride;
        const int c = 2 * (DIR - 1) * NV;
        F[(c + m) * fs] = fm;
        F[(c + NV + m) * fs] = fp;
      }
    }
  }
  __syncthreads();
  // the cell e (1..n1) of the pencil: its right face is interface e+1 (thread l+1)
  if (owned && e <= n1) {
    const long long at = base + (long long)(e + 1) * step;
#pragma unroll
    for (int m = 0; m < NV; ++m) qo[m * plane + at] = qi[m * plane + at] - dtdx * (sF[m][l + 1] - sF[NV + m][l]);
  }
  // z: the two ghost layers at each end of the pencil keep their y-updated values in
  // store1 as well (the reference's array holds them; binary output writes them). The end
  // interfaces hold both cells of their layer pair; z reads the scratch, so no race.
  if (DIR == 3 && valid && (e == 0 || e == n1 + 2)) {
    const long long atl = base + (long long)e * step;
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      qo[m * plane + atl] = qi[m * plane + atl];
      qo[m * plane + atl + step] = qi[m * plane + atl + step];
    }
  }
  for (int o = 16; o > 0; o >>= 1) cfl = dmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, o));
  if ((threadIdx.x & 31) == 0 && cfl > T(0)) atomic_max_nonneg(A.cflmax, (double)cfl);
}

// stash element of gadd / hadd for side s (1,2), offset d (-1..1), component m (0..NV-1)
template <int NV>
__device__ __forceinline__ int gidx(int s, int d, int m) { return 2 * NV + ((s - 1) * 3 + (d + 1)) * NV + m; }
template <int NV>
__device__ __forceinline__ int hidx(int s, int d, int m) { return 8 * NV + ((s - 1) * 3 + (d + 1)) * NV + m; }

// ------------------------------------------------------------------- faces
constexpr int FB_I = 8, FB_J = 4, FB_K = 4;  // face bricks: one warp per k-plane, a block per brick
template <class T, int NV>
__global__ void __launch_bounds__(128) face3_kernel(Step3Args A) {
  // face cells [face0[0], face0[np]): the level's, or one patch's through a one-patch view
  const long long first = A.face0[0], total = A.face0[A.np];
  const long long ss = A.stash_stride;
  const T* S = static_cast<const T*>(A.stash);
  for (long long t = first + (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int pi = find_patch(A.face0, A.np, t);
    const PatchDev& P = A.patches[A.plist[pi]];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
    // Thread t takes the face cells of its patch in brick order: slabs of FB_K k-planes,
    // rows of FB_J j-lines in a slab, bricks of FB_I faces in a row (the last of each
    // smaller), i fastest inside a brick. A warp then reads the j- and k-contiguous
    // stashes of the y and z sweeps in whole sectors, and the warps of a block share
    // them through L1. The sums of every face are the same; only which thread makes
    // them changes.
    const int NI = mx + 1, NJ = my + 1, NK = mz + 1;
    const long long loc = t - A.face0[pi];
    const long long slab = (long long)NI * NJ * FB_K;
    const int kb = (int)(loc / slab);
    const int kcnt = min(FB_K, NK - kb * FB_K);
    const long long r1 = loc - kb * slab;
    const long long row = (long long)NI * FB_J * kcnt;
    const int jb = (int)(r1 / row);
    const int jcnt = min(FB_J, NJ - jb * FB_J);
    const int r2 = (int)(r1 - jb * row);
    const int bsz = FB_I * jcnt * kcnt;
    const int ib = r2 / bsz;
    const int icnt = min(FB_I, NI - ib * FB_I);
    const int r3 = r2 - ib * bsz;
    const int i = ib * FB_I + r3 % icnt + 1;
    const int j = jb * FB_J + (r3 / icnt) % jcnt + 1;
    const int k = kb * FB_K + r3 / (icnt * jcnt) + 1;
    const long long bx = A.sweep0[pi], by = A.sweep0[(A.np + 1) + pi], bz = A.sweep0[2 * (A.np + 1) + pi];
    auto xs = [&](int jj, int kk, int ii) { return bx + ((long long)(kk * (my + 2) + jj) * (mx + 1) + (ii - 1)); };
    auto ys = [&](int ii, int kk, int jj) { return by + ((long long)(kk * (mx + 2) + ii) * (my + 1) + (jj - 1)); };
    auto zs = [&](int ii, int jj, int kk) { return bz + ((long long)(jj * (mx + 2) + ii) * (mz + 1) + (kk - 1)); };
    T* F = static_cast<T*>(A.flux) + A.face0[pi] + ((long long)(k - 1) * NJ + (j - 1)) * NI + (i - 1);
    const long long fs = A.flux_stride;
    if (j <= my && k <= mz) {  // x-face i
      T fm[NV], fp[NV];
      const long long sx = xs(j, k, i);
#pragma unroll
      for (int m = 0; m < NV; ++m) { fm[m] = T(0) + S[m * ss + sx]; fp[m] = T(0) + S[(NV + m) * ss + sx]; }
      // y-sweeps: k' = k-1, k, k+1 (d = +1, 0, -1); pencil i-1 (side 2) then i (side 1)
#pragma unroll
      for (int d = 1; d >= -1; --d) {
        const long long s2 = ys(i - 1, k - d, j), s1 = ys(i, k - d, j);
#pragma unroll
        for (int m = 0; m < NV; ++m) {
          const T t2 = S[hidx<NV>(2, d, m) * ss + s2];
          fm[m] = fm[m] + t2; fp[m] = fp[m] + t2;
          const T t1 = S[hidx<NV>(1, d, m) * ss + s1];
          fm[m] = fm[m] + t1; fp[m] = fp[m] + t1;
        }
      }
      // z-sweeps: j' = j-1, j, j+1 (d = +1, 0, -1); pencil i-1 (side 2) then i (side 1)
#pragma unroll
      for (int d = 1; d >= -1; --d) {
        const long long s2 = zs(i - 1, j - d, k), s1 = zs(i, j - d, k);
#pragma unroll
        for (int m = 0; m < NV; ++m) {
          const T t2 = S[gidx<NV>(2, d, m) * ss + s2];
          fm[m] = fm[m] + t2; fp[m] = fp[m] + t2;
          const T t1 = S[gidx<NV>(1, d, m) * ss + s1];
          fm[m] = fm[m] + t1; fp[m] = fp[m] + t1;
        }
      }
#pragma unroll
      for (int m = 0; m < NV; ++m) { F[(0 * NV + m) * fs] = fm[m]; F[(1 * NV + m) * fs] = fp[m]; }
    }
    if (i <= mx && k <= mz) {  // y-face j
      T gm[NV], gp[NV];
#pragma unroll
      for (int m = 0; m < NV; ++m) gm[m] = T(0);
      // x-sweeps: k' = k-1, k, k+1 (d = +1, 0, -1); pencil j-1 (side 2) then j (side 1)
#pragma unroll
      for (int d = 1; d >= -1; --d) {
        const long long s2 = xs(j - 1, k - d, i), s1 = xs(j, k - d, i);
#pragma unroll
        for (int m = 0; m < NV; ++m) {
          gm[m] = gm[m] + S[gidx<NV>(2, d, m) * ss + s2];
          gm[m] = gm[m] + S[gidx<NV>(1, d, m) * ss + s1];
        }
      }
      const long long sy = ys(i, k, j);
#pragma unroll
      for (int m = 0; m < NV; ++m) { gp[m] = gm[m] + S[(NV + m) * ss + sy]; gm[m] = gm[m] + S[m * ss + sy]; }
      // z-sweeps: j' = j-1 (side 2) for i' = i-1, i, i+1 (d = +1, 0, -1), then j' = j (side 1)
#pragma unroll
      for (int side = 2; side >= 1; --side) {
        const int jp = (side == 2) ? j - 1 : j;
#pragma unroll
        for (int d = 1; d >= -1; --d) {
          const long long sz = zs(i - d, jp, k);
#pragma unroll
          for (int m = 0; m < NV; ++m) {
            const T tv = S[hidx<NV>(side, d, m) * ss + sz];
            gm[m] = gm[m] + tv; gp[m] = gp[m] + tv;
          }
        }
      }
#pragma unroll
      for (int m = 0; m < NV; ++m) { F[(2 * NV + m) * fs] = gm[m]; F[(3 * NV + m) * fs] = gp[m]; }
    }
    if (i <= mx && j <= my) {  // z-face k
      T hm[NV], hp[NV];
#pragma unroll
      for (int m = 0; m < NV; ++m) hm[m] = T(0);
      // x-sweeps: k' = k-1 (side 2) for j' = j-1, j, j+1 (d = +1, 0, -1), then k' = k (side 1)
#pragma unroll
      for (int side = 2; side >= 1; --side) {
        const int kp = (side == 2) ? k - 1 : k;
#pragma unroll
        for (int d = 1; d >= -1; --d) {
          const long long sx = xs(j - d, kp, i);
#pragma unroll
          for (int m = 0; m < NV; ++m) hm[m] = hm[m] + S[hidx<NV>(side, d, m) * ss + sx];
        }
      }
      // y-sweeps: k' = k-1 (side 2) for i' = i-1, i, i+1, then k' = k (side 1)
#pragma unroll
      for (int side = 2; side >= 1; --side) {
        const int kp = (side == 2) ? k - 1 : k;
#pragma unroll
        for (int d = 1; d >= -1; --d) {
          const long long sy = ys(i - d, kp, j);
#pragma unroll
          for (int m = 0; m < NV; ++m) hm[m] = hm[m] + S[gidx<NV>(side, d, m) * ss + sy];
        }
      }
      const long long sz = zs(i, j, k);
#pragma unroll
      for (int m = 0; m < NV; ++m) { hp[m] = hm[m] + S[(NV + m) * ss + sz]; hm[m] = hm[m] + S[m * ss + sz]; }
#pragma unroll
      for (int m = 0; m < NV; ++m) { F[(4 * NV + m) * fs] = hm[m]; F[(5 * NV + m) * fs] = hp[m]; }
    }
  }
}

// ------------------------------------------------------------------- update
template <class T, int NV>
__global__ void __launch_bounds__(256) update3_kernel(Step3Args A) {
  const long long first = A.cell0[0], total = A.cell0[A.np];
  const long long fs = A.flux_stride;
  const double dt = A.dt_dev ? *A.dt_dev : A.dt;
  const T dtdx = (T)(dt / A.dx), dtdy = (T)(dt / A.dy), dtdz = (T)(dt / A.dz);
  for (long long t = first + (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int pi = find_patch(A.cell0, A.np, t);
    const PatchDev& P = A.patches[A.plist[pi]];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
    const long long loc = t - A.cell0[pi];
    const int i = (int)(loc % mx) + 1, j = (int)((loc / mx) % my) + 1, k = (int)(loc / ((long long)mx * my)) + 1;
    const long long f0 = A.face0[pi];
    auto fidx = [&](int ii, int jj, int kk) { return f0 + ((long long)(kk - 1) * (my + 1) + (jj - 1)) * (mx + 1) + (ii - 1); };
    const long long plane = (long long)P.mitot * P.mjtot * P.mktot;
    const long long at = ((long long)(k - 1 + NG3) * P.mjtot + (j - 1 + NG3)) * P.mitot + (i - 1 + NG3);
    const T* q = static_cast<const T*>(A.pool) + P.q[P.cur];
    T* qn = const_cast<T*>(static_cast<const T*>(A.pool)) + P.q[1 - P.cur];
    const long long c = fidx(i, j, k), cx = fidx(i + 1, j, k), cy = fidx(i, j + 1, k), cz = fidx(i, j, k + 1);
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      const T* F = static_cast<const T*>(A.flux) + (long long)m * fs;
      const T fmv = F[0 * NV * fs + cx], fpv = F[1 * NV * fs + c];
      const T gmv = F[2 * NV * fs + cy], gpv = F[3 * NV * fs + c];
      const T hmv = F[4 * NV * fs + cz], hpv = F[5 * NV * fs + c];
      qn[m * plane + at] = q[m * plane + at] - dtdx * (fmv - fpv) - dtdy * (gmv - gpv) - dtdz * (hmv - hpv);
    }
  }
}

// fluxsv.f:4-94: one register entry per thread
template <class T>
__global__ void fsv3_kernel(const T* flux, long long fs, const long long* face0, const PatchDev* patches, double* regs,
                            const Fsv3* e, int n, int nvar, double dtc, double hx, double hy, double hz, const double* dt_dev) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (dt_dev) dtc = *dt_dev;
  const Fsv3 E = e[t];
  const PatchDev& P = patches[E.patch];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
  auto fidx = [&](int ii, int jj, int kk) { return face0[E.pidx] + ((long long)(kk - 1) * (my + 1) + (jj - 1)) * (mx + 1) + (ii - 1); };
  int comp; long long c; double h1, h2;
  switch (E.side) {
    case 1: comp = 1; c = fidx(E.i, E.j, E.k); h1 = hy; h2 = hz; break;
    case 2: comp = 2; c = fidx(E.i, E.j + 1, E.k); h1 = hx; h2 = hz; break;
    case 3: comp = 0; c = fidx(E.i + 1, E.j, E.k); h1 = hy; h2 = hz; break;
    case 4: comp = 3; c = fidx(E.i, E.j, E.k); h1 = hx; h2 = hz; break;
    case 5: comp = 5; c = fidx(E.i, E.j, E.k); h1 = hx; h2 = hy; break;
    default: comp = 4; c = fidx(E.i, E.j, E.k + 1); h1 = hx; h2 = hy; break;
  }
  for (int m = 0; m < nvar; ++m) regs[E.dst + m] = -(double)flux[((long long)comp * nvar + m) * fs + c] * dtc * h1 * h2;
}

// fluxad.f:4-155: one coarse face (register) of a fine patch per thread
template <class T>
__global__ void fad3_kernel(const T* flux, long long fs, const long long* face0, const PatchDev* patches, double* regs,
                            const Fad3* e, int n, int nvar, double dtf, double hx, double hy, double hz, const double* dt_dev) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (dt_dev) dtf = *dt_dev;
  const Fad3 E = e[t];
  const PatchDev& P = patches[E.patch];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
  auto fidx = [&](int ii, int jj, int kk) { return face0[E.pidx] + ((long long)(kk - 1) * (my + 1) + (jj - 1)) * (mx + 1) + (ii - 1); };
  double* sv = regs + P.ffl + (long long)nvar * E.seg;
  int comp; double h1, h2;
  switch (E.side) {
    case 1: comp = 0; h1 = hy; h2 = hz; break;
    case 2: comp = 3; h1 = hx; h2 = hz; break;
    case 3: comp = 1; h1 = hy; h2 = hz; break;
    case 4: comp = 2; h1 = hx; h2 = hz; break;
    case 5: comp = 4; h1 = hx; h2 = hy; break;
    default: comp = 5; h1 = hx; h2 = hy; break;
  }
  // the fine faces in fluxad.f's order (ob outer, oa inner), loaded FAD_B at a time so
  // the loads are in flight together; the sum keeps that order
  constexpr int FAD_B = 4;
  const int nf = E.na * E.nb;
  for (int m = 0; m < nvar; ++m) {
    double acc = sv[m];
    const T* F = flux + ((long long)comp * nvar + m) * fs;
    for (int u0 = 0; u0 < nf; u0 += FAD_B) {
      T v[FAD_B];
#pragma unroll
      for (int w = 0; w < FAD_B; ++w) {
        v[w] = T(0);
        const int u = u0 + w;
        if (u < nf) {
          const int oa = u % E.na + 1, ob = u / E.na + 1;
          long long c;
          switch (E.side) {
            case 1: c = fidx(1, E.a0 + oa, E.b0 + ob); break;
            case 2: c = fidx(E.a0 + oa, my + 1, E.b0 + ob); break;
            case 3: c = fidx(mx + 1, E.a0 + oa, E.b0 + ob); break;
            case 4: c = fidx(E.a0 + oa, 1, E.b0 + ob); break;
            case 5: c = fidx(E.a0 + oa, E.b0 + ob, 1); break;
            default: c = fidx(E.a0 + oa, E.b0 + ob, mz + 1); break;
          }
          v[w] = __ldg(F + c);  // the fluxes are read-only in this kernel
        }
      }
#pragma unroll
      for (int w = 0; w < FAD_B; ++w)
        if (u0 + w < nf) acc = acc + (double)v[w] * dtf * h1 * h2;
    }
    sv[m] = acc;
  }
}

// qad.f:4-534: one register of one side of a fine patch per group of QAD_G lanes. The
// register sums ratio_a x ratio_b coarse-fine Riemann problems in a fixed order (fine rows
// of the slab outer, cells of the coarse face inner). The group's lanes solve QAD_G of
// them at a time, and the group's first lane adds their two terms per component into the
// register in that order, so the sum is the one a single thread would make.
constexpr int QAD_G = 4;
template <class T>
__global__ void __launch_bounds__(128) qad3_kernel(T* pool, double* regs, const PatchDev* patches, const Qad3Job* jobs, int njobs,
                                                   Step3Params sp, int nvar, double hx, double hy, double hz, double delt,
                                                   const double* dt_dev) {
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(gt % QAD_G), lead = (threadIdx.x & 31) & ~(QAD_G - 1);
  const long long t = gt / QAD_G;
  const bool live = t < njobs;
  if (dt_dev) delt = *dt_dev;
  // lanes past the last job stand in for it with no problems to solve (they still take
  // part in the group shuffles)
  const Qad3Job J = jobs[live ? t : njobs - 1];
  const int n = live ? J.ratio_a * J.ratio_b : 0;
  const int rounds = (int)__reduce_max_sync(0xffffffffu, (unsigned)((n + QAD_G - 1) / QAD_G));
  const PatchDev& P = patches[J.patch];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
  const long long plane = (long long)P.mitot * P.mjtot * P.mktot;
  const T* q = pool + P.q[P.cur];
  auto at = [&](int i, int j, int k) { return ((long long)(k - 1 + NG3) * P.mjtot + (j - 1 + NG3)) * P.mitot + (i - 1 + NG3); };
  double* sv = regs + P.ffl + (long long)nvar * J.reg0;
  T C[6], Fv[6];
  C[0] = T(0); Fv[0] = T(0);
  if (live) {
    const double* qc = regs + P.ffl + (long long)nvar * P.lenbc + (long long)nvar * J.reg0;
    for (int m = 1; m <= 5; ++m) C[m] = (T)qc[m - 1];
  }
  int dir; double sgn, h1, h2;
  switch (J.side) {
    case 1: dir = 1; sgn = 1.0; h1 = hy; h2 = hz; break;
    case 2: dir = 2; sgn = -1.0; h1 = hx; h2 = hz; break;
    case 3: dir = 1; sgn = -1.0; h1 = hy; h2 = hz; break;
    case 4: dir = 2; sgn = 1.0; h1 = hx; h2 = hz; break;
    case 5: dir = 3; sgn = 1.0; h1 = hx; h2 = hy; break;
    default: dir = 3; sgn = -1.0; h1 = hx; h2 = hy; break;
  }
  double acc[5];
  for (int m = 0; m < 5; ++m) acc[m] = (live && lane == 0) ? sv[m] : 0.0;
  for (int rd = 0; rd < rounds; ++rd) {
    const int u = rd * QAD_G + lane;
    double ta[5], tb[5];
    if (u < n) {
      const int ks = u / J.ratio_a + 1, l = u % J.ratio_a + 1;
      const int r = J.row0 + l;                    // fine index along the row, 1-based interior
      const int s = J.slab * J.ratio_b + ks;       // fine index across the rows
      int i, j, k;
      switch (J.side) {
        case 1: i = 0; j = r; k = s; break;
        case 2: i = r; j = my + 1; k = s; break;
        case 3: i = mx + 1; j = r; k = s; break;
        case 4: i = r; j = 0; k = s; break;
        case 5: i = r; j = s; k = 0; break;
        default: i = r; j = s; k = mz + 1; break;
      }
      const long long a = at(i, j, k);
      for (int m = 1; m <= 5; ++m) Fv[m] = q[(m - 1) * plane + a];
      T W[3][5], S[3], amT[5], apT[5];
      const bool low = (J.side == 1 || J.side == 4 || J.side == 5);
      if (low) euler3d_rpn((T)sp.gamma, (T)sp.gamma1, sp.efix != 0, dir, C, Fv, W, S, amT, apT);
      else euler3d_rpn((T)sp.gamma, (T)sp.gamma1, sp.efix != 0, dir, Fv, C, W, S, amT, apT);
      for (int m = 0; m < 5; ++m) {
        const double am = amT[m], ap = apT[m];  // the registers accumulate in FP64
        ta[m] = am * h1 * h2 * delt;
        tb[m] = ap * h1 * h2 * delt;
      }
    } else {
      for (int m = 0; m < 5; ++m) { ta[m] = 0.0; tb[m] = 0.0; }
    }
#pragma unroll
    for (int g = 0; g < QAD_G; ++g) {
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        const double a = __shfl_sync(0xffffffffu, ta[m], lead + g);
        const double b = __shfl_sync(0xffffffffu, tb[m], lead + g);
        if (lane == 0 && rd * QAD_G + g < n) {
          if (sgn > 0.0) acc[m] = acc[m] + a + b;
          else acc[m] = acc[m] - a - b;
        }
      }
    }
  }
  if (live && lane == 0)
    for (int m = 0; m < 5; ++m) sv[m] = acc[m];
}

// qad.f:4-534 for the swirl: the coarse-fine Riemann problem moves the jump with the
// normal face velocity of the fine patch (aux 1..3 are left-face velocities). On the
// low sides that is the first interior fine cell's own face; on the high sides the ghost
// cell beyond, at the cross-row index qad.f reads there (the coarse slab's first fine row
// plus the position l along the coarse face, qad.f:186-193, 245-252, 506-513).
template <class T>
__global__ void qad3_swirl_kernel(T* pool, double* regs, const PatchDev* patches, const Qad3Job* jobs, int njobs,
                                  double hx, double hy, double hz, double delt, const double* dt_dev) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= njobs) return;
  if (dt_dev) delt = *dt_dev;
  const Qad3Job J = jobs[t];
  const PatchDev& P = patches[J.patch];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
  const long long plane = (long long)P.mitot * P.mjtot * P.mktot;
  const T* q = pool + P.q[P.cur];
  const T* aux = pool + P.aux;
  auto at = [&](int i, int j, int k) { return ((long long)(k - 1 + NG3) * P.mjtot + (j - 1 + NG3)) * P.mitot + (i - 1 + NG3); };
  double* sv = regs + P.ffl + J.reg0;
  const T C = (T)regs[P.ffl + P.lenbc + J.reg0];
  double sgn, h1, h2;
  switch (J.side) {
    case 1: case 3: h1 = hy; h2 = hz; break;
    case 2: case 4: h1 = hx; h2 = hz; break;
    default: h1 = hx; h2 = hy; break;
  }
  sgn = (J.side == 1 || J.side == 4 || J.side == 5) ? 1.0 : -1.0;
  double acc = sv[0];
  for (int ks = 1; ks <= J.ratio_b; ++ks) {
    for (int l = 1; l <= J.ratio_a; ++l) {
      const int r = J.row0 + l;
      const int s = J.slab * J.ratio_b + ks;
      const int x = J.slab * J.ratio_b + l;  // qad.f's cross-row index of the high sides
      int i, j, k, ai, aj, ak, comp;
      switch (J.side) {
        case 1: i = 0; j = r; k = s; comp = 0; ai = 1; aj = r; ak = s; break;
        case 2: i = r; j = my + 1; k = s; comp = 1; ai = r; aj = my + 1; ak = x; break;
        case 3: i = mx + 1; j = r; k = s; comp = 0; ai = mx + 1; aj = r; ak = x; break;
        case 4: i = r; j = 0; k = s; comp = 1; ai = r; aj = 1; ak = s; break;
        case 5: i = r; j = s; k = 0; comp = 2; ai = r; aj = s; ak = 1; break;
        default: i = r; j = s; k = mz + 1; comp = 2; ai = r; aj = x; ak = mz + 1; break;
      }
      const T fv = q[at(i, j, k)];
      const T u = aux[comp * plane + at(ai, aj, ak)];
      const T w = (sgn > 0.0) ? fv - C : C - fv;   // right state minus left state
      const double am = dmin(u, T(0)) * w, ap = dmax(u, T(0)) * w;
      if (sgn > 0.0) acc = acc + am * h1 * h2 * delt + ap * h1 * h2 * delt;
      else acc = acc - am * h1 * h2 * delt - ap * h1 * h2 * delt;
    }
  }
  sv[0] = acc;
}

// b4step3 of the time-modulated swirl: aux = aux0 * c over the enlarged patches of plist
// (aux0, the setaux values, sits right after aux in the pool)
template <class T>
__global__ void b4step3_kernel(T* pool, const PatchDev* patches, const int* plist, int np, int naux, double c, const double* c_dev) {
  const int pi = blockIdx.y;
  if (pi >= np) return;
  if (c_dev) c = *c_dev;
  const PatchDev& P = patches[plist[pi]];
  const long long n = (long long)naux * P.mitot * P.mjtot * P.mktot;
  T* a = pool + P.aux;
  const T* a0 = a + n;
  for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x)
    a[x] = (T)((double)a0[x] * c);
}

// ------------------------------------------------------------------- ghost fill
// storage type T (double, or float in the FP32 form); the fill arithmetic is FP64
template <class T>
__device__ __forceinline__ T* fill3_dst(const Fill3Args& a, const Fill3Op& o, int& ni, int& nj, long long& plane) {
  if (o.dst_patch >= 0) {
    const PatchDev& P = a.patches[o.dst_patch];
    ni = P.mitot; nj = P.mjtot; plane = (long long)P.mitot * P.mjtot * P.mktot;
    return static_cast<T*>(a.pool) + P.q[P.cur];
  }
  const Rect3& R = a.rects[o.dst_rect];
  ni = R.ni; nj = R.nj; plane = (long long)R.ni * R.nj * R.nk;
  return static_cast<T*>(a.pool) + R.off;
}

template <class T>
__global__ void fill3_kernel(Fill3Args a) {
  const T* pool = static_cast<const T*>(a.pool);
  const int c = blockIdx.x;
  if (c >= a.nchunks) return;
  const Fill3Chunk ch = a.chunks[c];
  if ((int)threadIdx.x >= ch.count) return;
  const Fill3Op o = a.ops[ch.op];
  const long long cell = ch.start + threadIdx.x;
  const int nvar = a.nvar;
  if (o.kind == F3_RING) {
    // cstore.f:4-96: faces x-left, y-top, x-right, y-bottom, z-bottom, z-top
    const Rect3& R = a.rects[o.src];
    const int nr = R.ni, nc = R.nj, nf = R.nk;
    const long long s13 = (long long)(nf - 2) * (nc - 2), s24 = (long long)(nf - 2) * (nr - 2), s56 = (long long)(nc - 2) * (nr - 2);
    long long k = cell;
    int ii, jj, kk;
    if (k < s13) { ii = 1; kk = 2 + (int)(k / (nc - 2)); jj = 2 + (int)(k % (nc - 2)); }
    else if ((k -= s13) < s24) { jj = nc; kk = 2 + (int)(k / (nr - 2)); ii = 2 + (int)(k % (nr - 2)); }
    else if ((k -= s24) < s13) { ii = nr; kk = 2 + (int)(k / (nc - 2)); jj = 2 + (int)(k % (nc - 2)); }
    else if ((k -= s13) < s24) { jj = 1; kk = 2 + (int)(k / (nr - 2)); ii = 2 + (int)(k % (nr - 2)); }
    else if ((k -= s24) < s56) { kk = 1; jj = 2 + (int)(k / (nr - 2)); ii = 2 + (int)(k % (nr - 2)); }
    else { k -= s56; kk = nf; jj = 2 + (int)(k / (nr - 2)); ii = 2 + (int)(k % (nr - 2)); }
    const PatchDev& K = a.patches[o.dst_patch];
    double* qc1d = a.regs + K.ffl + (long long)nvar * K.lenbc + (long long)nvar * cell;
    const T* src = pool + R.off;
    const long long pl = (long long)nr * nc * nf;
    const long long idx = ((long long)(kk - 1) * nc + (jj - 1)) * nr + (ii - 1);
    for (int m = 0; m < nvar; ++m) qc1d[m] = (double)src[m * pl + idx];
    return;
  }
  const int ia = (int)(cell % o.ni), jb = (int)((cell / o.ni) % o.nj), kc = (int)(cell / ((long long)o.ni * o.nj));
  int dni, dnj; long long plane;
  T* dst = fill3_dst<T>(a, o, dni, dnj, plane);
  const long long dk = ((long long)(o.dk0 + kc) * dnj + (o.dj0 + jb)) * dni + (o.di0 + ia);
  if (o.kind == F3_COPY) {
    const PatchDev& S = a.patches[o.src];
    const long long sp = (long long)S.mitot * S.mjtot * S.mktot;
    const long long sk = ((long long)(o.sk0 + kc) * S.mjtot + (o.sj0 + jb)) * S.mitot + (o.si0 + ia);
    int mode = 0; double ai = 1.0, ac = 0.0;
    if (o.level >= 0) {
      const SrcMode& M = a.modes_dev ? *a.modes_dev : a.modes;
      mode = M.mode[o.level]; ai = M.alphai[o.level]; ac = M.alphac[o.level];
    }
    const T* qn = pool + S.q[S.cur];
    const T* qo = pool + S.q[1 - S.cur];
    for (int m = 0; m < nvar; ++m) {
      double v;
      if (mode == 0) v = (double)qn[m * sp + sk];
      else if (mode == 1) v = (double)qo[m * sp + sk];
      else v = (double)qn[m * sp + sk] * ai + (double)qo[m * sp + sk] * ac;
      dst[m * plane + dk] = (T)v;
    }
    return;
  }
  const Rect3& R = a.rects[o.src];
  const T* vc = pool + R.off;
  const long long cp = (long long)R.ni * R.nj * R.nk;
  if (o.kind == F3_PIECE) {
    const long long sk = ((long long)(o.sk0 + kc) * R.nj + (o.sj0 + jb)) * R.ni + (o.si0 + ia);
    for (int m = 0; m < nvar; ++m) dst[m * plane + dk] = vc[m * cp + sk];
    return;
  }
  auto VC = [&](int m, int i, int j, int k) { return (double)vc[m * cp + ((long long)(k - 1) * R.nj + (j - 1)) * R.ni + (i - 1)]; };
  const int lev = o.level;
  const int rx = a.lc.intratx[lev - 1], ry = a.lc.intraty[lev - 1], rz = a.lc.intratz[lev - 1];
  const int ifg = o.si0 + ia, jfg = o.sj0 + jb, kfg = o.sk0 + kc;
  const int icg = floordiv3(ifg, rx), jcg = floordiv3(jfg, ry), kcg = floordiv3(kfg, rz);
  const int ic = icg - o.cilo + 1, jc = jcg - o.cjlo + 1, kcc = kcg - o.cklo + 1;
  if (o.kind == F3_INTERP) {
    // filpatch.f:182-269 limited trilinear-slope interpolation
    const double hxf = a.lc.hx[lev], hyf = a.lc.hy[lev], hzf = a.lc.hz[lev];
    const double hxc = a.lc.hx[lev - 1], hyc = a.lc.hy[lev - 1], hzc = a.lc.hz[lev - 1];
    const double xlc = a.xlower + o.cilo * hxc, ybc = a.ylower + o.cjlo * hyc, zfc = a.zlower + o.cklo * hzc;
    const double eta1 = ((a.xlower + (ifg + 0.5) * hxf) - (xlc + (ic - 0.5) * hxc)) / hxc;
    const double eta2 = ((a.ylower + (jfg + 0.5) * hyf) - (ybc + (jc - 0.5) * hyc)) / hyc;
    const double eta3 = ((a.zlower + (kfg + 0.5) * hzf) - (zfc + (kcc - 0.5) * hzc)) / hzc;
    for (int m = 0; m < nvar; ++m) {
      const double valp100 = VC(m, ic + 1, jc, kcc), valm100 = VC(m, ic - 1, jc, kcc), valc = VC(m, ic, jc, kcc);
      const double valp010 = VC(m, ic, jc + 1, kcc), valm010 = VC(m, ic, jc - 1, kcc);
      const double valp001 = VC(m, ic, jc, kcc + 1), valm001 = VC(m, ic, jc, kcc - 1);
      const double dupc = valp100 - valc, dumc = valc - valm100, ducc = valp100 - valm100;
      double du = dmin(fabs(dupc), fabs(dumc));
      du = dmin(2.0 * du, 0.5 * fabs(ducc));
      const double fu = dmax(0.0, dsign(1.0, dupc * dumc));
      const double uslope = du * dsign(1.0, ducc) * fu;
      const double dvpc = valp010 - valc, dvmc = valc - valm010, dvcc = valp010 - valm010;
      double dv = dmin(fabs(dvpc), fabs(dvmc));
      dv = dmin(2.0 * dv, 0.5 * fabs(dvcc));
      const double fv = dmax(0.0, dsign(1.0, dvpc * dvmc));
      const double vslope = dv * dsign(1.0, dvcc) * fv;
      const double dwpc = valp001 - valc, dwmc = valc - valm001, dwcc = valp001 - valm001;
      double dw = dmin(fabs(dwpc), fabs(dwmc));
      dw = dmin(2.0 * dw, 0.5 * fabs(dwcc));
      const double fw = dmax(0.0, dsign(1.0, dwpc * dwmc));
      const double wslope = dw * dsign(1.0, dwcc) * fw;
      dst[m * plane + dk] = (T)(valc + eta1 * uslope + eta2 * vslope + eta3 * wslope);
    }
    return;
  }
  // F3_FILVAL: filval.f:84-137 minmod-limited interpolation into a new patch
  const int ico = ifg - icg * rx + 1, jco = jfg - jcg * ry + 1, kco = kfg - kcg * rz + 1;
  const double xoff = ((double)ico - .5) / rx - .5, yoff = ((double)jco - .5) / ry - .5, zoff = ((double)kco - .5) / rz - .5;
  for (int m = 0; m < nvar; ++m) {
    double slp = VC(m, ic + 1, jc, kcc) - VC(m, ic, jc, kcc), slm = VC(m, ic, jc, kcc) - VC(m, ic - 1, jc, kcc);
    double s = dmin(fabs(slp), fabs(slm)) * dsign(1.0, VC(m, ic + 1, jc, kcc) - VC(m, ic - 1, jc, kcc));
    const double dudx = (slm * slp > 0.0) ? s : 0.0;
    slp = VC(m, ic, jc + 1, kcc) - VC(m, ic, jc, kcc); slm = VC(m, ic, jc, kcc) - VC(m, ic, jc - 1, kcc);
    s = dmin(fabs(slp), fabs(slm)) * dsign(1.0, VC(m, ic, jc + 1, kcc) - VC(m, ic, jc - 1, kcc));
    const double dudy = (slm * slp > 0.0) ? s : 0.0;
    slp = VC(m, ic, jc, kcc + 1) - VC(m, ic, jc, kcc); slm = VC(m, ic, jc, kcc) - VC(m, ic, jc, kcc - 1);
    s = dmin(fabs(slp), fabs(slm)) * dsign(1.0, VC(m, ic, jc, kcc + 1) - VC(m, ic, jc, kcc - 1));
    const double dudz = (slm * slp > 0.0) ? s : 0.0;
    dst[m * plane + dk] = (T)(VC(m, ic, jc, kcc) + xoff * dudx + yoff * dudy + zoff * dudz);
  }
}

// One side of a boundary line: ghost cells lo..hi (1-based along the line, element g at
// line[(g-1)*st]) set from the interior. code 1 copies cell s_ext into each; code 3 (wall)
// mirrors cell refl-g into cell g and negates the normal momentum (neg). The sources of a
// side never overlap its ghost cells, so every source is loaded before the first store.
template <class T>
__device__ __forceinline__ void bc3_side(T* line, long long st, int lo, int hi, int code, int s_ext, int refl, bool neg) {
  if (code == 1) {
    const T x = line[(long long)(s_ext - 1) * st];
    for (int g = lo; g <= hi; ++g) line[(long long)(g - 1) * st] = x;
    return;
  }
  constexpr int MAXG = 4;
  const int n = hi - lo + 1;
  if (n <= MAXG) {
    T buf[MAXG];
#pragma unroll
    for (int u = 0; u < MAXG; ++u)
      if (u < n) buf[u] = line[(long long)(refl - (lo + u) - 1) * st];
#pragma unroll
    for (int u = 0; u < MAXG; ++u)
      if (u < n) line[(long long)(lo + u - 1) * st] = neg ? -buf[u] : buf[u];
    return;
  }
  for (int g = lo; g <= hi; ++g) {
    const T x = line[(long long)(refl - g - 1) * st];
    line[(long long)(g - 1) * st] = neg ? -x : x;
  }
}

// bc3amr.f90:70-380. phase 0: x sides per (j,k) row; 1: y sides per (i,k); 2: z sides per
// (i,j). A thread owns one (component, line) pair, lines fastest so that neighbouring
// threads touch neighbouring cells in phases 1 and 2. Within a line the low side is set
// before the high side, as in the reference: the two differ only on a patch narrower than
// its ghost regions, where the high side's mirror reads the low side's ghosts.
template <class T, int phase>
__global__ void __launch_bounds__(128, 8) bc3_kernel(Bc3Args a) {
  const int op = blockIdx.y;
  if (op >= a.nops) return;
  const Bc3Op o = a.ops[op];
  T* v;
  if (o.dst_patch >= 0) { const PatchDev& P = a.patches[o.dst_patch]; v = static_cast<T*>(a.pool) + P.q[P.cur]; }
  else v = static_cast<T*>(a.pool) + a.rects[o.dst_rect].off;
  const int nr = o.nrow, nc = o.ncol, nf = o.nfil;
  const long long plane = (long long)nr * nc * nf;
  const int lines = phase == 0 ? nc * nf : phase == 1 ? nr * nf : nr * nc;
  const long long items = (long long)lines * a.nvar;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < items; t += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(t / lines), l = (int)(t % lines);
    T* base = v + m * plane;
    if constexpr (phase == 0) {
      T* line = base + (long long)l * nr;  // row (j,k) = (l % nc + 1, l / nc + 1)
      if (o.nxl > 0 && (o.bxl == 1 || o.bxl == 3)) bc3_side(line, 1, 1, o.nxl, o.bxl, o.nxl + 1, 2 * o.nxl + 1, o.bxl == 3 && m == 1);
      if (o.ibeg > 0 && (o.bxr == 1 || o.bxr == 3)) bc3_side(line, 1, o.ibeg, nr, o.bxr, o.ibeg - 1, 2 * o.ibeg - 1, o.bxr == 3 && m == 1);
    } else if constexpr (phase == 1) {
      const int i = l % nr, k = l / nr;
      T* line = base + (long long)k * nc * nr + i;
      if (o.nyl > 0 && (o.byl == 1 || o.byl == 3)) bc3_side(line, nr, 1, o.nyl, o.byl, o.nyl + 1, 2 * o.nyl + 1, o.byl == 3 && m == 2);
      if (o.jbeg > 0 && (o.byr == 1 || o.byr == 3)) bc3_side(line, nr, o.jbeg, nc, o.byr, o.jbeg - 1, 2 * o.jbeg - 1, o.byr == 3 && m == 2);
    } else {
      T* line = base + l;  // column (i,j) = (l % nr + 1, l / nr + 1)
      const long long st = (long long)nr * nc;
      if (o.nzl > 0 && (o.bzl == 1 || o.bzl == 3)) bc3_side(line, st, 1, o.nzl, o.bzl, o.nzl + 1, 2 * o.nzl + 1, o.bzl == 3 && m == 3);
      if (o.kbeg > 0 && (o.bzr == 1 || o.bzr == 3)) bc3_side(line, st, o.kbeg, nf, o.bzr, o.kbeg - 1, 2 * o.kbeg - 1, o.bzr == 3 && m == 3);
    }
  }
}

// upbnd.f:4-94: one coarse cell per thread, its terms in listbc order
template <class T>
__global__ void upbnd3_kernel(T* pool, const double* regs, const PatchDev* patches, const Upbnd3Cell* cells, int n,
                              const Upbnd3Term* terms, double volume, int nvar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const Upbnd3Cell c = cells[t];
  const PatchDev& P = patches[c.patch];
  const long long plane = (long long)P.mitot * P.mjtot * P.mktot;
  T* q = pool + P.q[P.cur];
  const long long at = ((long long)c.ke * P.mjtot + c.je) * P.mitot + c.ie;
  for (int m = 0; m < nvar; ++m) {
    double v = (double)q[m * plane + at];
    for (int k = 0; k < c.count; ++k) {
      const Upbnd3Term tm = terms[c.first + k];
      v = v + tm.sgn * regs[tm.reg + m] / volume;
    }
    q[m * plane + at] = (T)v;
  }
}

// update.f:118-178: mean of the fine cells over each covered coarse cell
template <class T>
__global__ void average3_kernel(T* pool, const PatchDev* patches, const Avg3* rects, int n, int rx, int ry, int rz, int nvar) {
  const int r = blockIdx.y;
  if (r >= n) return;
  const Avg3 A = rects[r];
  const PatchDev& C = patches[A.cpatch];
  const PatchDev& F = patches[A.kpatch];
  const long long cpl = (long long)C.mitot * C.mjtot * C.mktot, fpl = (long long)F.mitot * F.mjtot * F.mktot;
  T* qc = pool + C.q[C.cur];
  const T* qf = pool + F.q[F.cur];
  const int totrat = rx * ry * rz;
  const int cells = A.ni * A.nj * A.nk;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cells; t += gridDim.x * blockDim.x) {
    const int a = t % A.ni, b = (t / A.ni) % A.nj, c = t / (A.ni * A.nj);
    const long long cat = ((long long)(A.ck0 + c) * C.mjtot + (A.cj0 + b)) * C.mitot + (A.ci0 + a);
    const int fi = A.fi0 + a * rx, fj = A.fj0 + b * ry, fk = A.fk0 + c * rz;
    for (int m = 0; m < nvar; ++m) {
      double v = 0.0;
      for (int kco = 0; kco < rz; ++kco)
        for (int jco = 0; jco < ry; ++jco)
          for (int ico = 0; ico < rx; ++ico) v = v + (double)qf[m * fpl + ((long long)(fk + kco) * F.mjtot + (fj + jco)) * F.mitot + (fi + ico)];
      qc[m * cpl + cat] = (T)(v / totrat);
    }
  }
}

// gauges_module.f90:376-430 trilinear sample
template <class T>
__global__ void gauges3_kernel(const T* pool, const PatchDev* patches, const Gauge3Job* jobs, int n, int nvar, double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const Gauge3Job J = jobs[t];
  const PatchDev& P = patches[J.patch];
  const long long plane = (long long)P.mitot * P.mjtot * P.mktot;
  const T* q = pool + P.q[P.cur];
  auto Q = [&](int m, int ii, int jj, int kk) { return (double)q[m * plane + ((long long)(kk - 1) * P.mjtot + (jj - 1)) * P.mitot + (ii - 1)]; };
  const double xoff = J.xoff, yoff = J.yoff, zoff = J.zoff;
  const int ii = J.ii, jj = J.jj, kk = J.kk;
  for (int m = 0; m < nvar; ++m) {
    double v = (1.0 - xoff) * (1.0 - yoff) * Q(m, ii, jj, kk) + xoff * (1.0 - yoff) * Q(m, ii + 1, jj, kk) +
               (1.0 - xoff) * yoff * Q(m, ii, jj + 1, kk) + xoff * yoff * Q(m, ii + 1, jj + 1, kk);
    v = v * (1.0 - zoff);
    v = v + zoff * ((1.0 - xoff) * (1.0 - yoff) * Q(m, ii, jj, kk + 1) + xoff * (1.0 - yoff) * Q(m, ii + 1, jj, kk + 1) +
                    (1.0 - xoff) * yoff * Q(m, ii, jj + 1, kk + 1) + xoff * yoff * Q(m, ii + 1, jj + 1, kk + 1));
    out[(long long)J.slot * nvar + m] = v;
  }
}

template <class T>
__global__ void mass3_kernel(const T* pool, const PatchDev* patches, const int* plist, int np, double* out) {
  const int p = blockIdx.y;
  if (p >= np) return;
  const PatchDev& P = patches[plist[p]];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
  const T* q = pool + P.q[P.cur];
  double s = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < mx * my * mz; t += gridDim.x * blockDim.x) {
    const int i = t % mx, j = (t / mx) % my, k = t / (mx * my);
    s += (double)q[((long long)(k + NG3) * P.mjtot + (j + NG3)) * P.mitot + (i + NG3)];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// interior values of the listed patches, [m][k][j][i] per patch: the solution (store1),
// or with aux set the patch's aux array (nvar = naux components)
template <class T>
__global__ void gather3_kernel(const T* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np, int nvar,
                               long long total, double* out, bool aux) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int pi = find_patch(cell0, np, t);
    const PatchDev& P = patches[plist[pi]];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
    const long long n = (long long)mx * my * mz;
    const long long loc = t - cell0[pi];
    const int i = (int)(loc % mx), j = (int)((loc / mx) % my), k = (int)(loc / ((long long)mx * my));
    const long long plane = (long long)P.mitot * P.mjtot * P.mktot;
    const T* q = pool + (aux ? P.aux : P.q[P.cur]);
    const long long at = ((long long)(k + NG3) * P.mjtot + (j + NG3)) * P.mitot + (i + NG3);
    for (int m = 0; m < nvar; ++m) out[cell0[pi] * nvar + m * n + loc] = (double)q[m * plane + at];
  }
}

// The whole arrays (ghost cells included) of the listed patches, q(m,i,j,k) with m fastest
// (the reference's layout), for binary output: enlarged cells [cell0[p], cell0[p+1]) of
// patch p. aux: the aux arrays. Otherwise a cell comes from store1 when the last step wrote
// it there (the interior, or after split steps the cells of interior i) and from the other
// buffer when it did not: that is the step's input, whose ghost cells its fill set (or,
// before any step, the second copy of the initial values, whose ghost cells are zero as
// the reference's are after setgrd.f swaps its stores).
template <class T>
__global__ void gather_enlarged3_kernel(const T* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np,
                                        int nvar, long long total, double* out, bool aux, int split) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int pi = find_patch(cell0, np, t);
    const PatchDev& P = patches[plist[pi]];
    const long long loc = t - cell0[pi];
    const long long mi = P.mitot, mj = P.mjtot, mk = P.mktot, plane = mi * mj * mk;
    const int ie = (int)(loc % mi), je = (int)((loc / mi) % mj), ke = (int)(loc / (mi * mj));
    const bool in_i = ie >= NG3 && ie < mi - NG3, in_j = je >= NG3 && je < mj - NG3, in_k = ke >= NG3 && ke < mk - NG3;
    const bool written = split ? in_i : (in_i && in_j && in_k);
    const T* q = pool + (aux ? P.aux : written ? P.q[P.cur] : P.q[1 - P.cur]);
    for (int m = 0; m < nvar; ++m) out[(cell0[pi] + loc) * nvar + m] = (double)q[m * plane + loc];
  }
}

// fluxad.f / qad.f work lists of a level, from the per-patch segment prefix: segment
// seg of a fine patch is (side, ac, bc) in cstore.f's order (sides 1..6, ac fastest)
__global__ void expand_fadqad3_kernel(const int* plist, const long long* pre, int np, const PatchDev* patches, int rx, int ry,
                                      int rz, long long total, Fad3* fad, Qad3Job* qad) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int pi = find_patch(pre, np, t);
    const int m = plist[pi];
    const PatchDev& P = patches[m];
    const int nxc = (P.ihi - P.ilo + 1) / rx, nyc = (P.jhi - P.jlo + 1) / ry, nzc = (P.khi - P.klo + 1) / rz;
    const int seg = (int)(t - pre[pi]);
    const int cnt[6] = {nyc * nzc, nxc * nzc, nyc * nzc, nxc * nzc, nxc * nyc, nxc * nyc};
    const int nas[6] = {nyc, nxc, nyc, nxc, nxc, nxc};
    const int ras[6] = {ry, rx, ry, rx, rx, rx}, rbs[6] = {rz, rz, rz, rz, ry, ry};
    int side = 0, r = seg;
    while (side < 5 && r >= cnt[side]) { r -= cnt[side]; ++side; }
    const int ac = r % nas[side], bc = r / nas[side];
    const int ra = ras[side], rb = rbs[side];
    fad[t] = Fad3{m, pi, side + 1, ac * ra, bc * rb, ra, rb, seg};
    Qad3Job q;
    q.patch = m; q.side = side + 1; q.slab = bc; q.row0 = ac * ra; q.nreg = 1; q.reg0 = seg; q.ratio_a = ra; q.ratio_b = rb;
    qad[t] = q;
  }
}

int grid_for(long long n, int block) {
  const long long g = (n + block - 1) / block;
  return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 64));
}

}  // namespace

template <class T, class PH>
static void set_sweep_smem() {
  static const bool done = [] {
    constexpr int smem = sweep3_smem_bytes<T, PH>();
    AMR_CUDA(cudaFuncSetAttribute(sweep3_kernel<1, T, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    AMR_CUDA(cudaFuncSetAttribute(sweep3_kernel<2, T, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    AMR_CUDA(cudaFuncSetAttribute(sweep3_kernel<3, T, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return true;
  }();
  (void)done;
}
// the three sweep directions of a level, one launch each: x on s, y and z on the side
// streams (if given) joined back before the face gather
template <class T, class PH>
static int launch_sweeps(const Step3Args& a, const long long items[3], cudaStream_t s, const SweepStreams* ss) {
  auto tiles = [](long long n) { return (unsigned)((n + SW_OWN - 1) / SW_OWN); };
  constexpr int smem = sweep3_smem_bytes<T, PH>();
  set_sweep_smem<T, PH>();
  int n = 0;
  cudaStream_t sy = s, sz = s;
  if (ss) {
    AMR_CUDA(cudaEventRecord(ss->fork, s));
    AMR_CUDA(cudaStreamWaitEvent(ss->side[0], ss->fork, 0));
    AMR_CUDA(cudaStreamWaitEvent(ss->side[1], ss->fork, 0));
    sy = ss->side[0]; sz = ss->side[1];
  }
  if (items[0] > 0) { sweep3_kernel<1, T, PH><<<tiles(items[0]), SW_T, smem, s>>>(a); ++n; }
  if (items[1] > 0) { sweep3_kernel<2, T, PH><<<tiles(items[1]), SW_T, smem, sy>>>(a); ++n; }
  if (items[2] > 0) { sweep3_kernel<3, T, PH><<<tiles(items[2]), SW_T, smem, sz>>>(a); ++n; }
  if (ss) {
    AMR_CUDA(cudaEventRecord(ss->join[0], ss->side[0]));
    AMR_CUDA(cudaEventRecord(ss->join[1], ss->side[1]));
    AMR_CUDA(cudaStreamWaitEvent(s, ss->join[0], 0));
    AMR_CUDA(cudaStreamWaitEvent(s, ss->join[1], 0));
  }
  return n;
}

template <class T, class PH>
static int launch_step3_t(const Step3Args& a, const long long items[3], long long faces, long long cells, cudaStream_t s,
                          const SweepStreams* ss) {
  auto tiles = [](long long n) { return (unsigned)((n + SW_OWN - 1) / SW_OWN); };
  constexpr int smem = sweep3_smem_bytes<T, PH>();
  int n = 0;
  if (a.queue) {
    static const bool smem_set = [] {
      AMR_CUDA(cudaFuncSetAttribute(sweep3_queue_kernel<T, PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      return true;
    }();
    (void)smem_set;
    const unsigned nx = tiles(items[0]), nxy = nx + tiles(items[1]), ntot = nxy + tiles(items[2]);
    if (ntot > 0) {
      // as many blocks as are resident at once (the queue hands out the tiles)
      static const int resident = [] {
        int dev = 0, sms = 0, per_sm = 0;
        AMR_CUDA(cudaGetDevice(&dev));
        AMR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        AMR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep3_queue_kernel<T, PH>, SW_T, smem));
        return std::max(1, sms * per_sm);
      }();
      AMR_CUDA(cudaMemsetAsync(a.queue, 0, sizeof(unsigned int), s));
      sweep3_queue_kernel<T, PH><<<std::min<unsigned>(ntot, (unsigned)resident), SW_T, smem, s>>>(a, nx, nxy, ntot);
      ++n;
    }
  } else {
    n += launch_sweeps<T, PH>(a, items, s, ss);
  }
  AMR_CUDA(cudaGetLastError());
  if (faces > 0) { face3_kernel<T, PH::NV><<<grid_for(faces, 128), 128, 0, s>>>(a); ++n; }
  if (cells > 0) { update3_kernel<T, PH::NV><<<grid_for(cells, 256), 256, 0, s>>>(a); ++n; }
  AMR_CUDA(cudaGetLastError());
  return n;
}
template <class T, class PH>
static int launch_split3_t(const Step3Args& a, const long long items[3], cudaStream_t s) {
  auto tiles = [](long long n) { return (unsigned)((n + SW_OWN - 1) / SW_OWN); };
  int n = 0;
  if (items[0] > 0) { split3_kernel<1, T, PH><<<tiles(items[0]), SW_T, 0, s>>>(a); ++n; }
  if (items[1] > 0) { split3_kernel<2, T, PH><<<tiles(items[1]), SW_T, 0, s>>>(a); ++n; }
  if (items[2] > 0) { split3_kernel<3, T, PH><<<tiles(items[2]), SW_T, 0, s>>>(a); ++n; }
  AMR_CUDA(cudaGetLastError());
  return n;
}
int launch_split3(const Step3Args& a, const long long items[3], cudaStream_t s, bool f32) {
  if (a.sp.solver == SOLVER3_SWIRL) {
    if (f32) return launch_split3_t<float, Swirl3Phys<float>>(a, items, s);
    return launch_split3_t<double, Swirl3Phys<double>>(a, items, s);
  }
  if (f32) return launch_split3_t<float, Euler3Phys<float>>(a, items, s);
  return launch_split3_t<double, Euler3Phys<double>>(a, items, s);
}

int launch_step3(const Step3Args& a, const long long items[3], long long faces, long long cells, cudaStream_t s, bool f32,
                 const SweepStreams* ss) {
  if (a.sp.solver == SOLVER3_SWIRL) {
    if (f32) return launch_step3_t<float, Swirl3Phys<float>>(a, items, faces, cells, s, ss);
    return launch_step3_t<double, Swirl3Phys<double>>(a, items, faces, cells, s, ss);
  }
  if (f32) return launch_step3_t<float, Euler3Phys<float>>(a, items, faces, cells, s, ss);
  return launch_step3_t<double, Euler3Phys<double>>(a, items, faces, cells, s, ss);
}

void launch_expand_fadqad3(const int* plist, const long long* pre, int np, const PatchDev* patches, int rx, int ry, int rz,
                           long long total, Fad3* fad, Qad3Job* qad, cudaStream_t s) {
  if (total <= 0) return;
  expand_fadqad3_kernel<<<grid_for(total, 256), 256, 0, s>>>(plist, pre, np, patches, rx, ry, rz, total, fad, qad);
  AMR_CUDA(cudaGetLastError());
}

void launch_fsv3(const void* flux, long long fs, const long long* face0, const PatchDev* patches, double* regs, const Fsv3* e, int n,
                 int nvar, double dtc, double hx, double hy, double hz, cudaStream_t s, bool f32, const double* dt_dev) {
  if (n <= 0) return;
  if (f32) fsv3_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<const float*>(flux), fs, face0, patches, regs, e, n, nvar, dtc, hx, hy, hz, dt_dev);
  else fsv3_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<const double*>(flux), fs, face0, patches, regs, e, n, nvar, dtc, hx, hy, hz, dt_dev);
  AMR_CUDA(cudaGetLastError());
}
void launch_fad3(const void* flux, long long fs, const long long* face0, const PatchDev* patches, double* regs, const Fad3* e, int n,
                 int nvar, double dtf, double hx, double hy, double hz, cudaStream_t s, bool f32, const double* dt_dev) {
  if (n <= 0) return;
  if (f32) fad3_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<const float*>(flux), fs, face0, patches, regs, e, n, nvar, dtf, hx, hy, hz, dt_dev);
  else fad3_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<const double*>(flux), fs, face0, patches, regs, e, n, nvar, dtf, hx, hy, hz, dt_dev);
  AMR_CUDA(cudaGetLastError());
}
void launch_qad3(void* pool, double* regs, const PatchDev* patches, const Qad3Job* jobs, int njobs, Step3Params sp, int nvar,
                 double hx, double hy, double hz, double delt, cudaStream_t s, bool f32, const double* dt_dev) {
  if (njobs <= 0) return;
  if (sp.solver == SOLVER3_SWIRL) {
    if (f32) qad3_swirl_kernel<<<(njobs + 127) / 128, 128, 0, s>>>(static_cast<float*>(pool), regs, patches, jobs, njobs, hx, hy, hz, delt, dt_dev);
    else qad3_swirl_kernel<<<(njobs + 127) / 128, 128, 0, s>>>(static_cast<double*>(pool), regs, patches, jobs, njobs, hx, hy, hz, delt, dt_dev);
    AMR_CUDA(cudaGetLastError());
    return;
  }
  const long long nthr = (long long)njobs * QAD_G;
  const unsigned nb = (unsigned)((nthr + 127) / 128);
  if (f32) qad3_kernel<<<nb, 128, 0, s>>>(static_cast<float*>(pool), regs, patches, jobs, njobs, sp, nvar, hx, hy, hz, delt, dt_dev);
  else qad3_kernel<<<nb, 128, 0, s>>>(static_cast<double*>(pool), regs, patches, jobs, njobs, sp, nvar, hx, hy, hz, delt, dt_dev);
  AMR_CUDA(cudaGetLastError());
}
template <class T>
__global__ void setaux3_kernel(T* pool, const Setaux3Job* jobs, int njobs, const double* fac, int copies) {
  const int jb = blockIdx.y;
  if (jb >= njobs) return;
  const Setaux3Job J = jobs[jb];
  const long long pl = (long long)J.mi * J.mj * J.mk;
  const double* ua = fac + J.f0;
  const double *va = ua + J.mi, *wa = va + J.mi, *ub = wa + J.mi, *vb = ub + J.mj, *wb = vb + J.mj;
  const double *uc = wb + J.mj, *vc = uc + J.mk, *wc = vc + J.mk;
  T* a = pool + J.aux;
  for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < pl; x += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(x % J.mi), j = (int)((x / J.mi) % J.mj), k = (int)(x / ((long long)J.mi * J.mj));
    const double u = ua[i] * ub[j] * uc[k], v = va[i] * vb[j] * vc[k], w = wa[i] * wb[j] * wc[k];
    for (int c = 0; c < copies; ++c) {
      T* o = a + (long long)c * 3 * pl;
      o[x] = (T)u; o[pl + x] = (T)v; o[2 * pl + x] = (T)w;
    }
  }
}
void launch_setaux3(void* pool, const Setaux3Job* jobs, int njobs, long long max_cells, const double* fac, int copies,
                    cudaStream_t s, bool f32) {
  if (njobs <= 0) return;
  const int bx = (int)std::max<long long>(1, std::min<long long>((max_cells + 255) / 256, 1024));
  for (int base = 0; base < njobs; base += 65535) {
    const int cnt = std::min(65535, njobs - base);
    if (f32) setaux3_kernel<<<dim3(bx, cnt), 256, 0, s>>>(static_cast<float*>(pool), jobs + base, cnt, fac, copies);
    else setaux3_kernel<<<dim3(bx, cnt), 256, 0, s>>>(static_cast<double*>(pool), jobs + base, cnt, fac, copies);
  }
  AMR_CUDA(cudaGetLastError());
}

// valout.f90:140-147: |q| < 1e-90 of the interior cells of plist set to 0 in place
template <class T>
__global__ void zero_tiny3_kernel(T* pool, const PatchDev* patches, const int* plist, int np, int nvar, bool aux) {
  const int pi = blockIdx.y;
  if (pi >= np) return;
  const PatchDev& P = patches[plist[pi]];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1, mz = P.khi - P.klo + 1;
  const long long plane = (long long)P.mitot * P.mjtot * P.mktot, n = (long long)mx * my * mz;
  T* q = pool + (aux ? P.aux : P.q[P.cur]);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n * nvar; t += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(t / n);
    const long long c = t - (long long)m * n;
    const int i = (int)(c % mx), j = (int)((c / mx) % my), k = (int)(c / ((long long)mx * my));
    T& v = q[m * plane + ((long long)(k + NG3) * P.mjtot + (j + NG3)) * P.mitot + (i + NG3)];
    if (fabs((double)v) < 1e-90) v = T(0);
  }
}
void launch_zero_tiny3(void* pool, const PatchDev* patches, const int* plist, int np, int nvar, cudaStream_t s, bool f32,
                       bool aux) {
  for (int base = 0; base < np; base += 65535) {
    const int cnt = std::min(65535, np - base);
    if (f32) zero_tiny3_kernel<<<dim3(8, cnt), 256, 0, s>>>(static_cast<float*>(pool), patches, plist + base, cnt, nvar, aux);
    else zero_tiny3_kernel<<<dim3(8, cnt), 256, 0, s>>>(static_cast<double*>(pool), patches, plist + base, cnt, nvar, aux);
  }
  AMR_CUDA(cudaGetLastError());
}
void launch_b4step3(void* pool, const PatchDev* patches, const int* plist, int np, int naux, long long max_cells, double c,
                    cudaStream_t s, bool f32, const double* c_dev) {
  if (np <= 0) return;
  const int bx = (int)std::max<long long>(1, std::min<long long>((naux * max_cells + 255) / 256, 1024));
  for (int base = 0; base < np; base += 65535) {
    const int cnt = std::min(65535, np - base);
    if (f32) b4step3_kernel<<<dim3(bx, cnt), 256, 0, s>>>(static_cast<float*>(pool), patches, plist + base, cnt, naux, c, c_dev);
    else b4step3_kernel<<<dim3(bx, cnt), 256, 0, s>>>(static_cast<double*>(pool), patches, plist + base, cnt, naux, c, c_dev);
  }
  AMR_CUDA(cudaGetLastError());
}
void launch_fill3(const Fill3Args& a, cudaStream_t s, bool f32) {
  if (a.nchunks <= 0) return;
  for (int base = 0; base < a.nchunks; base += 1 << 30) {
    Fill3Args b = a;
    b.chunks = a.chunks + base;
    b.nchunks = std::min(1 << 30, a.nchunks - base);
    if (f32) fill3_kernel<float><<<b.nchunks, 128, 0, s>>>(b);
    else fill3_kernel<double><<<b.nchunks, 128, 0, s>>>(b);
  }
  AMR_CUDA(cudaGetLastError());
}
// max_lines: the largest number of boundary lines an op of this phase has (nc*nf, nr*nf or
// nr*nc); a row of blocks per op covers them, one (component, line) pair per thread
void launch_bc3(const Bc3Args& a, int phase, cudaStream_t s, bool f32, long long max_lines) {
  if (a.nops <= 0) return;
  const int bx = (int)std::max<long long>(1, std::min<long long>((max_lines * a.nvar + 127) / 128, 1024));
  for (int base = 0; base < a.nops; base += 65535) {
    Bc3Args b = a;
    b.ops = a.ops + base;
    b.nops = std::min(65535, a.nops - base);
    const dim3 g(bx, b.nops);
    if (phase == 0) f32 ? bc3_kernel<float, 0><<<g, 128, 0, s>>>(b) : bc3_kernel<double, 0><<<g, 128, 0, s>>>(b);
    else if (phase == 1) f32 ? bc3_kernel<float, 1><<<g, 128, 0, s>>>(b) : bc3_kernel<double, 1><<<g, 128, 0, s>>>(b);
    else f32 ? bc3_kernel<float, 2><<<g, 128, 0, s>>>(b) : bc3_kernel<double, 2><<<g, 128, 0, s>>>(b);
  }
  AMR_CUDA(cudaGetLastError());
}
void launch_upbnd3(void* pool, const double* regs, const PatchDev* patches, const Upbnd3Cell* cells, int n, const Upbnd3Term* terms,
                   double volume, int nvar, cudaStream_t s, bool f32) {
  if (n <= 0) return;
  if (f32) upbnd3_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<float*>(pool), regs, patches, cells, n, terms, volume, nvar);
  else upbnd3_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<double*>(pool), regs, patches, cells, n, terms, volume, nvar);
  AMR_CUDA(cudaGetLastError());
}
void launch_average3(void* pool, const PatchDev* patches, const Avg3* r, int n, long long max_cells, int rx, int ry, int rz, int nvar,
                     cudaStream_t s, bool f32) {
  if (n <= 0) return;
  const int bx = (int)std::max<long long>(1, std::min<long long>((max_cells + 127) / 128, 1024));
  for (int base = 0; base < n; base += 65535) {
    const int cnt = std::min(65535, n - base);
    if (f32) average3_kernel<<<dim3(bx, cnt), 128, 0, s>>>(static_cast<float*>(pool), patches, r + base, cnt, rx, ry, rz, nvar);
    else average3_kernel<<<dim3(bx, cnt), 128, 0, s>>>(static_cast<double*>(pool), patches, r + base, cnt, rx, ry, rz, nvar);
  }
  AMR_CUDA(cudaGetLastError());
}
void launch_gauges3(const void* pool, const PatchDev* patches, const Gauge3Job* jobs, int n, int nvar, double* out, cudaStream_t s,
                    bool f32) {
  if (n <= 0) return;
  if (f32) gauges3_kernel<<<(n + 63) / 64, 64, 0, s>>>(static_cast<const float*>(pool), patches, jobs, n, nvar, out);
  else gauges3_kernel<<<(n + 63) / 64, 64, 0, s>>>(static_cast<const double*>(pool), patches, jobs, n, nvar, out);
  AMR_CUDA(cudaGetLastError());
}
void launch_mass3(const void* pool, const PatchDev* patches, const int* plist, int np, double* out, cudaStream_t s, bool f32) {
  if (np <= 0) return;
  for (int base = 0; base < np; base += 65535) {
    const int cnt = std::min(65535, np - base);
    if (f32) mass3_kernel<<<dim3(8, cnt), 128, 0, s>>>(static_cast<const float*>(pool), patches, plist + base, cnt, out);
    else mass3_kernel<<<dim3(8, cnt), 128, 0, s>>>(static_cast<const double*>(pool), patches, plist + base, cnt, out);
  }
  AMR_CUDA(cudaGetLastError());
}
void launch_gather_enlarged3(const void* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np, int nvar,
                             long long total, double* out, bool aux, int split, cudaStream_t s, bool f32) {
  if (total <= 0) return;
  if (f32) gather_enlarged3_kernel<<<grid_for(total, 256), 256, 0, s>>>(static_cast<const float*>(pool), patches, plist, cell0, np, nvar, total, out, aux, split);
  else gather_enlarged3_kernel<<<grid_for(total, 256), 256, 0, s>>>(static_cast<const double*>(pool), patches, plist, cell0, np, nvar, total, out, aux, split);
  AMR_CUDA(cudaGetLastError());
}
void launch_gather3(const void* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np, int nvar,
                    long long total, double* out, cudaStream_t s, bool f32, bool aux) {
  if (total <= 0) return;
  if (f32) gather3_kernel<<<grid_for(total, 256), 256, 0, s>>>(static_cast<const float*>(pool), patches, plist, cell0, np, nvar, total, out, aux);
  else gather3_kernel<<<grid_for(total, 256), 256, 0, s>>>(static_cast<const double*>(pool), patches, plist, cell0, np, nvar, total, out, aux);
  AMR_CUDA(cudaGetLastError());
}

}  // namespace amrb
