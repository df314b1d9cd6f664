// 2D kernels of the patch-advance path (sm_100a, FP64, built without FMA contraction).
//
//   step2_kernel   fused patch step: Riemann solves, wave limiter, second-order and
//                  transverse corrections, flux differencing, CFL reduction, and the
//                  flux-register epilogue (fluxsv on coarse faces, fluxad on fine
//                  boundary faces). Replaces stepgrid/step2/flux2/limiter/fluxsv/fluxad
//                  (src/2d/stepgrid.f:24-232, step2.f90:7-169, flux2.f:25-237,
//                  inlinelimiter.f:4-108, fluxsv.f:10-109, fluxad.f:7-96).
//   fill_kernel    ghost-fill op executor: same-level copies with time interpolation,
//                  limited coarse interpolation, periodic pieces, new-grid filval
//                  interpolation and the cstore ring (intfil.f90, filpatch.f90:246-327,
//                  prefilp.f90, filval.f90:150-185, cstore.f).
//   bc kernels     bc2amr.f90 extrapolation / wall in two phases (x then y).
//   qad2_kernel    coarse/fine interface Riemann problems (qad.f:9-360).
//   upbnd/average  level sync (upbnd.f:18-127, update.f:95-175).
#include "kernels2d.cuh"
#include <algorithm>

namespace amrb {

__device__ __forceinline__ int floordiv(int a, int b) { int q = a / b; if ((a % b != 0) && ((a < 0) != (b < 0))) --q; return q; }

// ------------------------------------------------------------------ bulk-copy staging
// The tile rows reach shared memory through the TMA engine's untiled bulk copy
// (cp.async.bulk global -> shared, completion counted in bytes on an mbarrier). A bulk copy
// wants 16-byte aligned source and destination and a multiple of 16 bytes: each row is
// copied from its start rounded down to 16 bytes to its end rounded up, into a staging row
// of RW elements, and read from the element offset the rounding left. The pool's blocks are
// 256-byte aligned and sized in whole 256-byte granules, so the widened rows stay inside
// the row's own block.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// waits for the phase with the given parity, at most about a second of SM clock
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > 2000000000LL) return false;
  return true;
}
// elements of a staging row: the widest row (QW) plus the rounding on both ends
template <class R, int QW>
__host__ __device__ constexpr int stage_row() {
  constexpr int E = 16 / (int)sizeof(R);
  return (QW + 2 * (E - 1) + E - 1) / E * E;
}

// ======================================================================= patch step
template <class S>
struct Step2Layout {
  static constexpr int ME = S::MEQN, MW = S::MWAVES;
  static constexpr int T = TILE2;
  static constexpr int QW = T + 4;
  static constexpr int NQ = ME * QW * QW;
  static constexpr int NF = ME * (T + 1) * T;
  static constexpr int NTR = (T + 2) * T * 2 * ME;
  static constexpr int WREC = MW * ME + MW + 2 * ME;
  static constexpr int NW = STEP2_RC * (T + 3) * WREC;
  static constexpr int XREC = 4 * ME;
  static constexpr int NX = STEP2_RC * (T + 1) * XREC;
  // aux of the tile and its two ghost layers, [m][b][a] like the staged q (solvers that read aux)
  static constexpr int NA = S::NAUX > 0 ? MAXAUX2 : 0;
  static constexpr int NAQ = NA * QW * QW;
  static constexpr int TOTAL = NQ + 4 * NF + NTR + NW + NX + NAQ + 32;
};

// aux values a plugin reads at one cell of a staged aux tile ([m][b][a], QW x QW)
template <class S, class R>
struct AuxCell {
  R v[S::NAUX > 0 ? S::NAUX : 1];
  __device__ __forceinline__ void load(const R* As, int QW, int b, int a) {
#pragma unroll
    for (int m = 0; m < S::NAUX; ++m) v[m] = As[(m * QW + b) * QW + a];
  }
};

// flux2.f:136-194 at one face from the wave records (waves, speeds, amdq, apdq) of the face
// (rc) and of its neighbours (rm: face f-1, rp: face f+1): limiter.f's limited waves, the
// second-order correction cqxx, fm = (0 + amdq) + cqxx/2 and fp = (0 - apdq) + cqxx/2
// dl, dr: dtdx1d of the cells left and right of the face (dt/dx, divided by the capacity of
// the cell when there is one: step2.f90:83-88)
template <class S, class R>
__device__ __forceinline__ void face_fluxes(const StepParams& sp, const R* rm, const R* rc, const R* rp, R dl, R dr,
                                            R (&amdq)[S::MEQN], R (&apdq)[S::MEQN], R (&cqxx)[S::MEQN],
                                            R (&fm)[S::MEQN], R (&fp)[S::MEQN]) {
  constexpr int ME = S::MEQN, MW = S::MWAVES;
#pragma unroll
  for (int m = 0; m < ME; ++m) { amdq[m] = rc[MW * ME + MW + m]; apdq[m] = rc[MW * ME + MW + ME + m]; }
#pragma unroll
  for (int m = 0; m < ME; ++m) { fm[m] = R(0) + amdq[m]; fp[m] = R(0) - apdq[m]; cqxx[m] = R(0); }
  if (sp.order == 1) return;
  R wl[MW][ME];
#pragma unroll
  for (int mw = 0; mw < MW; ++mw) {
    const R smw = rc[MW * ME + mw];
#pragma unroll
    for (int m = 0; m < ME; ++m) wl[mw][m] = rc[mw * ME + m];
    if (sp.mthlim[mw] == 0) continue;
    R wn2 = R(0), dotl = R(0), dotr = R(0);
#pragma unroll
    for (int m = 0; m < ME; ++m) {
      wn2 = wn2 + rc[mw * ME + m] * rc[mw * ME + m];
      dotl = dotl + rm[mw * ME + m] * rc[mw * ME + m];
      dotr = dotr + rc[mw * ME + m] * rp[mw * ME + m];
    }
    if (wn2 == R(0)) continue;
    const R r = (smw > R(0)) ? dotl / wn2 : dotr / wn2;
    R wlim = R(0);
    switch (sp.mthlim[mw]) {
      case 1: wlim = dmax(R(0), dmin(R(1), r)); break;
      case 2: wlim = dmax(R(0), dmax(dmin(R(1), R(2) * r), dmin(R(2), r))); break;
      case 3: wlim = (r + fabs(r)) / (R(1) + fabs(r)); break;
      case 4: { const R c = (R(1) + r) / R(2); wlim = dmax(R(0), dmin(c, dmin(R(2), R(2) * r))); } break;
      case 5: wlim = r; break;
    }
#pragma unroll
    for (int m = 0; m < ME; ++m) wl[mw][m] = wlim * wl[mw][m];
  }
  const R dtdxave = R(0.5) * (dl + dr);
#pragma unroll
  for (int m = 0; m < ME; ++m) {
    R c = R(0);
#pragma unroll
    for (int mw = 0; mw < MW; ++mw) {
      const R smw = rc[MW * ME + mw];
      const R abs_sign = sp.use_fwaves ? dsign(R(1), smw) : fabs(smw);
      c = c + abs_sign * (R(1) - fabs(smw) * dtdxave) * wl[mw][m];
    }
    cqxx[m] = c;
    fm[m] = fm[m] + R(0.5) * c;
    fp[m] = fp[m] + R(0.5) * c;
  }
}

// rpn2 at one face into its wave record: waves [MW][ME], speeds [MW], amdq [ME], apdq [ME].
// auxL, auxR: aux of the cells left and right of the face; dl, dr: their dtdx1d (flux2.f's
// Courant number takes dtdx1d(i)*s and -dtdx1d(i-1)*s)
template <class S, class R>
__device__ __forceinline__ void face_record(const StepParams& sp, int ixy, const R* qL, const R* qR, const R* auxL,
                                            const R* auxR, R* rec, R dl, R dr, bool count_cfl, R& cfl) {
  constexpr int ME = S::MEQN, MW = S::MWAVES;
  R wave[MW][ME], s[MW], amdq[ME], apdq[ME];
  S::template rpn<R>(sp.prob, ixy, qL, qR, auxL, auxR, wave, s, amdq, apdq);
#pragma unroll
  for (int mw = 0; mw < MW; ++mw) {
#pragma unroll
    for (int m = 0; m < ME; ++m) rec[mw * ME + m] = wave[mw][m];
    rec[MW * ME + mw] = s[mw];
  }
#pragma unroll
  for (int m = 0; m < ME; ++m) { rec[MW * ME + MW + m] = amdq[m]; rec[MW * ME + MW + ME + m] = apdq[m]; }
  if (count_cfl) {
#pragma unroll
    for (int mw = 0; mw < MW; ++mw) cfl = dmax(cfl, dmax(dr * s[mw], -dl * s[mw]));
  }
}

// One sweep direction of flux2.f over the tile. IXY = 1: lines are rows, IXY = 2: columns.
// As: the staged aux tile (Step2Layout::NA components, null without aux)
template <class S, int IXY, class R>
__device__ void step2_sweep(const StepParams& sp, const R* Qs, const R* As, R* W, R* X, R* TR, R* F1,
                            R* F2, int i0, int j0, int tw, int th, R dtdx, R& cfl) {
  using L = Step2Layout<S>;
  constexpr int ME = L::ME, T = L::T, QW = L::QW;
  const bool capa = L::NA > 0 && sp.mcapa > 0;
  const int tid = threadIdx.x;
  // along-line extents
  const int na = (IXY == 1) ? tw : th;       // cells along the line inside the tile
  const int nl = (IXY == 1) ? th + 2 : tw + 2;  // lines: tile +-1
  const int a0 = (IXY == 1) ? i0 : j0;        // first tile cell along the line
  const int l0 = (IXY == 1) ? j0 - 1 : i0 - 1;  // first line
  const int nfr = na + 3;                     // faces for the normal solve: a0-1 .. a0+na+1
  const int nfl = na + 1;                     // limited faces: a0 .. a0+na
  auto qptr = [&](int m, int line, int pos) -> const R* {
    // returns &Q(m, ...) ; Q layout [m][b][a] with a = i-(i0-2), b = j-(j0-2)
    if (IXY == 1) return &Qs[(m * QW + (line - (j0 - 2))) * QW + (pos - (i0 - 2))];
    return &Qs[(m * QW + (pos - (j0 - 2))) * QW + (line - (i0 - 2))];
  };
  auto loadq = [&](R* q, int line, int pos) {
#pragma unroll
    for (int m = 0; m < ME; ++m) q[m] = *qptr(m, line, pos);
  };
  // staged aux coordinates (b, a) of a cell of the sweep, as qptr
  auto abt = [&](int line, int pos) { return (IXY == 1) ? line - (j0 - 2) : pos - (j0 - 2); };
  auto aat = [&](int line, int pos) { return (IXY == 1) ? pos - (i0 - 2) : line - (i0 - 2); };
  auto auxc = [&](AuxCell<S, R>& c, int line, int pos) { if (S::NAUX > 0) c.load(As, QW, abt(line, pos), aat(line, pos)); };
  // dtdx1d of a cell (step2.f90:83-88)
  auto d1d = [&](int line, int pos) -> R {
    if (!capa) return dtdx;
    return dtdx / As[((sp.mcapa - 1) * QW + abt(line, pos)) * QW + aat(line, pos)];
  };
  for (int lc0 = 0; lc0 < nl; lc0 += STEP2_RC) {
    const int nlc = min(STEP2_RC, nl - lc0);
    // phase 1: normal Riemann problems
    for (int it = tid; it < nlc * nfr; it += STEP2_THREADS) {
      const int rr = it / nfr, ff = it % nfr;
      const int line = l0 + lc0 + rr, f = a0 - 1 + ff;
      R qL[ME], qR[ME];
      loadq(qL, line, f - 1);
      loadq(qR, line, f);
      AuxCell<S, R> aL, aR;
      auxc(aL, line, f - 1);
      auxc(aR, line, f);
      face_record<S, R>(sp, IXY, qL, qR, aL.v, aR.v, W + (rr * (T + 3) + ff) * L::WREC, d1d(line, f - 1), d1d(line, f),
                        ff >= 1 && ff <= nfl, cfl);
    }
    __syncthreads();
    // phase 2: limiter, second-order correction, transverse splitting
    for (int it = tid; it < nlc * nfl; it += STEP2_THREADS) {
      const int rr = it / nfl, fa = it % nfl;
      const int line = l0 + lc0 + rr, f = a0 + fa;
      const R* rm = W + (rr * (T + 3) + fa) * L::WREC;       // face f-1
      const R* rc = rm + L::WREC;                             // face f
      const R* rp = rc + L::WREC;                             // face f+1
      R amdq[ME], apdq[ME], cqxx[ME], fm[ME], fp[ME];
      const R dl = d1d(line, f - 1), dr = d1d(line, f);
      face_fluxes<S, R>(sp, rm, rc, rp, dl, dr, amdq, apdq, cqxx, fm, fp);
      // flux increments into the tile's face arrays (interior lines only)
      const int lin = (IXY == 1) ? line - j0 : line - i0;
      if (lin >= 0 && lin < ((IXY == 1) ? th : tw)) {
        if (IXY == 1) {
#pragma unroll
          for (int m = 0; m < ME; ++m) {
            F1[(m * T + lin) * (T + 1) + fa] = fm[m];   // FM init
            F2[(m * T + lin) * (T + 1) + fa] = fp[m];   // FP init
          }
        } else {
#pragma unroll
          for (int m = 0; m < ME; ++m) {
            F1[(m * (T + 1) + fa) * T + lin] = F1[(m * (T + 1) + fa) * T + lin] + fm[m];  // GM += faddm
            F2[(m * (T + 1) + fa) * T + lin] = F2[(m * (T + 1) + fa) * T + lin] + fp[m];  // GP += faddp
          }
        }
      }
      R* xr = X + (rr * (T + 1) + fa) * L::XREC;
      if (sp.trans != 0) {
        R am2[ME], ap2[ME];
#pragma unroll
        for (int m = 0; m < ME; ++m) {
          am2[m] = amdq[m]; ap2[m] = apdq[m];
          if (sp.order > 1 && sp.trans == 2) { am2[m] = amdq[m] + cqxx[m]; ap2[m] = apdq[m] - cqxx[m]; }
        }
        R qL[ME], qR[ME];
        loadq(qL, line, f - 1);
        loadq(qR, line, f);
        // the aux of the split's cell (f-1 for amdq, f for apdq) in the rows below, at and above
        AuxCell<S, R> b1, b2, b3, c1, c2, c3;
        auxc(b1, line - 1, f - 1); auxc(b2, line, f - 1); auxc(b3, line + 1, f - 1);
        auxc(c1, line - 1, f); auxc(c2, line, f); auxc(c3, line + 1, f);
        R bm1[ME], bp1[ME], bm2[ME], bp2[ME];
        S::template rpt<R>(sp.prob, IXY, 1, qL, qR, b1.v, b2.v, b3.v, am2, bm1, bp1);
        S::template rpt<R>(sp.prob, IXY, 2, qL, qR, c1.v, c2.v, c3.v, ap2, bm2, bp2);
#pragma unroll
        for (int m = 0; m < ME; ++m) {
          xr[0 * ME + m] = R(0.5) * dl * bm1[m];
          xr[1 * ME + m] = R(0.5) * dl * bp1[m];
          xr[2 * ME + m] = R(0.5) * dr * bm2[m];
          xr[3 * ME + m] = R(0.5) * dr * bp2[m];
        }
      }
    }
    __syncthreads();
    // phase 3: per-cell transverse parts (gadd(:,i,1) and gadd(:,i,2) of flux2.f)
    if (sp.trans != 0) {
      for (int it = tid; it < nlc * na; it += STEP2_THREADS) {
        const int rr = it / na, ca = it % na;
        const R* xa = X + (rr * (T + 1) + ca + 1) * L::XREC;  // face c+1 (amdq part)
        const R* xb = X + (rr * (T + 1) + ca) * L::XREC;      // face c   (apdq part)
        R* tr = TR + (((lc0 + rr) * T + ca) * 2) * ME;
#pragma unroll
        for (int m = 0; m < ME; ++m) {
          tr[m] = (R(0) - xa[0 * ME + m]) - xb[2 * ME + m];
          tr[ME + m] = (R(0) - xa[1 * ME + m]) - xb[3 * ME + m];
        }
      }
    } else {
      for (int it = tid; it < nlc * na; it += STEP2_THREADS) {
        const int rr = it / na, ca = it % na;
        R* tr = TR + (((lc0 + rr) * T + ca) * 2) * ME;
#pragma unroll
        for (int m = 0; m < ME; ++m) { tr[m] = R(0); tr[ME + m] = R(0); }
      }
    }
    __syncthreads();
  }
}

// The flux-register epilogue of a tile (fluxsv.f:10-109 on coarse faces next to finer grids,
// fluxad.f:7-96 on this patch's fine boundary faces). FM, FP: [ME][xrows][T+1] x-faces of
// the tile's rows starting at row 0 of FM / FP; GM, GP: [ME][T+1][T] y-faces. Register
// values stay FP64 in both forms.
template <int ME, class R>
__device__ __forceinline__ void register_epilogue(const StepArgs& a, const StepWork& wk, const PatchDev& P, int i0, int j0,
                                                  int tw, int th, double dt, const R* FM, const R* FP, const R* GM,
                                                  const R* GP, int xrows) {
  constexpr int T = TILE2;
  const int tid = threadIdx.x;
  for (int it = tid; it < wk.fsv_count * ME; it += STEP2_THREADS) {
    const FsvEntry e = a.fsv[wk.fsv_start + it / ME];
    const int m = it % ME;
    const int ca = e.ic - i0, rb = e.jc - j0;
    double v = 0.0;
    if (e.side == 1) v = -(double)FP[(m * xrows + rb) * (T + 1) + ca] * dt * a.dy;
    else if (e.side == 2) v = -(double)GM[(m * (T + 1) + rb + 1) * T + ca] * dt * a.dx;
    else if (e.side == 3) v = -(double)FM[(m * xrows + rb) * (T + 1) + ca + 1] * dt * a.dy;
    else v = -(double)GP[(m * (T + 1) + rb) * T + ca] * dt * a.dx;
    a.regs[e.dst + m] = v;
  }
  for (int it = tid; it < wk.fad_count * ME; it += STEP2_THREADS) {
    const FadEntry e = a.fad[wk.fad_start + it / ME];
    const int m = it % ME;
    const int r = e.pad;
    double* svd = a.regs + P.ffl + (long long)ME * e.seg + m;
    double s = *svd;
    for (int l = 0; l < r; ++l) {
      const int f = e.f0 + l;
      if (e.side == 1) s = s + (double)FM[(m * xrows + (f - j0)) * (T + 1) + 0] * dt * a.dy;
      else if (e.side == 2) s = s + (double)GP[(m * (T + 1) + th) * T + (f - i0)] * dt * a.dx;
      else if (e.side == 3) s = s + (double)FP[(m * xrows + (f - j0)) * (T + 1) + tw] * dt * a.dy;
      else s = s + (double)GM[(m * (T + 1) + 0) * T + (f - i0)] * dt * a.dx;
    }
    *svd = s;
  }
}

// Block maximum of the Courant number into the level maximum (bit pattern of a non-negative double).
template <class R>
__device__ __forceinline__ void cfl_to_level(R cfl, R* red, unsigned long long* cflmax) {
  const int tid = threadIdx.x;
  for (int off = 16; off > 0; off >>= 1) cfl = dmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
  if ((tid & 31) == 0) red[tid >> 5] = cfl;
  __syncthreads();
  if (tid == 0) {
    R c = R(0);
    for (int k = 0; k < STEP2_THREADS / 32; ++k) c = dmax(c, red[k]);
    atomicMax(cflmax, (unsigned long long)__double_as_longlong((double)c));
  }
}

// The shared-memory layout of a step block.
template <class S, class R>
struct Step2Smem {
  using L = Step2Layout<S>;
  R *Qs, *FM, *FP, *GM, *GP, *TR, *W, *X, *As, *red;
  __device__ explicit Step2Smem(unsigned char* raw) {
    Qs = reinterpret_cast<R*>(raw);
    FM = Qs + L::NQ; FP = FM + L::NF; GM = FP + L::NF; GP = GM + L::NF; TR = GP + L::NF;
    W = TR + L::NTR; X = W + L::NW; As = X + L::NX; red = As + L::NAQ;
  }
};

// One tile of one patch: stepgrid.f / step2.f90 / flux2.f over the tile, its update and its
// flux-register epilogue, with the Courant number of its faces folded into cfl. s_bar is the
// block's bulk-copy barrier and phase the parity of its next phase. Returns false (after
// flagging a.cflmax as infinite) if the tile's bulk copies did not complete in time.
template <class S, class R>
__device__ __forceinline__ bool step2_tile(const StepArgs& a, const StepWork& wk, const Step2Smem<S, R>& sm,
                                           unsigned long long& s_bar, int& s_ok, unsigned& phase, R& cfl) {
  using L = Step2Layout<S>;
  constexpr int ME = L::ME, T = L::T, QW = L::QW;
  constexpr int SE = 16 / (int)sizeof(R), RW = stage_row<R, QW>();
  static_assert(ME * QW * RW <= L::NW + L::NX, "bulk-copy staging must fit in W and X");
  static_assert(((L::NQ + 4 * L::NF + L::NTR) * sizeof(R)) % 16 == 0 && (RW * sizeof(R)) % 16 == 0,
                "staging rows must be 16-byte aligned");
  R *Qs = sm.Qs, *FM = sm.FM, *FP = sm.FP, *GM = sm.GM, *GP = sm.GP, *TR = sm.TR, *W = sm.W, *X = sm.X, *As = sm.As;
  (void)X;
  const int tid = threadIdx.x;
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;
  const R dtdx = (R)(dt / a.dx), dtdy = (R)(dt / a.dy);
  const bool capa = L::NA > 0 && a.sp.mcapa > 0;
  const PatchDev P = a.patches[wk.patch];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
  const int mitot = P.mitot, mjtot = P.mjtot;
  const int i0 = wk.ti0, j0 = wk.tj0;
  const int tw = min(T, mx - i0 + 1), th = min(T, my - j0 + 1);
  R* qout = static_cast<R*>(a.pool) + P.q[1 - P.cur];
  const long long plane = (long long)mitot * mjtot;
  // load the tile with its two ghost layers: interior (i,j) -> enlarged 0-based (i+1, j+1).
  // Each row (m, b) of lw values starts at pool element rowg(m, b); thread r < ME*lh
  // announces its row's bytes on the barrier and issues the bulk copy into staging row r
  // (W and X, free between tiles); thread 0 arrives once every row is announced.
  const int lw = tw + 4, lh = th + 4;
  const long long q0 = P.q[P.cur] + (long long)(j0 - 1) * mitot + (i0 - 1);
  auto rowg = [&](int m, int b) { return q0 + m * plane + (long long)b * mitot; };
  if (tid < ME * lh) {
    const int m = tid / lh, b = tid % lh;
    const long long g = rowg(m, b), g0 = g & ~(long long)(SE - 1), g1 = (g + lw + SE - 1) & ~(long long)(SE - 1);
    const unsigned bytes = (unsigned)((g1 - g0) * (long long)sizeof(R));
    mbar_expect_tx(&s_bar, bytes);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    bulk_g2s(W + tid * RW, static_cast<const R*>(a.pool) + g0, bytes, &s_bar);
  }
  __syncthreads();
  if (tid == 0) {
    mbar_arrive(&s_bar);
    s_ok = mbar_wait_bounded(&s_bar, phase) ? 1 : 0;
  }
  __syncthreads();
  // every thread observes the completed phase itself (it completed: no wait)
  if (s_ok && tid != 0) mbar_wait_bounded(&s_bar, phase);
  phase ^= 1u;
  if (!s_ok) {
    // the copies did not complete: flag the level's Courant number as infinite (the host
    // stops on it) and leave once this block's copies have landed or their wait ran out
    if (tid == 0) {
      atomicMax(a.cflmax, 0x7FF0000000000000ull);
      mbar_wait_bounded(&s_bar, phase ^ 1u);
    }
    return false;
  }
  for (int it = tid; it < ME * lw * lh; it += STEP2_THREADS) {
    const int m = it / (lw * lh), rem = it % (lw * lh);
    const int b = rem / lw, aa = rem % lw;
    const int off = (int)(rowg(m, b) & (SE - 1));
    Qs[(m * QW + b) * QW + aa] = W[(m * lh + b) * RW + off + aa];
  }
  if (L::NA > 0) {
    const R* aux = static_cast<const R*>(a.pool) + P.aux;
    const int na = min(L::NA, a.sp.prob.naux);
    for (int it = tid; it < na * lw * lh; it += STEP2_THREADS) {
      const int m = it / (lw * lh), rem = it % (lw * lh);
      const int b = rem / lw, aa = rem % lw;
      const int ie = (i0 - 2 + aa) + 1, je = (j0 - 2 + b) + 1;
      As[(m * QW + b) * QW + aa] = aux[m * plane + (long long)je * mitot + ie];
    }
  }
  __syncthreads();
  // x-sweeps: FM/FP initialised, per-cell transverse parts in TR
  step2_sweep<S, 1, R>(a.sp, Qs, As, W, X, TR, FM, FP, i0, j0, tw, th, dtdx, cfl);
  // GX(c, f) = (0 + part2(row f-1)) + part1(row f) -> GM and GP
  for (int it = tid; it < ME * (th + 1) * tw; it += STEP2_THREADS) {
    const int m = it / ((th + 1) * tw), rem = it % ((th + 1) * tw);
    const int fb = rem / tw, ca = rem % tw;
    const R up = TR[((fb * T + ca) * 2) * ME + ME + m];        // row f-1 = line index fb
    const R dn = TR[(((fb + 1) * T + ca) * 2) * ME + m];       // row f   = line index fb+1
    const R g = (R(0) + up) + dn;
    GM[(m * (T + 1) + fb) * T + ca] = g;
    GP[(m * (T + 1) + fb) * T + ca] = g;
  }
  __syncthreads();
  // y-sweeps: GM/GP += faddm/faddp, per-cell transverse parts in TR
  step2_sweep<S, 2, R>(a.sp, Qs, As, W, X, TR, GM, GP, i0, j0, tw, th, dtdy, cfl);
  // FM(f, r) = (FM + part2(col f-1)) + part1(col f)
  for (int it = tid; it < ME * th * (tw + 1); it += STEP2_THREADS) {
    const int m = it / (th * (tw + 1)), rem = it % (th * (tw + 1));
    const int rb = rem / (tw + 1), fa = rem % (tw + 1);
    const R up = TR[((fa * T + rb) * 2) * ME + ME + m];        // column f-1 = line index fa
    const R dn = TR[(((fa + 1) * T + rb) * 2) * ME + m];       // column f   = line index fa+1
    const int k = (m * T + rb) * (T + 1) + fa;
    FM[k] = (FM[k] + up) + dn;
    FP[k] = (FP[k] + up) + dn;
  }
  __syncthreads();
  // conservative update (stepgrid.f:154-173; with a capacity array the flux difference is
  // divided by kappa)
  for (int it = tid; it < ME * th * tw; it += STEP2_THREADS) {
    const int m = it / (th * tw), rem = it % (th * tw);
    const int rb = rem / tw, ca = rem % tw;
    const R q = Qs[(m * QW + rb + 2) * QW + ca + 2];
    const R fmr = FM[(m * T + rb) * (T + 1) + ca + 1], fpl = FP[(m * T + rb) * (T + 1) + ca];
    const R gmt = GM[(m * (T + 1) + rb + 1) * T + ca], gpb = GP[(m * (T + 1) + rb) * T + ca];
    const R qn = capa ? q - (dtdx * (fmr - fpl) + dtdy * (gmt - gpb)) / As[((a.sp.mcapa - 1) * QW + rb + 2) * QW + ca + 2]
                      : q - dtdx * (fmr - fpl) - dtdy * (gmt - gpb);
    const int ie = i0 + ca + 1, je = j0 + rb + 1;
    qout[m * plane + (long long)je * mitot + ie] = qn;
  }
  register_epilogue<ME, R>(a, wk, P, i0, j0, tw, th, dt, FM, FP, GM, GP, T);
  __syncthreads();
  return true;
}

// the bulk-copy barrier of a step block: one arrival per phase (thread 0), the rows' bytes
// as its transactions
__device__ __forceinline__ void step2_barrier_init(unsigned long long& s_bar) {
  if (threadIdx.x == 0) {
    mbar_init(&s_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

template <class S, class R>
__global__ void __launch_bounds__(STEP2_THREADS) step2_kernel(StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Step2Smem<S, R> sm(smem_raw);
  __shared__ int s_item;
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ int s_ok;
  step2_barrier_init(s_bar);
  unsigned phase = 0;
  const int tid = threadIdx.x;
  R cfl = R(0);
  int iter = 0;
  while (true) {
    int w;
    if (a.queue) {
      if (tid == 0) s_item = atomicAdd(a.queue, 1);
      __syncthreads();
      w = s_item;
      __syncthreads();
    } else {
      w = blockIdx.x + iter * gridDim.x;
    }
    ++iter;
    if (w >= a.nwork) break;
    if (!step2_tile<S, R>(a, a.work[w], sm, s_bar, s_ok, phase, cfl)) return;
  }
  cfl_to_level(cfl, sm.red, a.cflmax);
}

// The level substeps of several solves in one launch (cross-request batching): the tiles of
// member k are items [work0[k], work0[k+1]) of the combined list, each stepped with member
// k's arguments exactly as step2_kernel steps it. A block's Courant number goes to a
// member's level maximum whenever the block moves on to the next member.
template <class S, class R>
__global__ void __launch_bounds__(STEP2_THREADS) step2_batch_kernel(const __grid_constant__ StepBatch B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Step2Smem<S, R> sm(smem_raw);
  __shared__ __align__(8) unsigned long long s_bar;
  __shared__ int s_ok;
  step2_barrier_init(s_bar);
  unsigned phase = 0;
  R cfl = R(0);
  int cur = -1;
  for (int w = blockIdx.x; w < B.work0[B.n]; w += gridDim.x) {
    int k = 0;
    while (w >= B.work0[k + 1]) ++k;
    if (k != cur) {
      if (cur >= 0) cfl_to_level(cfl, sm.red, B.m[cur].cflmax);
      cfl = R(0);
      cur = k;
    }
    const StepArgs& a = B.m[k];
    if (!step2_tile<S, R>(a, a.work[w - B.work0[k]], sm, s_bar, s_ok, phase, cfl)) return;
  }
  if (cur >= 0) cfl_to_level(cfl, sm.red, B.m[cur].cflmax);
}

// ======================================================================= Godunov-split patch step
// stepgrid_dimSplit.f:4-201 with step2x.f90, step2y.f90 and flux2_dimSplit.f over one tile.
// The reference sweeps x along every row of the enlarged patch (ghost rows included) and
// x-updates every row's interior cells before the y-sweeps read them, so the tile sweeps
// its own rows and two rows on each side (all staged with the tile), x-updates them, then
// sweeps y along its columns over the x-updated values and y-updates. The Courant number
// takes every face each tile computes (the maximum is unchanged by faces counted twice).
// Face fluxes are fm = (0 + amdq) + cqxx/2, fp = (0 - apdq) + cqxx/2: flux2_dimSplit's
// faddm = amdq, faddp = -apdq (+ cqxx/2) added to zeroed arrays give the same values.
template <class S>
struct Split2Layout {
  static constexpr int ME = S::MEQN, MW = S::MWAVES, T = TILE2, QW = T + 4;
  static constexpr int NQ = ME * QW * QW;           // staged q of the tile and two ghost layers
  static constexpr int NFX = ME * QW * (T + 1);      // fm / fp of every staged row
  static constexpr int NQX = ME * QW * T;            // x-updated q of the tile's columns
  static constexpr int NG = ME * (T + 1) * T;        // gm / gp
  static constexpr int WREC = MW * ME + MW + 2 * ME;
  static constexpr int NW = STEP2_RC * (T + 3) * WREC;
  static constexpr int NA = S::NAUX > 0 ? MAXAUX2 : 0;
  static constexpr int NAQ = NA * QW * QW;           // staged aux, [m][b][a] like Qs
  static constexpr int TOTAL = NQ + 2 * NFX + NQX + 2 * NG + NW + NAQ + 32;
};

template <class S, class R>
__global__ void __launch_bounds__(STEP2_THREADS) step2s_kernel(StepArgs a) {
  using L = Split2Layout<S>;
  constexpr int ME = L::ME, T = L::T, QW = L::QW, WREC = L::WREC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* Qs = reinterpret_cast<R*>(smem_raw);
  R* FXm = Qs + L::NQ;
  R* FXp = FXm + L::NFX;
  R* Qx = FXp + L::NFX;
  R* GM = Qx + L::NQX;
  R* GP = GM + L::NG;
  R* W = GP + L::NG;
  R* As = W + L::NW;
  R* red = As + L::NAQ;
  __shared__ int s_item;
  const int tid = threadIdx.x;
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;
  const R dtdx = (R)(dt / a.dx), dtdy = (R)(dt / a.dy);
  const bool capa = L::NA > 0 && a.sp.mcapa > 0;
  // kappa of staged cell (b, c); dtdx1d of it for the step d (flux2_dimSplit.f with capa)
  auto kap = [&](int b, int c) -> R { return As[((a.sp.mcapa - 1) * QW + b) * QW + c]; };
  auto d1d = [&](R d, int b, int c) -> R { return capa ? d / kap(b, c) : d; };
  R cfl = R(0);
  int iter = 0;
  while (true) {
    int w;
    if (a.queue) {
      if (tid == 0) s_item = atomicAdd(a.queue, 1);
      __syncthreads();
      w = s_item;
      __syncthreads();
    } else {
      w = blockIdx.x + iter * gridDim.x;
    }
    ++iter;
    if (w >= a.nwork) break;
    const StepWork wk = a.work[w];
    const PatchDev P = a.patches[wk.patch];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
    const int mitot = P.mitot, mjtot = P.mjtot;
    const int i0 = wk.ti0, j0 = wk.tj0;
    const int tw = min(T, mx - i0 + 1), th = min(T, my - j0 + 1);
    const R* qin = static_cast<const R*>(a.pool) + P.q[P.cur];
    R* qout = static_cast<R*>(a.pool) + P.q[1 - P.cur];
    const long long plane = (long long)mitot * mjtot;
    const int lw = tw + 4, lh = th + 4;
    for (int it = tid; it < ME * lw * lh; it += STEP2_THREADS) {
      const int m = it / (lw * lh), rem = it % (lw * lh);
      const int b = rem / lw, aa = rem % lw;
      const int ie = (i0 - 2 + aa) + 1, je = (j0 - 2 + b) + 1;
      Qs[(m * QW + b) * QW + aa] = qin[m * plane + (long long)je * mitot + ie];
    }
    if (L::NA > 0) {
      const R* aux = static_cast<const R*>(a.pool) + P.aux;
      const int na = min(L::NA, a.sp.prob.naux);
      for (int it = tid; it < na * lw * lh; it += STEP2_THREADS) {
        const int m = it / (lw * lh), rem = it % (lw * lh);
        const int b = rem / lw, aa = rem % lw;
        const int ie = (i0 - 2 + aa) + 1, je = (j0 - 2 + b) + 1;
        As[(m * QW + b) * QW + aa] = aux[m * plane + (long long)je * mitot + ie];
      }
    }
    __syncthreads();
    // step2x.f90: rows b (j = j0-2+b), faces ff (i = i0-1+ff, between staged columns ff, ff+1)
    {
      const int nfr = tw + 3, nfl = tw + 1;
      for (int b0 = 0; b0 < lh; b0 += STEP2_RC) {
        const int nb = min(STEP2_RC, lh - b0);
        for (int it = tid; it < nb * nfr; it += STEP2_THREADS) {
          const int rr = it / nfr, ff = it % nfr, b = b0 + rr;
          R qL[ME], qR[ME];
#pragma unroll
          for (int m = 0; m < ME; ++m) { qL[m] = Qs[(m * QW + b) * QW + ff]; qR[m] = Qs[(m * QW + b) * QW + ff + 1]; }
          AuxCell<S, R> aL, aR;
          if (S::NAUX > 0) { aL.load(As, QW, b, ff); aR.load(As, QW, b, ff + 1); }
          face_record<S, R>(a.sp, 1, qL, qR, aL.v, aR.v, W + (rr * (T + 3) + ff) * WREC, d1d(dtdx, b, ff),
                            d1d(dtdx, b, ff + 1), ff >= 1 && ff <= nfl, cfl);
        }
        __syncthreads();
        for (int it = tid; it < nb * nfl; it += STEP2_THREADS) {
          const int rr = it / nfl, fa = it % nfl, b = b0 + rr;
          const R* rm = W + (rr * (T + 3) + fa) * WREC;
          R amdq[ME], apdq[ME], cqxx[ME], fm[ME], fp[ME];
          face_fluxes<S, R>(a.sp, rm, rm + WREC, rm + 2 * WREC, d1d(dtdx, b, fa + 1), d1d(dtdx, b, fa + 2), amdq, apdq,
                            cqxx, fm, fp);
#pragma unroll
          for (int m = 0; m < ME; ++m) {
            FXm[(m * QW + b) * (T + 1) + fa] = fm[m];
            FXp[(m * QW + b) * (T + 1) + fa] = fp[m];
          }
        }
        __syncthreads();
      }
    }
    // stepgrid_dimSplit.f:88-103: x-update of every staged row's tile cells. The rows that
    // are the patch's ghost rows (below row 1 or above row my) keep their x-updated values
    // in the new store1, as the reference's array does (binary output writes them).
    for (int it = tid; it < ME * lh * tw; it += STEP2_THREADS) {
      const int m = it / (lh * tw), rem = it % (lh * tw);
      const int b = rem / tw, c = rem % tw;
      const R df = dtdx * (FXm[(m * QW + b) * (T + 1) + c + 1] - FXp[(m * QW + b) * (T + 1) + c]);
      const R v = Qs[(m * QW + b) * QW + c + 2] - (capa ? df / kap(b, c + 2) : df);
      Qx[(m * QW + b) * T + c] = v;
      const int jrow = j0 - 2 + b;
      if (jrow < 1 || jrow > my) qout[m * plane + (long long)(jrow + 1) * mitot + (i0 + c + 1)] = v;
    }
    __syncthreads();
    // step2y.f90: columns c (i = i0+c), faces ff (j = j0-1+ff, between x-updated rows ff, ff+1)
    {
      const int nfr = th + 3, nfl = th + 1;
      for (int c0 = 0; c0 < tw; c0 += STEP2_RC) {
        const int nc = min(STEP2_RC, tw - c0);
        for (int it = tid; it < nc * nfr; it += STEP2_THREADS) {
          const int rr = it / nfr, ff = it % nfr, c = c0 + rr;
          R qL[ME], qR[ME];
#pragma unroll
          for (int m = 0; m < ME; ++m) { qL[m] = Qx[(m * QW + ff) * T + c]; qR[m] = Qx[(m * QW + ff + 1) * T + c]; }
          AuxCell<S, R> aL, aR;
          if (S::NAUX > 0) { aL.load(As, QW, ff, c + 2); aR.load(As, QW, ff + 1, c + 2); }
          face_record<S, R>(a.sp, 2, qL, qR, aL.v, aR.v, W + (rr * (T + 3) + ff) * WREC, d1d(dtdy, ff, c + 2),
                            d1d(dtdy, ff + 1, c + 2), ff >= 1 && ff <= nfl, cfl);
        }
        __syncthreads();
        for (int it = tid; it < nc * nfl; it += STEP2_THREADS) {
          const int rr = it / nfl, fb = it % nfl, c = c0 + rr;
          const R* rm = W + (rr * (T + 3) + fb) * WREC;
          R amdq[ME], apdq[ME], cqxx[ME], fm[ME], fp[ME];
          face_fluxes<S, R>(a.sp, rm, rm + WREC, rm + 2 * WREC, d1d(dtdy, fb + 1, c + 2), d1d(dtdy, fb + 2, c + 2), amdq,
                            apdq, cqxx, fm, fp);
#pragma unroll
          for (int m = 0; m < ME; ++m) {
            GM[(m * (T + 1) + fb) * T + c] = fm[m];
            GP[(m * (T + 1) + fb) * T + c] = fp[m];
          }
        }
        __syncthreads();
      }
    }
    // stepgrid_dimSplit.f:118-133: y-update of the tile's cells into the other buffer
    for (int it = tid; it < ME * th * tw; it += STEP2_THREADS) {
      const int m = it / (th * tw), rem = it % (th * tw);
      const int rb = rem / tw, ca = rem % tw;
      const R dg = dtdy * (GM[(m * (T + 1) + rb + 1) * T + ca] - GP[(m * (T + 1) + rb) * T + ca]);
      const R qn = Qx[(m * QW + rb + 2) * T + ca] - (capa ? dg / kap(rb + 2, ca + 2) : dg);
      qout[m * plane + (long long)(j0 + rb + 1) * mitot + (i0 + ca + 1)] = qn;
    }
    // the tile's own rows start at staged row 2 of FXm / FXp
    register_epilogue<ME, R>(a, wk, P, i0, j0, tw, th, dt, FXm + 2 * (T + 1), FXp + 2 * (T + 1), GM, GP, QW);
    __syncthreads();
  }
  cfl_to_level(cfl, red, a.cflmax);
}

template <class S, class R>
static void launch_step2_t(const StepArgs& a, int grid, cudaStream_t s) {
  if (a.sp.split) {
    const size_t sm = sizeof(R) * Split2Layout<S>::TOTAL;
    static const bool attr = [&] {
      AMR_CUDA(cudaFuncSetAttribute(step2s_kernel<S, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      return true;
    }();
    (void)attr;
    if (grid <= 0) return;
    step2s_kernel<S, R><<<grid, STEP2_THREADS, sm, s>>>(a);
    AMR_CUDA(cudaGetLastError());
    return;
  }
  const size_t sm = sizeof(R) * Step2Layout<S>::TOTAL;
  // once per process (thread-safe static initialisation; contexts may run on several host threads)
  static const bool attr = [&] {
    AMR_CUDA(cudaFuncSetAttribute(step2_kernel<S, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    return true;
  }();
  (void)attr;
  if (grid <= 0) return;
  step2_kernel<S, R><<<grid, STEP2_THREADS, sm, s>>>(a);
  AMR_CUDA(cudaGetLastError());
}

template <class R>
static void launch_step2_r(int solver, const StepArgs& a, int grid, cudaStream_t s) {
  switch (solver) {
    case SOLVER_ADVECTION: launch_step2_t<Advection2, R>(a, grid, s); break;
    case SOLVER_ACOUSTICS: launch_step2_t<Acoustics2, R>(a, grid, s); break;
    case SOLVER_EULER: launch_step2_t<Euler2, R>(a, grid, s); break;
    case SOLVER_VC_ADVECTION: launch_step2_t<VcAdvection2, R>(a, grid, s); break;
    default: throw std::runtime_error("launch_step2: unsupported solver");
  }
}

void launch_step2(int solver, const StepArgs& a, int grid, cudaStream_t s, bool f32) {
  if (f32) launch_step2_r<float>(solver, a, grid, s);
  else launch_step2_r<double>(solver, a, grid, s);
}

template <class S, class R>
static void launch_step2_batch_t(const StepBatch& b, int grid, cudaStream_t s) {
  const size_t sm = sizeof(R) * Step2Layout<S>::TOTAL;
  static const bool attr = [&] {
    AMR_CUDA(cudaFuncSetAttribute(step2_batch_kernel<S, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    return true;
  }();
  (void)attr;
  if (grid <= 0) return;
  step2_batch_kernel<S, R><<<grid, STEP2_THREADS, sm, s>>>(b);
  AMR_CUDA(cudaGetLastError());
}
template <class R>
static void launch_step2_batch_r(int solver, const StepBatch& b, int grid, cudaStream_t s) {
  switch (solver) {
    case SOLVER_ADVECTION: launch_step2_batch_t<Advection2, R>(b, grid, s); break;
    case SOLVER_ACOUSTICS: launch_step2_batch_t<Acoustics2, R>(b, grid, s); break;
    case SOLVER_EULER: launch_step2_batch_t<Euler2, R>(b, grid, s); break;
    case SOLVER_VC_ADVECTION: launch_step2_batch_t<VcAdvection2, R>(b, grid, s); break;
    default: throw std::runtime_error("launch_step2_batch: unsupported solver");
  }
}
void launch_step2_batch(int solver, const StepBatch& b, int grid, cudaStream_t s, bool f32) {
  if (f32) launch_step2_batch_r<float>(solver, b, grid, s);
  else launch_step2_batch_r<double>(solver, b, grid, s);
}

size_t step2_smem_bytes(int solver, bool f32) {
  const size_t w = f32 ? sizeof(float) : sizeof(double);
  switch (solver) {
    case SOLVER_ADVECTION: return w * Step2Layout<Advection2>::TOTAL;
    case SOLVER_ACOUSTICS: return w * Step2Layout<Acoustics2>::TOTAL;
    case SOLVER_EULER: return w * Step2Layout<Euler2>::TOTAL;
    case SOLVER_VC_ADVECTION: return w * Step2Layout<VcAdvection2>::TOTAL;
  }
  return 0;
}

// ======================================================================= ghost fill
// Storage type T (double, or float in the FP32 form); the fill arithmetic is FP64.
template <class T>
__device__ __forceinline__ T* fill_dst(const FillArgs& a, const FillOp& o, int& ldi, long long& plane) {
  if (o.dst_patch >= 0) {
    const PatchDev& P = a.patches[o.dst_patch];
    ldi = P.mitot; plane = (long long)P.mitot * P.mjtot;
    return static_cast<T*>(a.pool) + P.q[P.cur];
  }
  const ScratchRect& R = a.rects[o.dst_rect];
  ldi = R.ni; plane = (long long)R.ni * R.nj;
  return static_cast<T*>(a.pool) + R.off;
}

// one 128-cell chunk c of a fill program (one block)
template <class T>
__device__ __forceinline__ void fill_chunk(const FillArgs& a, int c) {
  const T* pool = static_cast<const T*>(a.pool);
  const FillChunk ch = a.chunks[c];
  if ((int)threadIdx.x >= ch.count) return;
  const FillOp o = a.ops[ch.op];
  const int cell = ch.start + threadIdx.x;
  const int ia = cell % o.ni, jb = cell / o.ni;
  const int nvar = a.nvar;
  if (o.kind == FILL_RING) {
    // cstore.f:4-63: ring of coarse values around a fine grid into qc1d of the kid
    const ScratchRect& R = a.rects[o.src];
    const int nrow = R.ni, ncol = R.nj;
    int k = cell, ii, jj;  // 0-based position in the rect
    if (k < ncol - 2) { ii = 0; jj = 1 + k; }
    else if ((k -= ncol - 2) < nrow - 2) { ii = 1 + k; jj = ncol - 1; }
    else if ((k -= nrow - 2) < ncol - 2) { ii = nrow - 1; jj = 1 + k; }
    else { k -= ncol - 2; ii = 1 + k; jj = 0; }
    const PatchDev& K = a.patches[o.dst_patch];
    double* qc1d = a.regs + K.ffl + (long long)nvar * K.lenbc + (long long)nvar * cell;
    const T* src = pool + R.off;
    const long long pl = (long long)nrow * ncol;
    for (int m = 0; m < nvar; ++m) qc1d[m] = (double)src[m * pl + (long long)jj * nrow + ii];
    return;
  }
  int ldi; long long plane;
  T* dst = fill_dst<T>(a, o, ldi, plane);
  const long long dk = (long long)(o.dj0 + jb) * ldi + (o.di0 + ia);
  if (o.kind == FILL_COPY) {
    const PatchDev& S = a.patches[o.src];
    const long long sp = (long long)S.mitot * S.mjtot;
    const long long sk = (long long)(o.sj0 + jb) * S.mitot + (o.si0 + ia);
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
  if (o.kind == FILL_PIECE) {
    const ScratchRect& R = a.rects[o.src];
    const long long sp = (long long)R.ni * R.nj;
    const long long sk = (long long)(o.sj0 + jb) * R.ni + (o.si0 + ia);
    const T* src = pool + R.off;
    for (int m = 0; m < nvar; ++m) dst[m * plane + dk] = src[m * sp + sk];
    return;
  }
  const ScratchRect& R = a.rects[o.src];
  const T* vc = pool + R.off;
  const long long cp = (long long)R.ni * R.nj;
  const int lev = o.level;
  const int rx = a.lc.intratx[lev - 1], ry = a.lc.intraty[lev - 1];
  const int ifg = o.si0 + ia, jfg = o.sj0 + jb;
  if (o.kind == FILL_INTERP) {
    // filpatch.f90:259-327 limited interpolation from the coarse scratch rect
    const double dxf = a.lc.hx[lev], dyf = a.lc.hy[lev], dxc = a.lc.hx[lev - 1], dyc = a.lc.hy[lev - 1];
    const int icg = floordiv(ifg, rx), jcg = floordiv(jfg, ry);
    const int ic = icg - o.cilo + 1, jc = jcg - o.cjlo + 1;  // 1-based in the coarse rect
    const double xlow_c = a.xlower + o.cilo * dxc, ylow_c = a.ylower + o.cjlo * dyc;
    const double ycc = ylow_c + (jc - 0.5) * dyc;
    const double ycf = a.ylower + (jfg + 0.5) * dyf;
    const double eta2 = (ycf - ycc) / dyc;
    const double xcc = xlow_c + (ic - 0.5) * dxc;
    const double xcf = a.xlower + (ifg + 0.5) * dxf;
    const double eta1 = (xcf - xcc) / dxc;
    auto CI = [&](int m, int i, int j) { return (double)vc[m * cp + (long long)(j - 1) * R.ni + (i - 1)]; };
    for (int m = 0; m < nvar; ++m) {
      const double valp10 = CI(m, ic + 1, jc), valm10 = CI(m, ic - 1, jc), valc = CI(m, ic, jc);
      const double valp01 = CI(m, ic, jc + 1), valm01 = CI(m, ic, jc - 1);
      const double dupc = valp10 - valc, dumc = valc - valm10, ducc = valp10 - valm10;
      double du = dmin(fabs(dupc), fabs(dumc));
      du = dmin(2.0 * du, 0.5 * fabs(ducc));
      const double fu = dmax(0.0, dsign(1.0, dupc * dumc));
      const double uslope = du * dsign(1.0, ducc) * fu;
      const double dvpc = valp01 - valc, dvmc = valc - valm01, dvcc = valp01 - valm01;
      double dv = dmin(fabs(dvpc), fabs(dvmc));
      dv = dmin(2.0 * dv, 0.5 * fabs(dvcc));
      const double fv = dmax(0.0, dsign(1.0, dvpc * dvmc));
      const double vslope = dv * dsign(1.0, dvcc) * fv;
      dst[m * plane + dk] = (T)(valc + eta1 * uslope + eta2 * vslope);
    }
    return;
  }
  if (o.kind == FILL_FIXCAPA) {
    // fixcapaq.f:4-62 for one coarse cell of an interpolated region: conserve kappa*q over
    // the coarse cell, adding the difference over kappa to each of its fine cells
    const PatchDev& F = a.patches[o.dst_patch];
    const T* kap = pool + F.aux + (long long)(a.mcapa - 1) * plane;
    const int bi = o.si0 + ia * rx, bj = o.sj0 + jb * ry;  // global fine index of the block origin
    const int i = floordiv(bi, rx) - o.cilo + 1, j = floordiv(bj, ry) - o.cjlo + 1;  // 1-based in valc
    const long long k0 = (long long)(o.dj0 + jb * ry) * ldi + (o.di0 + ia * rx);
    const double kc = a.capa[o.capa0 + (long long)(j - 1) * R.ni + (i - 1)];
    for (int m = 0; m < nvar; ++m) {
      double capaqfine = 0.0;
      for (int ico = 0; ico < rx; ++ico)
        for (int jco = 0; jco < ry; ++jco) {
          const long long k = k0 + (long long)jco * ldi + ico;
          capaqfine = capaqfine + (double)kap[k] * (double)dst[m * plane + k];
        }
      const double dcapaq = kc * (double)vc[m * cp + (long long)(j - 1) * R.ni + (i - 1)] - capaqfine / (double)(rx * ry);
      for (int ico = 0; ico < rx; ++ico)
        for (int jco = 0; jco < ry; ++jco) {
          const long long k = k0 + (long long)jco * ldi + ico;
          dst[m * plane + k] = (T)((double)dst[m * plane + k] + dcapaq / (double)kap[k]);
        }
    }
    return;
  }
  if (o.kind == FILL_FILVAL) {
    // filval.f90:150-185 minmod-limited interpolation into an uncovered new-grid cell
    const int icg = floordiv(ifg, rx), jcg = floordiv(jfg, ry);
    const int ico = ifg - icg * rx + 1, jco = jfg - jcg * ry + 1;
    const int i = icg - o.cilo + 1, j = jcg - o.cjlo + 1;  // 1-based in valc
    auto VC = [&](int m, int ii, int jj) { return (double)vc[m * cp + (long long)(jj - 1) * R.ni + (ii - 1)]; };
    const double yoff = ((double)jco - 0.5) / ry - 0.5;
    const double xoff = ((double)ico - 0.5) / rx - 0.5;
    for (int m = 0; m < nvar; ++m) {
      double s1p = VC(m, i + 1, j) - VC(m, i, j), s1m = VC(m, i, j) - VC(m, i - 1, j);
      double slopex = dmin(fabs(s1p), fabs(s1m)) * dsign(1.0, VC(m, i + 1, j) - VC(m, i - 1, j));
      if (s1m * s1p <= 0.0) slopex = 0.0;
      s1p = VC(m, i, j + 1) - VC(m, i, j); s1m = VC(m, i, j) - VC(m, i, j - 1);
      double slopey = dmin(fabs(s1p), fabs(s1m)) * dsign(1.0, VC(m, i, j + 1) - VC(m, i, j - 1));
      if (s1m * s1p <= 0.0) slopey = 0.0;
      dst[m * plane + dk] = (T)(VC(m, i, j) + xoff * slopex + yoff * slopey);
    }
    return;
  }
}

template <class T>
__global__ void fill_kernel(FillArgs a) {
  const int c = blockIdx.x;
  if (c >= a.nchunks) return;
  fill_chunk<T>(a, c);
}
// the chunks of two independent programs in one launch: a's, then b's
template <class T>
__global__ void fill_pair_kernel(FillArgs a, FillArgs b) {
  const int c = blockIdx.x;
  if (c < a.nchunks) fill_chunk<T>(a, c);
  else if (c - a.nchunks < b.nchunks) fill_chunk<T>(b, c - a.nchunks);
}

void launch_fill(const FillArgs& a, cudaStream_t s, bool f32) {
  if (a.nchunks <= 0) return;
  if (f32) fill_kernel<float><<<a.nchunks, 128, 0, s>>>(a);
  else fill_kernel<double><<<a.nchunks, 128, 0, s>>>(a);
  AMR_CUDA(cudaGetLastError());
}
void launch_fill_pair(const FillArgs& a, const FillArgs& b, cudaStream_t s, bool f32) {
  const long long n = (long long)a.nchunks + b.nchunks;
  if (n <= 0) return;
  if (n >= (1LL << 31)) throw std::runtime_error("fill program too large for one launch");
  if (f32) fill_pair_kernel<float><<<(unsigned)n, 128, 0, s>>>(a, b);
  else fill_pair_kernel<double><<<(unsigned)n, 128, 0, s>>>(a, b);
  AMR_CUDA(cudaGetLastError());
}

// phase 0: x-sides over all rows; phase 1: y-sides over all columns (after phase 0)
template <class T>
__device__ __forceinline__ void bc_op(const BcArgs& a, int op, int phase) {
  const BcOp o = a.ops[op];
  T* v; int nrow = o.nrow, ncol = o.ncol;
  if (o.dst_patch >= 0) { const PatchDev& P = a.patches[o.dst_patch]; v = static_cast<T*>(a.pool) + P.q[P.cur]; }
  else v = static_cast<T*>(a.pool) + a.rects[o.dst_rect].off;
  const long long plane = (long long)nrow * ncol;
  auto V = [&](int m, int i, int j) -> T& { return v[m * plane + (long long)(j - 1) * nrow + (i - 1)]; };
  const int nvar = a.nvar;
  if (phase == 0) {
    const int nl = (o.nxl > 0 && (o.bxl == 1 || o.bxl == 3)) ? o.nxl : 0;
    const int nr = (o.ibeg > 0 && (o.bxr == 1 || o.bxr == 3)) ? nrow - o.ibeg + 1 : 0;
    const int tot = (nl + nr) * ncol;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
      const int j = t / (nl + nr) + 1, k = t % (nl + nr);
      if (k < nl) {
        const int i = k + 1;
        const int src = (o.bxl == 1) ? o.nxl + 1 : 2 * o.nxl + 1 - i;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, src, j);
        if (o.bxl == 3) V(1, i, j) = -V(1, i, j);
      } else {
        const int i = o.ibeg + (k - nl);
        const int src = (o.bxr == 1) ? o.ibeg - 1 : 2 * o.ibeg - 1 - i;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, src, j);
        if (o.bxr == 3) V(1, i, j) = -V(1, i, j);
      }
    }
  } else {
    const int nb = (o.nyb > 0 && (o.byl == 1 || o.byl == 3)) ? o.nyb : 0;
    const int nt = (o.jbeg > 0 && (o.byr == 1 || o.byr == 3)) ? ncol - o.jbeg + 1 : 0;
    const int tot = (nb + nt) * nrow;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
      const int i = t % nrow + 1, k = t / nrow;
      if (k < nb) {
        const int j = k + 1;
        const int src = (o.byl == 1) ? o.nyb + 1 : 2 * o.nyb + 1 - j;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, i, src);
        if (o.byl == 3) V(2, i, j) = -V(2, i, j);
      } else {
        const int j = o.jbeg + (k - nb);
        const int src = (o.byr == 1) ? o.jbeg - 1 : 2 * o.jbeg - 1 - j;
        for (int m = 0; m < nvar; ++m) V(m, i, j) = V(m, i, src);
        if (o.byr == 3) V(2, i, j) = -V(2, i, j);
      }
    }
  }
}

template <class T>
__global__ void bc_kernel(BcArgs a, int phase) {
  const int op = blockIdx.y;
  if (op >= a.nops) return;
  bc_op<T>(a, op, phase);
}
// the ops of two independent programs, one block per op doing phase 0 then phase 1 (the
// y-sides read the corners the x-sides wrote; each op has its own destination array)
template <class T>
__global__ void bc_pair_kernel(BcArgs a, BcArgs b) {
  const int op = blockIdx.y;
  const bool first = op < a.nops;
  const BcArgs& A = first ? a : b;
  const int o = first ? op : op - a.nops;
  if (o >= A.nops) return;
  bc_op<T>(A, o, 0);
  __syncthreads();
  bc_op<T>(A, o, 1);
}
void launch_bc_pair(const BcArgs& a, const BcArgs& b, cudaStream_t s, bool f32) {
  const int n = a.nops + b.nops;
  if (n <= 0) return;
  if (n > 65535) {  // more ops than one grid column: one program at a time, both phases
    for (const BcArgs* x : {&a, &b}) {
      if (x->nops <= 0) continue;
      launch_bc(*x, 0, s, f32);
      launch_bc(*x, 1, s, f32);
    }
    return;
  }
  if (f32) bc_pair_kernel<float><<<dim3(1, n), 128, 0, s>>>(a, b);
  else bc_pair_kernel<double><<<dim3(1, n), 128, 0, s>>>(a, b);
  AMR_CUDA(cudaGetLastError());
}
void launch_bc(const BcArgs& a, int phase, cudaStream_t s, bool f32) {
  if (a.nops <= 0) return;
  for (int base = 0; base < a.nops; base += 65535) {
    BcArgs b = a;
    b.ops = a.ops + base;
    b.nops = std::min(65535, a.nops - base);
    dim3 grid(2, b.nops);
    if (f32) bc_kernel<float><<<grid, 128, 0, s>>>(b, phase);
    else bc_kernel<double><<<grid, 128, 0, s>>>(b, phase);
    AMR_CUDA(cudaGetLastError());
  }
}

// ======================================================================= qad
template <class S, class T>
__global__ void qad2_kernel(T* pool, double* regs, const PatchDev* patches, const QadJob* jobs, int njobs,
                            ProbDev prob, LevelConst lc, double delt, const double* dt_dev) {
  constexpr int ME = S::MEQN, MW = S::MWAVES;
  const int jb = blockIdx.x;
  if (jb >= njobs) return;
  if (dt_dev) delt = *dt_dev;
  const QadJob J = jobs[jb];
  const PatchDev P = patches[J.patch];
  const int lev = P.level;
  const int rx = lc.intratx[lev - 1], ry = lc.intraty[lev - 1];
  const double hx = lc.hx[lev], hy = lc.hy[lev];
  const T* q = pool + P.q[P.cur];
  const T* aux = pool + P.aux;
  const long long plane = (long long)P.mitot * P.mjtot;
  constexpr int NA = S::NAUX > 0 ? S::NAUX : 1;
  for (int sgi = threadIdx.x; sgi < J.nseg; sgi += blockDim.x) {
    const int seg = J.seg0 + sgi;
    double* svd = regs + P.ffl + (long long)ME * seg;
    const double* qc = regs + P.ffl + (long long)ME * P.lenbc + (long long)ME * seg;
    // auxc1d(:, seg) of the saved coarse ring (cstore.f), after svdflx and qc1d
    const double* ac = regs + P.ffl + (long long)2 * ME * P.lenbc + (long long)prob.naux * seg;
    double sv[ME];
#pragma unroll
    for (int m = 0; m < ME; ++m) sv[m] = svd[m];
    const int r = (J.side == 1 || J.side == 3) ? ry : rx;
    for (int l = 1; l <= r; ++l) {
      const int f = sgi * r + l;  // fine row (sides 1,3) or column (sides 2,4), 1-based interior
      T qf[ME], qcr[ME];
      long long k;
      if (J.side == 1) k = (long long)(f + 1) * P.mitot + 1;
      else if (J.side == 2) k = (long long)(P.mjtot - 2) * P.mitot + (f + 1);
      else if (J.side == 3) k = (long long)(f + 1) * P.mitot + (P.mitot - 2);
      else k = (long long)1 * P.mitot + (f + 1);
#pragma unroll
      for (int m = 0; m < ME; ++m) { qf[m] = q[m * plane + k]; qcr[m] = (T)qc[m]; }
      // qad.f:79-89, 160-185, 231-256, 298-308: the fine cell's aux, except that the aux of
      // the state across the interface is the coarse ring's, or the fine cell's own face
      // value for a face-type component on that face (xleft on sides 1 and 3, yleft on 2, 4)
      T af[NA], ax[NA];
      if (S::NAUX > 0) {
        const int face_type = (J.side == 1 || J.side == 3) ? AUX_XLEFT : AUX_YLEFT;
        // sides 1 and 4: the fine state's aux is the ghost cell's, or the first interior
        // cell's (its lower face is the interface) for the face-type component
        const long long kin = (J.side == 1) ? k + 1 : (J.side == 4) ? k + P.mitot : k;
#pragma unroll
        for (int m = 0; m < S::NAUX; ++m) {
          const bool ft = prob.auxtype[m] == face_type;
          if (J.side == 1 || J.side == 4) { af[m] = ft ? aux[m * plane + kin] : aux[m * plane + k]; ax[m] = (T)ac[m]; }
          else { af[m] = aux[m * plane + k]; ax[m] = ft ? aux[m * plane + k] : (T)ac[m]; }
        }
      }
      T wave[MW][ME], s[MW], amdq[ME], apdq[ME];
      if (J.side == 1) S::template rpn<T>(prob, 1, qcr, qf, ax, af, wave, s, amdq, apdq);
      else if (J.side == 2) S::template rpn<T>(prob, 2, qf, qcr, af, ax, wave, s, amdq, apdq);
      else if (J.side == 3) S::template rpn<T>(prob, 1, qf, qcr, af, ax, wave, s, amdq, apdq);
      else S::template rpn<T>(prob, 2, qcr, qf, ax, af, wave, s, amdq, apdq);
#pragma unroll
      for (int m = 0; m < ME; ++m) {
        const double am = amdq[m], ap = apdq[m];  // registers accumulate in FP64
        if (J.side == 1) sv[m] = sv[m] + am * hy * delt + ap * hy * delt;
        else if (J.side == 2) sv[m] = sv[m] - am * hx * delt - ap * hx * delt;
        else if (J.side == 3) sv[m] = sv[m] - am * hy * delt - ap * hy * delt;
        else sv[m] = sv[m] + am * hx * delt + ap * hx * delt;
      }
    }
#pragma unroll
    for (int m = 0; m < ME; ++m) svd[m] = sv[m];
  }
}

template <class T>
static void launch_qad2_t(int solver, T* pool, double* regs, const PatchDev* patches, const QadJob* jobs, int njobs,
                          const ProbDev& prob, LevelConst lc, double delt, cudaStream_t s, const double* dt_dev) {
  switch (solver) {
    case SOLVER_ADVECTION: qad2_kernel<Advection2, T><<<njobs, 64, 0, s>>>(pool, regs, patches, jobs, njobs, prob, lc, delt, dt_dev); break;
    case SOLVER_ACOUSTICS: qad2_kernel<Acoustics2, T><<<njobs, 64, 0, s>>>(pool, regs, patches, jobs, njobs, prob, lc, delt, dt_dev); break;
    case SOLVER_EULER: qad2_kernel<Euler2, T><<<njobs, 64, 0, s>>>(pool, regs, patches, jobs, njobs, prob, lc, delt, dt_dev); break;
    case SOLVER_VC_ADVECTION: qad2_kernel<VcAdvection2, T><<<njobs, 64, 0, s>>>(pool, regs, patches, jobs, njobs, prob, lc, delt, dt_dev); break;
  }
}

void launch_qad2(int solver, void* pool, double* regs, const PatchDev* patches, const QadJob* jobs, int njobs,
                 const ProbDev& prob, int nvar, LevelConst lc, double delt, cudaStream_t s, bool f32, const double* dt_dev) {
  if (njobs <= 0) return;
  (void)nvar;
  if (f32) launch_qad2_t(solver, static_cast<float*>(pool), regs, patches, jobs, njobs, prob, lc, delt, s, dt_dev);
  else launch_qad2_t(solver, static_cast<double*>(pool), regs, patches, jobs, njobs, prob, lc, delt, s, dt_dev);
  AMR_CUDA(cudaGetLastError());
}

// ======================================================================= update
template <class T>
__global__ void upbnd_kernel(T* pool, const double* regs, const PatchDev* patches, const UpbndCell* cells,
                             int ncells, const UpbndTerm* terms, double area, int nvar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ncells * nvar) return;
  const int c = t / nvar, m = t % nvar;
  const UpbndCell C = cells[c];
  const PatchDev& P = patches[C.patch];
  T* v = pool + P.q[P.cur] + (long long)m * P.mitot * P.mjtot + (long long)C.je * P.mitot + C.ie;
  double val = (double)*v;
  for (int k = 0; k < C.count; ++k) {
    const UpbndTerm U = terms[C.first + k];
    val = val + U.sgn * regs[U.reg + m] / area;
  }
  *v = (T)val;
}

void launch_upbnd(void* pool, const double* regs, const PatchDev* patches, const UpbndCell* cells, int ncells,
                  const UpbndTerm* terms, double area, int nvar, cudaStream_t s, bool f32) {
  if (ncells <= 0) return;
  const int n = ncells * nvar;
  if (f32) upbnd_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<float*>(pool), regs, patches, cells, ncells, terms, area, nvar);
  else upbnd_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<double*>(pool), regs, patches, cells, ncells, terms, area, nvar);
  AMR_CUDA(cudaGetLastError());
}

// update.f:133-163: the average of the fine cells over a coarse cell, kappa-weighted and
// divided by totrat * kappa of the coarse cell when there is a capacity (mcapa > 0)
template <class T>
__global__ void average_kernel(T* pool, const PatchDev* patches, const AvgRect* rects, int nrects, int rx, int ry,
                               int nvar, int mcapa) {
  const int r = blockIdx.y;
  if (r >= nrects) return;
  const AvgRect A = rects[r];
  const PatchDev& C = patches[A.cpatch];
  const PatchDev& K = patches[A.kpatch];
  T* qc = pool + C.q[C.cur];
  const T* qf = pool + K.q[K.cur];
  const long long cpl = (long long)C.mitot * C.mjtot, fpl = (long long)K.mitot * K.mjtot;
  const double totrat = (double)(rx * ry);
  const int n = A.ni * A.nj * nvar;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int m = t / (A.ni * A.nj), rem = t % (A.ni * A.nj);
    const int b = rem / A.ni, aa = rem % A.ni;
    const int fi = A.fi0 + aa * rx, fj = A.fj0 + b * ry;
    double s = 0.0;
    const long long kc = (long long)(A.cj0 + b) * C.mitot + (A.ci0 + aa);
    if (mcapa == 0) {
      for (int jco = 0; jco < ry; ++jco)
        for (int ico = 0; ico < rx; ++ico) s = s + (double)qf[m * fpl + (long long)(fj + jco) * K.mitot + (fi + ico)];
      s = s / totrat;
    } else {
      const T* kf = pool + K.aux + (long long)(mcapa - 1) * fpl;
      const T* kcap = pool + C.aux + (long long)(mcapa - 1) * cpl;
      for (int jco = 0; jco < ry; ++jco)
        for (int ico = 0; ico < rx; ++ico) {
          const long long kk = (long long)(fj + jco) * K.mitot + (fi + ico);
          s = s + (double)qf[m * fpl + kk] * (double)kf[kk];
        }
      s = s / (totrat * (double)kcap[kc]);
    }
    qc[m * cpl + kc] = (T)s;
  }
}

void launch_average(void* pool, const PatchDev* patches, const AvgRect* rects, int nrects, int rx, int ry, int nvar,
                    cudaStream_t s, bool f32, int mcapa) {
  for (int base = 0; base < nrects; base += 65535) {
    const int n = std::min(65535, nrects - base);
    dim3 grid(4, n);
    if (f32) average_kernel<<<grid, 128, 0, s>>>(static_cast<float*>(pool), patches, rects + base, n, rx, ry, nvar, mcapa);
    else average_kernel<<<grid, 128, 0, s>>>(static_cast<double*>(pool), patches, rects + base, n, rx, ry, nvar, mcapa);
    AMR_CUDA(cudaGetLastError());
  }
}

// ======================================================================= flags, gauges, misc
template <class T>
__global__ void flags2_kernel(const T* pool, const PatchDev* patches, const int* plist, const long long* outoff,
                              int use_old, int flag_component, double tolsp, int nvar, int8_t* out) {
  const int pi = blockIdx.y;
  const PatchDev P = patches[plist[pi]];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
  const T* q = pool + P.q[use_old ? 1 - P.cur : P.cur];
  const long long plane = (long long)P.mitot * P.mjtot;
  const int m0 = flag_component > 0 ? flag_component - 1 : 0, m1 = flag_component > 0 ? flag_component - 1 : nvar - 1;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < mx * my; t += gridDim.x * blockDim.x) {
    const int i = t % mx + 1, j = t / mx + 1;  // interior, 1-based
    const int ie = i + 1, je = j + 1;
    int8_t f = 0;
    for (int m = m0; m <= m1; ++m) {
      const T* qm = q + m * plane;
      const double dqi = fabs((double)qm[(long long)je * P.mitot + ie + 1] - (double)qm[(long long)je * P.mitot + ie - 1]);
      const double dqj = fabs((double)qm[(long long)(je + 1) * P.mitot + ie] - (double)qm[(long long)(je - 1) * P.mitot + ie]);
      const double dq = dmax(0.0, dmax(dqi, dqj));
      if (dq > tolsp) { f = 1; break; }
    }
    out[outoff[pi] + t] = f;
  }
}

void launch_flags2(const void* pool, const PatchDev* patches, const int* plist, const long long* outoff, int np,
                   int use_old, int flag_component, double tolsp, int nvar, int8_t* out, cudaStream_t s, bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    dim3 grid(8, n);
    if (f32)
      flags2_kernel<<<grid, 128, 0, s>>>(static_cast<const float*>(pool), patches, plist + base, outoff + base, use_old, flag_component,
                                         tolsp, nvar, out);
    else
      flags2_kernel<<<grid, 128, 0, s>>>(static_cast<const double*>(pool), patches, plist + base, outoff + base, use_old, flag_component,
                                         tolsp, nvar, out);
    AMR_CUDA(cudaGetLastError());
  }
}

template <class T>
__global__ void gauges2_kernel(const T* pool, const PatchDev* patches, const GaugeJob* jobs, int njobs, int nvar,
                               double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= njobs) return;
  const GaugeJob G = jobs[t];
  const PatchDev& P = patches[G.patch];
  const T* q = pool + P.q[P.cur];
  const long long plane = (long long)P.mitot * P.mjtot;
  const double xo = G.xoff, yo = G.yoff;
  // Q(n, ii, jj) with ii, jj 1-based enlarged indices
  auto Q = [&](int m, int i, int j) { return (double)q[m * plane + (long long)(j - 1) * P.mitot + (i - 1)]; };
  for (int m = 0; m < nvar; ++m) {
    double v = (1.0 - xo) * (1.0 - yo) * Q(m, G.ii, G.jj) + xo * (1.0 - yo) * Q(m, G.ii + 1, G.jj) +
               (1.0 - xo) * yo * Q(m, G.ii, G.jj + 1) + xo * yo * Q(m, G.ii + 1, G.jj + 1);
    if (fabs(v) < 1e-90) v = 0.0;
    out[(long long)G.slot * nvar + m] = v;
  }
}

void launch_gauges2(const void* pool, const PatchDev* patches, const GaugeJob* jobs, int njobs, int nvar,
                    double* out, cudaStream_t s, bool f32) {
  if (njobs <= 0) return;
  if (f32) gauges2_kernel<<<(njobs + 63) / 64, 64, 0, s>>>(static_cast<const float*>(pool), patches, jobs, njobs, nvar, out);
  else gauges2_kernel<<<(njobs + 63) / 64, 64, 0, s>>>(static_cast<const double*>(pool), patches, jobs, njobs, nvar, out);
  AMR_CUDA(cudaGetLastError());
}

__global__ void flip_kernel(PatchDev* patches, const int* plist, int np) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < np) patches[plist[t]].cur ^= 1;
}
void launch_flip(PatchDev* patches, const int* plist, int np, cudaStream_t s) {
  if (np <= 0) return;
  flip_kernel<<<(np + 127) / 128, 128, 0, s>>>(patches, plist, np);
  AMR_CUDA(cudaGetLastError());
}

template <class T>
__global__ void zero_tiny_kernel(T* pool, const PatchDev* patches, const int* plist, int nvar) {
  const PatchDev P = patches[plist[blockIdx.y]];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
  T* q = pool + P.q[P.cur];
  const long long plane = (long long)P.mitot * P.mjtot;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < mx * my * nvar; t += gridDim.x * blockDim.x) {
    const int m = t / (mx * my), rem = t % (mx * my);
    const int i = rem % mx + 2, j = rem / mx + 2;
    T& v = q[m * plane + (long long)j * P.mitot + i];
    if (fabs((double)v) < 1e-90) v = (T)0;
  }
}
void launch_zero_tiny(void* pool, const PatchDev* patches, const int* plist, int np, int nvar, cudaStream_t s, bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    if (f32) zero_tiny_kernel<<<dim3(4, n), 128, 0, s>>>(static_cast<float*>(pool), patches, plist + base, nvar);
    else zero_tiny_kernel<<<dim3(4, n), 128, 0, s>>>(static_cast<double*>(pool), patches, plist + base, nvar);
    AMR_CUDA(cudaGetLastError());
  }
}

// conck.f:44-60: the first component over the interior, times kappa with a capacity
template <class T>
__global__ void mass2_kernel(const T* pool, const PatchDev* patches, const int* plist, int np, double* out, int mcapa) {
  double s = 0.0;
  for (int pi = blockIdx.y; pi < np; pi += gridDim.y) {
    const PatchDev P = patches[plist[pi]];
    const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
    const T* q = pool + P.q[P.cur];
    const T* kap = mcapa > 0 ? pool + P.aux + (long long)(mcapa - 1) * P.mitot * P.mjtot : nullptr;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < mx * my; t += gridDim.x * blockDim.x) {
      const long long k = (long long)(t / mx + 2) * P.mitot + (t % mx + 2);
      s += kap ? (double)q[k] * (double)kap[k] : (double)q[k];
    }
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}
void launch_mass2(const void* pool, const PatchDev* patches, const int* plist, int np, double* out, cudaStream_t s, bool f32,
                  int mcapa) {
  if (np <= 0) return;
  if (f32) mass2_kernel<<<dim3(4, std::min(np, 4096)), 128, 0, s>>>(static_cast<const float*>(pool), patches, plist, np, out, mcapa);
  else mass2_kernel<<<dim3(4, std::min(np, 4096)), 128, 0, s>>>(static_cast<const double*>(pool), patches, plist, np, out, mcapa);
  AMR_CUDA(cudaGetLastError());
}

template <class T>
__global__ void gather_interior2_kernel(const T* pool, const PatchDev* patches, const int* plist,
                                        const long long* outoff, int nvar, double* out) {
  const PatchDev P = patches[plist[blockIdx.y]];
  const int mx = P.ihi - P.ilo + 1, my = P.jhi - P.jlo + 1;
  const T* q = pool + P.q[P.cur];
  const long long plane = (long long)P.mitot * P.mjtot;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < mx * my * nvar; t += gridDim.x * blockDim.x) {
    const int m = t / (mx * my), rem = t % (mx * my);
    const int i = rem % mx + 2, j = rem / mx + 2;
    out[outoff[blockIdx.y] + t] = (double)q[m * plane + (long long)j * P.mitot + i];
  }
}
void launch_gather_interior2(const void* pool, const PatchDev* patches, const int* plist, const long long* outoff,
                             int np, int nvar, double* out, cudaStream_t s, bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    if (f32)
      gather_interior2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<const float*>(pool), patches, plist + base, outoff + base, nvar, out);
    else
      gather_interior2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<const double*>(pool), patches, plist + base, outoff + base, nvar, out);
    AMR_CUDA(cudaGetLastError());
  }
}

// The whole arrays (ghost cells included) of the listed patches, q(m,i,j) with m fastest,
// for binary output: a cell comes from store1 when the last step wrote it there (the
// interior, or after split steps the cells of interior i) and else from the other buffer:
// the step's input, whose ghost cells that step's fill set (or, before any step, the second
// copy of the initial values, whose ghost cells are zero as the reference's are after
// setgrd.f swaps its stores).
template <class T>
__global__ void gather_enlarged2_kernel(const T* pool, const PatchDev* patches, const int* plist, const long long* outoff,
                                        int nvar, double* out, int split) {
  const PatchDev P = patches[plist[blockIdx.y]];
  const long long plane = (long long)P.mitot * P.mjtot;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < plane; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % P.mitot), j = (int)(c / P.mitot);
    const bool in_i = i >= 2 && i < P.mitot - 2, in_j = j >= 2 && j < P.mjtot - 2;
    const bool written = split ? in_i : (in_i && in_j);
    const T* q = pool + (written ? P.q[P.cur] : P.q[1 - P.cur]);
    for (int m = 0; m < nvar; ++m) out[outoff[blockIdx.y] + c * nvar + m] = (double)q[m * plane + c];
  }
}
void launch_gather_enlarged2(const void* pool, const PatchDev* patches, const int* plist, const long long* outoff, int np,
                             int nvar, double* out, int split, cudaStream_t s, bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    if (f32)
      gather_enlarged2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<const float*>(pool), patches, plist + base, outoff + base, nvar, out, split);
    else
      gather_enlarged2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<const double*>(pool), patches, plist + base, outoff + base, nvar, out, split);
    AMR_CUDA(cudaGetLastError());
  }
}

// ======================================================================= Richardson estimation
// coarsen.f:4-33: 2x2 means of scratch rect rect_of[k] (twice the ghost width) into the
// first buffer of virtual patch k (its enlarged array, ghost cells included); FP64 sums
template <class T>
__global__ void coarsen2_kernel(T* pool, const ScratchRect* rects, const int* rect_of, const PatchDev* vp, int nvar) {
  const int k = blockIdx.y;
  const PatchDev P = vp[k];
  const ScratchRect R = rects[rect_of[k]];
  const T* src = pool + R.off;
  T* dst = pool + P.q[0];
  const long long splane = (long long)R.ni * R.nj, dplane = (long long)P.mitot * P.mjtot;
  const int n = P.mitot * P.mjtot;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n * nvar; t += gridDim.x * blockDim.x) {
    const int m = t / n, rem = t % n;
    const int i = rem % P.mitot, j = rem / P.mitot;
    const T* s0 = src + m * splane + (long long)(2 * j) * R.ni + 2 * i;
    const double v = ((((double)s0[0] + (double)s0[1]) + (double)s0[R.ni]) + (double)s0[R.ni + 1]) / 4.0;
    dst[m * dplane + (long long)j * P.mitot + i] = (T)v;
  }
}
void launch_coarsen2(void* pool, const ScratchRect* rects, const int* rect_of, const PatchDev* vp, int np, int nvar,
                     cudaStream_t s, bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    if (f32) coarsen2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<float*>(pool), rects, rect_of + base, vp + base, nvar);
    else coarsen2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<double*>(pool), rects, rect_of + base, vp + base, nvar);
    AMR_CUDA(cudaGetLastError());
  }
}

// errf1.f:40-71: for each 2x2 block of interior cells of patch k, the mean of component 1
// after the regular step (second buffer of virtual patch np+k) against the coarse cell
// after the big step (second buffer of virtual patch k); one byte est >= tol per block,
// blocks i fastest from outoff[k]
template <class T>
__global__ void errf2_kernel(const T* pool, const PatchDev* vp, int np, int ng, double order, double tol,
                             const long long* outoff, int8_t* out) {
  const int k = blockIdx.y;
  const PatchDev C = vp[k], F = vp[np + k];
  const int nxc = (F.ihi - F.ilo + 1) / 2, nyc = (F.jhi - F.jlo + 1) / 2;
  const T* fine = pool + F.q[1];
  const T* crse = pool + C.q[1];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nxc * nyc; t += gridDim.x * blockDim.x) {
    const int ic = t % nxc, jc = t / nxc;
    const T* f0 = fine + (long long)(2 * jc + ng) * F.mitot + (2 * ic + ng);
    const double t1 = (double)f0[0], t2 = (double)f0[1], t3 = (double)f0[F.mitot + 1], t4 = (double)f0[F.mitot];
    const double aval = (((t1 + t2) + t3) + t4) / 4.0;
    const double est = fabs((aval - (double)crse[(long long)(jc + ng) * C.mitot + (ic + ng)]) / order);
    out[outoff[k] + t] = est >= tol ? 1 : 0;
  }
}
void launch_errf2(const void* pool, const PatchDev* vp, int np, int ng, double order, double tol, const long long* outoff,
                  int8_t* out, cudaStream_t s, bool f32) {
  for (int base = 0; base < np; base += 65535) {
    const int n = std::min(65535, np - base);
    // virtual patches base..base+n-1 and their regular-step partners np+base..: pass the
    // array from base with the partner distance np unchanged
    if (f32)
      errf2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<const float*>(pool), vp + base, np, ng, order, tol, outoff + base, out);
    else
      errf2_kernel<<<dim3(8, n), 128, 0, s>>>(static_cast<const double*>(pool), vp + base, np, ng, order, tol, outoff + base, out);
    AMR_CUDA(cudaGetLastError());
  }
}

}  // namespace amrb
