/* amrgpu_riemann.cuh: the device Riemann-solver plugin contract of amrclaw_b200.
 *
 * The reference calls user-supplied Fortran routines per 1D slice:
 *   rpn2(ixy, maxm, meqn, mwaves, maux, mbc, mx, ql, qr, auxl, auxr, wave, s, amdq, apdq)
 *     at src/2d/flux2.f:125-126 and src/2d/qad.f:129-130,207-208,268-269,334-335;
 *   rpt2(ixy, imp, maxm, meqn, mwaves, maux, mbc, mx, ql, qr, aux1, aux2, aux3, asdq,
 *        bmasdq, bpasdq)  at src/2d/flux2.f:202-204 (imp = 1) and :219-221 (imp = 2);
 *   rpn3 / rpt3(ixyz, icoor, imp, ...) / rptt3(ixyz, icoor, imp, impt, ...)
 *     at src/3d/flux3.f:220-226, 302-365 and 411-422, 538-545.
 * Device code cannot call Fortran, so a plugin here is a device functor evaluated at ONE
 * interface per call, with the same argument meaning; the patch-step kernels are
 * templates instantiated on it, and amrgpu_set_solver selects a registered plugin by
 * name and sets its constants (the reference's /cparam/ common block).
 *
 * 2D plugin (a struct S; R is float or double; P is the constants struct):
 *   static constexpr int MEQN, MWAVES, NAUX;
 *   __device__ static void rpn(const P&, int ixy, const R* qL, const R* qR,
 *                              const R* auxL, const R* auxR,
 *                              R (&wave)[MWAVES][MEQN], R (&s)[MWAVES],
 *                              R (&amdq)[MEQN], R (&apdq)[MEQN]);
 *       qL: the state left of the interface (cell i-1), qR: right of it (cell i);
 *       auxL, auxR: their aux values (the reference's auxr(:,i-1), auxl(:,i));
 *   __device__ static void rpt(const P&, int ixy, int imp, const R* qL, const R* qR,
 *                              const R* aux1, const R* aux2, const R* aux3,
 *                              const R* asdq, R (&bmasdq)[MEQN], R (&bpasdq)[MEQN]);
 *       imp = 1 splits amdq (cell i-1), imp = 2 splits apdq (cell i); aux1/aux2/aux3 are
 *       the aux values of that cell in the rows below, at and above the sweep's row (the
 *       reference's aux1/aux2/aux3 slices at index i-2+imp).
 *   NAUX: the leading aux components the plugin reads (0: none; the aux pointers may then
 *   be null).
 *
 * 3D plugin (a struct S<R> holding the interface's per-call state):
 *   static constexpr int NV (meqn), NW (mwaves);
 *   template <int DIR> __device__ void load(pool, patch, base, step, plane, e);
 *       reads the aux values the interface needs (nothing for Euler);
 *   template <int DIR> __device__ void rpn(const Step3Params&, const R* QL, const R* QR,
 *                                          R (&W)[NW][NV], R* S, R* AM, R* AP);
 *   template <int DIR> __device__ void rpt(int imp, int icoor, const R* in, R* m, R* p) const;
 *   template <int DIR> __device__ void rptt(int imp, int icoor, int impt, const R* in,
 *                                           R* m, R* p) const;
 *       DIR = ixyz; icoor 2: the y-like, 3: the z-like transverse direction of the sweep;
 *       impt: the side (1 minus, 2 plus) of the first transverse split.
 *
 * Every expression of a plugin must be evaluated in a fixed order (the library is built
 * without FMA contraction) so FP64 results are bit-identical to the CPU restatement.
 */
#ifndef AMRGPU_RIEMANN_CUH
#define AMRGPU_RIEMANN_CUH

#include <type_traits>
#include <utility>

namespace amrgpu_plugin {

/* Compile-time check of the 2D contract: instantiated on every registered 2D plugin. */
template <class S, class P, class R>
struct Check2D {
  static constexpr int ME = S::MEQN, MW = S::MWAVES;
  using Rpn = decltype(S::template rpn<R>(std::declval<const P&>(), 1, (const R*)nullptr, (const R*)nullptr,
                                         (const R*)nullptr, (const R*)nullptr, std::declval<R (&)[MW][ME]>(),
                                         std::declval<R (&)[MW]>(), std::declval<R (&)[ME]>(), std::declval<R (&)[ME]>()));
  using Rpt = decltype(S::template rpt<R>(std::declval<const P&>(), 1, 1, (const R*)nullptr, (const R*)nullptr,
                                         (const R*)nullptr, (const R*)nullptr, (const R*)nullptr, (const R*)nullptr,
                                         std::declval<R (&)[ME]>(), std::declval<R (&)[ME]>()));
  static constexpr bool value = ME >= 1 && MW >= 1 && S::NAUX >= 0 && std::is_void<Rpn>::value && std::is_void<Rpt>::value;
};

/* Compile-time check of the 3D contract: instantiated on every registered 3D plugin. */
template <class S, class SP, class R>
struct Check3D {
  static constexpr int NV = S::NV, NW = S::NW;
  using Rpn = decltype(std::declval<S&>().template rpn<1>(std::declval<const SP&>(), (const R*)nullptr,
                                                         (const R*)nullptr, std::declval<R (&)[NW][NV]>(),
                                                         (R*)nullptr, (R*)nullptr, (R*)nullptr));
  using Rpt = decltype(std::declval<const S&>().template rpt<1>(1, 2, (const R*)nullptr, (R*)nullptr, (R*)nullptr));
  using Rptt = decltype(std::declval<const S&>().template rptt<1>(1, 2, 1, (const R*)nullptr, (R*)nullptr, (R*)nullptr));
  static constexpr bool value =
      NV >= 1 && NW >= 1 && std::is_void<Rpn>::value && std::is_void<Rpt>::value && std::is_void<Rptt>::value;
};

}  // namespace amrgpu_plugin

#endif /* AMRGPU_RIEMANN_CUH */
