// Work items and launch wrappers of the 3D patch-advance kernels (kernels3d.cu).
#pragma once
#include "common.cuh"
#include "riemann3d.cuh"

namespace amrb {

// Number of per-cell values a sweep leaves for the face kernel for nv equations:
// faddm(nv), faddp(nv), gadd(2 sides x 3 offsets x nv), hadd(2 x 3 x nv).
__host__ __device__ constexpr int stash_values(int nv) { return 14 * nv; }
constexpr int STASH3 = stash_values(5);

// Riemann plugins of the 3D device path (the problem's rpn3/rpt3/rptt3)
enum Solver3 { SOLVER3_EULER = 0, SOLVER3_SWIRL = 1 };

struct Step3Params {
  int solver;  // Solver3
  double gamma, gamma1;
  int efix;
  int mthlim[3];
  int order;   // method(2)
  int m3, m4;  // method(3) = 10*m3 + m4
};

// All patches of a level: prefix sums of the sweep items and face cells per patch.
// pool, stash and flux hold double, or float in the FP32 form (offsets count elements)
struct Step3Args {
  const void* pool;
  double* newq;              // nullptr: update in place is not used; q[1-cur] is written
  const PatchDev* patches;
  const int* plist;          // patch ids of the level, in level order
  int np;
  const long long* sweep0;   // [3][np+1]: first stash slot of each patch, per direction ((n1+1) per pencil)
  const long long* comp0;    // [3][np+1]: first interface of each patch, per direction ((n1+3) per pencil)
  const long long* face0;    // [np+1]: first face cell of each patch ((mx+1)(my+1)(mz+1) each)
  const long long* cell0;    // [np+1]: first interior cell of each patch (mx*my*mz each)
  long long stash_stride;    // slots of one direction region x 3 (SoA stride)
  void* stash;               // [stash_values(meqn)][stash_stride]
  void* flux;                // [6 comps][meqn][face cells]
  long long flux_stride;     // face cells of the level
  double dt, dx, dy, dz;
  const double* dt_dev;      // if set, the time step is read here (a captured graph replays the launch)
  unsigned long long* cflmax;
  unsigned int* queue;       // if set: the sweeps of all three directions run as one persistent work-queue launch
  Step3Params sp;
  // dimensionally split step (stepgrid_dimSplit.f): [3][np+1] first interface of each patch
  // per direction over the split pencils, [np+1] first enlarged cell of each patch in the
  // level's split scratch (the y-updated values), and that scratch
  const long long* scomp0 = nullptr;
  const long long* ecell0 = nullptr;
  void* split = nullptr;
};

// fluxsv.f:4-94 entries (coarse patch faces next to a kid) and fluxad.f:4-155 registers.
struct Fsv3 { int patch; int pidx; int i, j, k, side; long long dst; };  // i,j,k: 1-based interior cell
struct Fad3 { int patch; int pidx; int side; int a0, b0; int na, nb; int seg; };  // one coarse face of a fine patch

struct Qad3Job { int patch; int side; int slab; int row0; int nreg; int reg0; int ratio_a, ratio_b; };

// ghost fill (filpatch.f / intfil.f / filval.f / cstore.f as programs)
// F3_PIECE: a scratch rect's cells (src, from si0, sj0, sk0) copied into place: the pieces
// prefilp.f fills at periodically shifted indices
enum Fill3Kind { F3_COPY = 0, F3_INTERP = 1, F3_FILVAL = 2, F3_RING = 3, F3_PIECE = 4 };
struct Rect3 { long long off; int ni, nj, nk; };
struct Fill3Op {
  int kind;
  int dst_patch, dst_rect;
  int di0, dj0, dk0;     // origin (0-based) in the destination array
  int ni, nj, nk;        // extent
  int src;               // COPY: patch; INTERP/FILVAL/RING: rect
  int si0, sj0, sk0;     // COPY/PIECE: origin in the source array; INTERP/FILVAL: global fine index of the origin
  int level;             // COPY: source level for time modes (-1: current); INTERP/FILVAL: fine level
  int cilo, cjlo, cklo;  // global coarse index of the rect origin
};
struct Fill3Chunk { int op; long long start; int count; };
struct Bc3Op {
  int dst_patch, dst_rect;
  int nrow, ncol, nfil;
  int nxl, ibeg, nyl, jbeg, nzl, kbeg;   // ghost extents (0: side inside the domain)
  int bxl, bxr, byl, byr, bzl, bzr;      // boundary codes (1 extrapolation, 3 wall)
};
struct Fill3Args {
  void* pool; double* regs;
  const PatchDev* patches;
  const Rect3* rects;
  const Fill3Op* ops;
  const Fill3Chunk* chunks; int nchunks;
  int nvar;
  SrcMode modes;
  const SrcMode* modes_dev;  // if set, the time-interpolation modes are read here (captured graphs)
  LevelConst lc;
  double xlower, ylower, zlower;
};
struct Bc3Args { void* pool; const PatchDev* patches; const Rect3* rects; const Bc3Op* ops; int nops; int nvar; };

struct Avg3 { int cpatch, kpatch; int ci0, cj0, ck0, ni, nj, nk; int fi0, fj0, fk0; };
struct Upbnd3Cell { int patch; int ie, je, ke; int first, count; };
struct Upbnd3Term { long long reg; double sgn; };
struct Gauge3Job { int patch; int ii, jj, kk; int slot; double xoff, yoff, zoff; };

// Launch wrappers (kernels3d.cu). f32: the FP32 form (float storage, Riemann solves and
// flux differencing; FP64 registers, register corrections, averages and totals).
// interfaces_per_dir: the interfaces (comp0 ranges) of each sweep direction.
// returns the number of kernels launched
// Two side streams and the events that fork them off the solve's stream and join them back:
// the three sweep directions of a level (independent of one another) then run at once, and
// the tail blocks of one direction overlap the others instead of leaving SMs idle.
struct SweepStreams {
  cudaStream_t side[2];
  cudaEvent_t fork, join[2];
};
int launch_step3(const Step3Args& a, const long long interfaces_per_dir[3], long long faces, long long cells, cudaStream_t s, bool f32,
                 const SweepStreams* ss = nullptr);
// the Godunov-split step of the level (stepgrid_dimSplit.f): x, y and z sweeps with their
// updates, interfaces_per_dir counting the split pencils (scomp0); returns launches made
int launch_split3(const Step3Args& a, const long long interfaces_per_dir[3], cudaStream_t s, bool f32);
// pencils of a patch of mx x my x mz cells in the split sweep of direction d (0, 1, 2):
// x along every (j, k) row of the enlarged patch, y along the interior i and every k,
// z along the interior (i, j)
__host__ __device__ inline long long split_pencils(int d, long long mx, long long my, long long mz) {
  return d == 0 ? (my + 4) * (mz + 4) : d == 1 ? mx * (mz + 4) : mx * my;
}
// Builds the level's fluxad/qad work lists on the device: pre[np+1] is the prefix of the
// register segments (lenbc) of the patches in plist (0 for patches without registers).
void launch_expand_fadqad3(const int* plist, const long long* pre, int np, const PatchDev* patches, int rx, int ry, int rz,
                           long long total, Fad3* fad, Qad3Job* qad, cudaStream_t s);
// dt_dev / c_dev: if set, the scalar is read from device memory instead (captured graphs)
void launch_fsv3(const void* flux, long long flux_stride, const long long* face0, const PatchDev* patches, double* regs,
                 const Fsv3* e, int n, int nvar, double dtc, double hx, double hy, double hz, cudaStream_t s, bool f32,
                 const double* dt_dev = nullptr);
void launch_fad3(const void* flux, long long flux_stride, const long long* face0, const PatchDev* patches, double* regs,
                 const Fad3* e, int n, int nvar, double dtf, double hx, double hy, double hz, cudaStream_t s, bool f32,
                 const double* dt_dev = nullptr);
void launch_qad3(void* pool, double* regs, const PatchDev* patches, const Qad3Job* jobs, int njobs, Step3Params sp,
                 int nvar, double hx, double hy, double hz, double delt, cudaStream_t s, bool f32, const double* dt_dev = nullptr);
// setaux of the swirl from its one-dimensional factors: for a patch whose enlarged array
// has mi x mj x mk cells and whose aux block starts at pool offset `aux`, fac + f0 holds
// ua, va, wa [mi], ub, vb, wb [mj], uc, vc, wc [mk]; the kernel writes
// aux = (ua*ub)*uc, (va*vb)*vc, (wa*wb)*wc in [3][k][j][i], `copies` times (the
// time-modulated field keeps a second, unscaled copy)
struct Setaux3Job { long long aux, f0; int mi, mj, mk, pad; };
void launch_setaux3(void* pool, const Setaux3Job* jobs, int njobs, long long max_cells, const double* fac, int copies,
                    cudaStream_t s, bool f32);
// valout.f90:140-147: |q| < 1e-90 of the interior cells of plist set to 0 in place
void launch_zero_tiny3(void* pool, const PatchDev* patches, const int* plist, int np, int nvar, cudaStream_t s, bool f32,
                       bool aux = false);
// b4step3 of the time-modulated swirl: aux = c * aux0 over the enlarged patches of plist
// (max_cells: the largest enlarged patch)
void launch_b4step3(void* pool, const PatchDev* patches, const int* plist, int np, int naux, long long max_cells, double c,
                    cudaStream_t s, bool f32, const double* c_dev = nullptr);
void launch_fill3(const Fill3Args& a, cudaStream_t s, bool f32);
void launch_bc3(const Bc3Args& a, int phase, cudaStream_t s, bool f32, long long max_lines);
void launch_upbnd3(void* pool, const double* regs, const PatchDev* patches, const Upbnd3Cell* cells, int n,
                   const Upbnd3Term* terms, double volume, int nvar, cudaStream_t s, bool f32);
void launch_average3(void* pool, const PatchDev* patches, const Avg3* r, int n, long long max_cells, int rx, int ry, int rz, int nvar,
                     cudaStream_t s, bool f32);
void launch_gauges3(const void* pool, const PatchDev* patches, const Gauge3Job* jobs, int n, int nvar, double* out, cudaStream_t s,
                    bool f32);
void launch_mass3(const void* pool, const PatchDev* patches, const int* plist, int np, double* out, cudaStream_t s, bool f32);
// whole arrays (ghost cells included) in the reference's q(m,i,j,k) order, for binary output
void launch_gather_enlarged3(const void* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np, int nvar,
                             long long total, double* out, bool aux, int split, cudaStream_t s, bool f32);
void launch_gather3(const void* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np, int nvar,
                    long long total, double* out, cudaStream_t s, bool f32, bool aux = false);

}  // namespace amrb
