// Work-item and op structures shared by the 2D host orchestrator and its kernels.
#pragma once
#include "common.cuh"
#include "riemann2d.cuh"

namespace amrb {

constexpr int TILE2 = 16;      // interior cells per tile side in the 2D patch step
constexpr int STEP2_THREADS = 256;
constexpr int STEP2_RC = 6;    // rows per Riemann chunk

// One tile of one patch (the batched path launches all tiles of a level at once).
struct StepWork {
  int patch;
  int ti0, tj0;          // tile origin, 1-based interior indices
  int fsv_start, fsv_count;  // fluxsv entries owned by this tile
  int fad_start, fad_count;  // fluxad segments owned by this tile
};

// fluxsv.f:10-109: coarse flux at a face next to a finer grid, written into the kid's register.
struct FsvEntry {
  int ic, jc;            // coarse cell, 1-based interior indices
  int side;              // listbc side code 1..4
  int pad;
  long long dst;         // register-pool offset of svdflx(:, lkid) of the kid
};
// fluxad.f:7-96: fine fluxes over one coarse segment, accumulated into the patch's own register.
struct FadEntry {
  int side;              // 1 left, 2 top, 3 right, 4 bottom (register order of fluxad.f)
  int f0;                // first fine row (sides 1,3) or column (sides 2,4), 1-based interior
  int seg;               // 0-based register index (lind-1)
  int pad;
};

struct StepParams {
  ProbDev prob;
  int mthlim[MAXVAR];
  int order;             // method(2)
  int trans;             // method(3)
  int use_fwaves;
  int mcapa;
  int split;             // dimensional_split: 0 unsplit (stepgrid.f), 1 Godunov (stepgrid_dimSplit.f)
};

// pool: the patch pool, of double, or of float in the FP32 form (offsets count elements)
struct StepArgs {
  void* pool;
  double* regs;
  const PatchDev* patches;
  const StepWork* work;
  int nwork;
  int* queue;            // dynamic work queue counter (nullptr: static assignment)
  const FsvEntry* fsv;
  const FadEntry* fad;
  double dt, dx, dy;
  const double* dt_dev;  // if set, the time step is read here (a captured graph replays the launch)
  unsigned long long* cflmax;  // max Courant number of the level (bit pattern of a non-negative double)
  StepParams sp;
};

// The level substeps of up to STEP2_BATCH_MAX solves (of one Riemann plugin and one
// precision) in one launch: member k's tiles are items [work0[k], work0[k+1]) of the
// combined work list, stepped with m[k]. Passed to the kernel by value.
constexpr int STEP2_BATCH_MAX = 16;
struct StepBatch {
  int n;
  int work0[STEP2_BATCH_MAX + 1];
  StepArgs m[STEP2_BATCH_MAX];
};
static_assert(sizeof(StepBatch) < 32000, "a StepBatch must fit in the kernel parameter space");
// one launch of the batched step over b's members (grid: blocks; 0 launches nothing)
void launch_step2_batch(int solver, const StepBatch& b, int grid, cudaStream_t s, bool f32);

// ---------------------------------------------------------------- ghost-fill programs
enum FillKind { FILL_COPY = 0, FILL_INTERP = 1, FILL_PIECE = 2, FILL_FILVAL = 3, FILL_RING = 4, FILL_FIXCAPA = 5 };

struct ScratchRect {
  long long off;         // pool offset (doubles), layout [m][j][i]
  int ni, nj;
};

struct FillOp {
  int kind;
  int dst_patch;         // >= 0: store1 of this patch (enlarged array); -1: scratch rect dst_rect
  int dst_rect;
  int di0, dj0;          // region origin (0-based) inside the destination array
  int ni, nj;            // region extent
  int src;               // COPY: source patch; others: source scratch rect
  int si0, sj0;          // COPY/PIECE: origin in the source array (0-based); INTERP/FILVAL: global fine index of the region origin
  int level;             // COPY: source level for the time mode (-1: always store1); INTERP/FILVAL: fine level
  int cilo, cjlo;        // INTERP/FILVAL: global coarse index of the source rect origin
  int capa0;             // FIXCAPA: first of the source rect's coarse kappa values in FillArgs::capa
};
// FIXCAPA (fixcapaq.f): di0/dj0 and si0/sj0 as FILVAL (the fine region's origin), ni x nj the
// coarse cells the region covers; each unit is one coarse cell and its fine block.

struct FillChunk { int op, start, count; };

// bc2amr.f90:84-297 applied to one whole array (a patch or a scratch rect).
struct BcOp {
  int dst_patch, dst_rect;
  int nrow, ncol;
  int nxl, ibeg, nyb, jbeg;      // ghost extents (0: side not outside the domain)
  int bxl, bxr, byl, byr;        // boundary codes (1 extrap, 3 wall, 0/2 none)
};

struct FillArgs {
  void* pool;
  double* regs;
  const PatchDev* patches;
  const ScratchRect* rects;
  const FillOp* ops;
  const FillChunk* chunks;
  int nchunks;
  int nvar;
  SrcMode modes;
  const SrcMode* modes_dev;  // if set, the time-interpolation modes are read here (captured graphs)
  LevelConst lc;
  double xlower, ylower;
  int mcapa;                 // capacity component of the patches' aux (FIXCAPA)
  const double* capa;        // coarse kappa of the FIXCAPA ops' source rects
};

struct BcArgs {
  void* pool;
  const PatchDev* patches;
  const ScratchRect* rects;
  const BcOp* ops;
  int nops;
  int nvar;
};

// ---------------------------------------------------------------- registers, update
struct QadJob { int patch; int side; int seg0; int nseg; int pos0; };  // one side of one fine patch

struct UpbndCell { int patch; int ie, je; int first, count; };   // upbnd.f:62-124, per coarse cell
struct UpbndTerm { long long reg; double sgn; };
struct AvgRect { int cpatch, kpatch; int ci0, cj0, ni, nj; int fi0, fj0; };  // update.f:95-175

struct GaugeJob { int patch; int ii, jj; int slot; double xoff, yoff; };

// Launch wrappers (kernels2d.cu). f32: the pool holds float (the FP32 form): storage,
// Riemann solves and flux differencing in FP32; flux registers, register corrections,
// time interpolation weights, averages and totals in FP64.
void launch_step2(int solver, const StepArgs& a, int grid, cudaStream_t s, bool f32);
void launch_fill(const FillArgs& a, cudaStream_t s, bool f32);
// one launch over the chunks of two independent programs (b may have no chunks)
void launch_fill_pair(const FillArgs& a, const FillArgs& b, cudaStream_t s, bool f32);
// both boundary phases of the ops of two independent programs in one launch
void launch_bc_pair(const BcArgs& a, const BcArgs& b, cudaStream_t s, bool f32);
void launch_bc(const BcArgs& a, int phase, cudaStream_t s, bool f32);
// dt_dev: if set, delt is read there (captured graphs)
void launch_qad2(int solver, void* pool, double* regs, const PatchDev* patches, const QadJob* jobs, int njobs,
                 const ProbDev& prob, int nvar, LevelConst lc, double delt, cudaStream_t s, bool f32,
                 const double* dt_dev = nullptr);
void launch_upbnd(void* pool, const double* regs, const PatchDev* patches, const UpbndCell* cells, int ncells,
                  const UpbndTerm* terms, double area, int nvar, cudaStream_t s, bool f32);
// mcapa > 0: kappa-weighted averages (update.f:150-160)
void launch_average(void* pool, const PatchDev* patches, const AvgRect* rects, int nrects, int rx, int ry, int nvar,
                    cudaStream_t s, bool f32, int mcapa = 0);
void launch_flags2(const void* pool, const PatchDev* patches, const int* plist, const long long* outoff, int np,
                   int use_old, int flag_component, double tolsp, int nvar, int8_t* out, cudaStream_t s, bool f32);
void launch_gauges2(const void* pool, const PatchDev* patches, const GaugeJob* jobs, int njobs, int nvar,
                    double* out, cudaStream_t s, bool f32);
void launch_zero_tiny(void* pool, const PatchDev* patches, const int* plist, int np, int nvar, cudaStream_t s, bool f32);
void launch_mass2(const void* pool, const PatchDev* patches, const int* plist, int np, double* out, cudaStream_t s, bool f32,
                  int mcapa = 0);
// whole arrays (ghost cells included) in the reference's q(m,i,j) order, for binary output
void launch_gather_enlarged2(const void* pool, const PatchDev* patches, const int* plist, const long long* outoff, int np,
                             int nvar, double* out, int split, cudaStream_t s, bool f32);
void launch_gather_interior2(const void* pool, const PatchDev* patches, const int* plist, const long long* outoff,
                             int np, int nvar, double* out, cudaStream_t s, bool f32);
size_t step2_smem_bytes(int solver, bool f32);
// Richardson estimation (errest.f): rect_of[k] is the scratch rect of virtual patch k
void launch_coarsen2(void* pool, const ScratchRect* rects, const int* rect_of, const PatchDev* vp, int np, int nvar,
                     cudaStream_t s, bool f32);
// vp[0..np): the big-step patches, vp[np..2np): the regular-step patches
void launch_errf2(const void* pool, const PatchDev* vp, int np, int ng, double order, double tol, const long long* outoff,
                  int8_t* out, cudaStream_t s, bool f32);

}  // namespace amrb
