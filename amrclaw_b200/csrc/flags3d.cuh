// Level-wide int8 flag arrays of 3D regridding on the device (flglvl.f and the
// routines it drives). An array of level L covers (0:is+1, 0:js+1, 0:ks+1) with is,
// js, ks the level's cell counts (iregsz, jregsz, kregsz), i fastest, the ring of one
// cell on every side as in the reference's integer*1 arrays.
#pragma once
#include "common.cuh"
#include "kernels3d.cuh"

namespace amrb {

struct LvlDims {
  int is, js, ks;
  __host__ __device__ long long size() const { return (long long)(is + 2) * (js + 2) * (ks + 2); }
  __host__ __device__ long long at(int i, int j, int k) const { return i + (long long)(is + 2) * (j + (long long)(js + 2) * k); }
};

// One box (array coordinates, inclusive) of domprep.f (value 1) or projec.f (3 where 0).
struct LvlBox { int i0, i1, j0, j1, k0, k1; };

// per: periodic directions (bit 0 x, bit 1 y, bit 2 z). The border ring of a periodic
// direction is the periodic image of the far interior layer, over the whole ring face.
// domprep.f:4-169: zero, the boxes set to 1, then the border ring.
void launch_domprep(int8_t* a, LvlDims d, const LvlBox* boxes, int nbox, cudaStream_t s, int per = 0);
// domshrink.f:4-93: 27-cell erosion of `in` into a fresh `out` (zero ring), then
// extend_borders in the non-periodic directions (the periodic ones keep the zero ring).
void launch_domshrink(const int8_t* in, int8_t* out, LvlDims d, cudaStream_t s, int per = 0);
// domup.f:4-185: a fresh fine array from the coarse one, then the border ring.
void launch_domup(const int8_t* crse, LvlDims cd, int8_t* fine, LvlDims fd, int rx, int ry, int rz, cudaStream_t s, int per = 0);
// domcopy.f:4-82: the border ring of the copied array (extend_borders, all directions).
void launch_domcopy_borders(int8_t* a, LvlDims d, cudaStream_t s, int per);
// spest.f: the interior of `f` set to 0 (the ring keeps its values).
void launch_zero_interior(int8_t* f, LvlDims d, cudaStream_t s);
// spest.f + flag2refine.f + setflags.f: BADPT (2) or GOODPT (0) into the level array for
// every interior cell of the patches in plist (patch cells at [cell0[p], cell0[p+1])).
// f32: the pool holds floats (the FP32 form); the differences are taken in FP64.
void launch_flag_cells3(const void* pool, const PatchDev* patches, const int* plist, const long long* cell0, int np,
                        long long ncells, int flag_pressure, double gamma1, double tolsp, int nvar, int8_t* f, LvlDims d,
                        cudaStream_t s, bool f32);
// bufnst.f + projec.f + shiftset.f: project the boxes (3 where 0), zero the ring, then
// add the ibuff-dilated flags (t1, t2: scratch arrays of the same dims).
void launch_bufnst3(int8_t* f, LvlDims d, const LvlBox* proj, int nproj, int ibuff, int8_t* t1, int8_t* t2, cudaStream_t s);
// colate.f:4-78: f = min(f, dom) over the interior.
void launch_colate3(int8_t* f, const int8_t* dom, LvlDims d, cudaStream_t s);

// A cluster's box in the level array (1-based interior indices, inclusive).
struct SigBox { int lo[3], hi[3]; };
// signs.f:4-86: for every box, the counts of flagged cells (f != 0) per i, per j and per k
// of the box: hist[off[b] .. +ni) per i, then nj per j, then nk per k. total: ints of
// hist; maxlen: the largest ni+nj+nk; maxrows: the largest nj*nk (i-rows of a box).
void launch_signatures3(const int8_t* f, LvlDims d, const SigBox* boxes, int nbox, const int* off, int total, int maxlen,
                        long long maxrows, int* hist, cudaStream_t s);
// 2D: the level's flag array as a one-plane array (d.ks = 1): zeroed, then 1 at every point
// (pts: n pairs of 0-based level indices i, j) at array position (i+1, j+1, 1)
void launch_scatter_points2(const int* pts, int n, int8_t* f, LvlDims d, cudaStream_t s);

// Richardson estimation (errest.f, coarsen.f, errf1.f). vp[0..np): virtual patches of the
// coarsened grids, vp[np..2np): those of the regular step (same index boxes as the grids).
// coarsen.f:1-25: the 2x2x2 means of scratch rect rect_of[k] (twice the ghost width) into
// the first buffer of vp[k], ghost cells included; FP64 sums.
void launch_coarsen3(void* pool, const Rect3* rects, const int* rect_of, const PatchDev* vp, int np, int nvar, cudaStream_t s,
                     bool f32);
// errf1.f:55-116 + setflags.f: for every 2x2x2 block of interior cells of grid k, the mean
// of component 1 after the regular step (second buffer of vp[np+k]) against the coarse
// cell after the big step (second buffer of vp[k]); where |difference / order| >= tol,
// BADPT is added to the block's eight cells of the level array f.
void launch_errf3(const void* pool, const PatchDev* vp, int np, double order, double tol, int8_t* f, LvlDims d, cudaStream_t s,
                  bool f32);

}  // namespace amrb
