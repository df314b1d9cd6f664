// Shared device/host definitions for the B200 patch-advance path.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#define AMR_CUDA(x)                                                                       \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess)                                                                \
      throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e_) +      \
                               " at " + __FILE__ + ":" + std::to_string(__LINE__));       \
  } while (0)

namespace amrb {

constexpr int MAXLV = 10;
constexpr int MAXVAR = 5;

// Flag values of the reference (src/2d/amr_module.f90:163-168), stored as int8 codes.
constexpr int8_t FLAG_UNSET = -1, FLAG_DONT = 0, FLAG_DO = 2, FLAG_BADPRO = 3;

// Device descriptor of one patch (one grid number of the reference's node/rnode tables,
// src/2d/amr_module.f90:30-151). Storage lives in the pool; layout per variable is
// [m][j][i] over the enlarged patch (ghost cells included), i fastest.
struct PatchDev {
  long long q[2];      // pool offsets (Reals) of the two solution buffers; q[cur] is store1
  long long ffl;       // register-pool offset (doubles) of the fine-side flux registers, -1 if none
  int cur;             // which buffer holds the current solution
  int ilo, ihi, jlo, jhi, klo, khi;
  int mitot, mjtot, mktot;
  int level;
  int lenbc;
  int pad;
  long long aux;       // pool offset of the aux array [maux][k][j][i] of the enlarged patch (3D), -1 if none
};

// Per-level constants that device code needs (spacing, ratios, domain sizes).
struct LevelConst {
  double hx[MAXLV + 2], hy[MAXLV + 2], hz[MAXLV + 2];
  int iregsz[MAXLV + 2], jregsz[MAXLV + 2], kregsz[MAXLV + 2];
  int intratx[MAXLV + 2], intraty[MAXLV + 2], intratz[MAXLV + 2];
};

// Time-interpolation mode of one source level for a ghost fill (intfil.f90:183-232).
struct SrcMode {
  int mode[MAXLV + 2];     // 0: store1 (new), 1: store2 (old), 2: alphai*new + alphac*old
  double alphai[MAXLV + 2], alphac[MAXLV + 2];
};

// cur ^= 1 for every patch in plist (the step wrote the other buffer); kernels2d.cu.
void launch_flip(PatchDev* patches, const int* plist, int np, cudaStream_t s);

}  // namespace amrb
