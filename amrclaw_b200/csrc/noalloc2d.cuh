// Fixed-scratch ghost-fill executor (noalloc2d.cu).
#pragma once
#include "kernels2d.cuh"

#include <string>

namespace amrb {

// Capacity of the fixed device scratch array: 4 Mi doubles (32 MiB).
constexpr long long NOALLOC_SCRATCH_DOUBLES = 4LL << 20;

// Address of the fixed scratch array on the current device. The first call on
// a device looks the address up (cudaGetSymbolAddress); later calls return the
// cached value. Returns non-zero with a message on failure.
int fixed_scratch_address(double** out, std::string& err);

// The fill and boundary-condition kernels with scratch rect r placed at
// scratch + (rects[r].off - off0).
void launch_fill_fixed(const FillArgs& a, const double* scratch, long long off0, cudaStream_t s);
void launch_bc_fixed(const BcArgs& a, int phase, const double* scratch, long long off0, cudaStream_t s);

}  // namespace amrb
