// The interface the C ABI drives: one AMR solve on one device (2D or 3D).
#pragma once
#include <algorithm>
#include <cuda_runtime.h>
#include <string>
#include <vector>

namespace amrb {

class AmrSolver {
 public:
  virtual ~AmrSolver() = default;
  virtual int num_dim() const = 0;
  virtual cudaStream_t stream() const = 0;  // the stream the solve's work is ordered on
  virtual void set_batched(bool on) = 0;
  virtual void set_profile(bool on) = 0;
  // replay each level substep from captured CUDA graphs (3D path)
  virtual void set_graphs(bool on) = 0;
  // sweep schedule of the batched 3D path: 0 autotune, 1 per direction, 2 work queue
  virtual void set_schedule(int s) = 0;
  // the Riemann solver plugin by registry name and its problem constants (the reference's
  // link-time choice of rpn2/rpt2 (rpn3/rpt3/rptt3) and setprob's /cparam/ common block);
  // std::invalid_argument for an unknown name, a wrong number of constants or a solver
  // whose equations and waves do not match the run
  virtual void set_solver(const std::string& name, const std::vector<double>& params) = 0;
  // cap the device pools (patch storage and scratch, flux registers) at `bytes` in all;
  // growth past it throws PoolLimitError. 0 removes the cap. The pools already hold
  // pool_bytes(); a cap below that is refused (std::invalid_argument).
  virtual void set_pool_limit(long long bytes) = 0;
  // hand each batched level step to the process's step batcher, which launches the steps
  // that solves of the same plugin and precision submit within window_us together (2D);
  // 0 launches them alone. std::invalid_argument for a negative window or a 3D solve.
  virtual void set_step_batching(int window_us) = 0;
  virtual void run(int max_cycles) = 0;                    // tick.f
  virtual double level_advance(int level, double* cfl) = 0;  // advanc.f; returns dtnew
  virtual void update_level(int level) = 0;                 // update.f
  virtual void regrid_from(int lbase) = 0;                  // regrid.f
  virtual void valout(const char* dir) = 0;                 // valout.f90 (dir == nullptr: the run's output dir)
  virtual void write_checkpoint(const char* path) = 0;      // check.f (path == nullptr: fort.chkNNNNN in the output dir)
  virtual double mass() = 0;                                // conck.f, level 1
  virtual std::vector<double> info() = 0;
  virtual std::vector<int> grid_rows() = 0;                 // 2 + 2*num_dim ints per grid
  virtual std::vector<double> values() = 0;
  // the number of doubles values() returns, without gathering them
  virtual long long value_count() = 0;
  // values() written straight into out (room for value_count() doubles)
  virtual void values_into(double* out) {
    const std::vector<double> v = values();
    std::copy(v.begin(), v.end(), out);
  }
  virtual std::vector<double> gauge_rows() = 0;             // (3 + nvar) doubles per sample
};

// Builds and initialises the 3D solver (amr3d.cu) from the data files in rundir.
// f32: the FP32 form (float storage, Riemann solves and fluxes; FP64 registers and totals)
AmrSolver* make_solver3(const std::string& rundir, const std::string& outdir, bool write_output, bool f32);
// Builds and initialises the 1D solver (amr1d.cu); FP64 only
AmrSolver* make_solver1(const std::string& rundir, const std::string& outdir, bool write_output);

}  // namespace amrb
