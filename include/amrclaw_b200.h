/* amrclaw_b200: C ABI of the B200 patch-advance path of AMRClaw.
 *
 * The reference (mjberger/amrclaw) runs its level integrator inside the Fortran
 * program amr2/amr3; these entry points are what a Fortran 90 driver binds through
 * ISO_C_BINDING to hand that path to the GPU. All entry points
 * return an int status (AMRGPU_OK = 0); no exception crosses the boundary and the
 * text of the last error is available from amrgpu_last_error(). Host arrays passed
 * in are borrowed for the duration of the call. One context is used by one host
 * thread at a time.
 */
#ifndef AMRCLAW_B200_H
#define AMRCLAW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AMRGPU_OK 0
#define AMRGPU_ERROR 1
#define AMRGPU_EINVAL 2
#define AMRGPU_ENOMEM 3  /* a capped device pool would have to grow past its cap */

typedef struct amrgpu_ctx amrgpu_ctx;

/* Message of the last failed call on this thread (empty when none). */
const char* amrgpu_last_error(void);

/* Reads claw.data, amr.data, regions.data, gauges.data and setprob.data from
 * rundir (the files setrun.py writes), builds the initial hierarchy on the device
 * and writes frame 0 when output_t0 is set. num_dim in claw.data selects the 2D
 * path (amr2) or the 3D path (amr3: Euler equations, or advection in the swirl's
 * face-centred velocity field with aux arrays set by the problem's setaux).
 * Replaces the start-up of src/2d/amr2.f90:140-612 (input reading :148-394,
 * domain.f:4-110, setgrd.f:4-142, ginit.f:17-86, conck.f:6-73) and of
 * src/3d/amr3.f90 (domain.f, setgrd.f, ginit.f of src/3d). */
int amrgpu_init(const char* rundir, const char* outdir, int write_output, amrgpu_ctx** ctx);

/* amrgpu_init with a choice of precision. precision_bits = 64: the FP64 path, bit-
 * identical to the reference's arithmetic. precision_bits = 32: the FP32 form (2D and 3D):
 * patch storage, ghost values, aux arrays, Riemann solves and flux differencing in FP32; flux
 * registers (fluxsv/fluxad/qad sums), register corrections, averaging sums, totals and
 * time/dt bookkeeping in FP64. No counterpart in the reference (FP64 only). */
int amrgpu_init_precision(const char* rundir, const char* outdir, int write_output, int precision_bits, amrgpu_ctx** ctx);

/* 1: advance every patch of a level in one launch (batched path, default);
 * 0: one launch per patch (plain per-patch path). */
int amrgpu_set_batched(amrgpu_ctx* ctx, int batched);

/* 1: capture each level substep as two CUDA graphs (ghost fill, saveqc, qad; then CFL
 * reset, (3D) b4step3, the step kernels, fluxsv/fluxad, the store swap and the CFL
 * read-back) and replay them, re-capturing when a regrid changes the level's plans; the
 * per-substep scalars (dt, time-interpolation weights, the b4step3 factor) are copied to
 * the device before each replay. Results are identical to direct launches. 0: launch
 * directly (default). No counterpart in the reference. */
int amrgpu_set_graphs(amrgpu_ctx* ctx, int on);

/* Writes a checkpoint of the run at the current coarse-step boundary (check.f:4-104):
 * the scheduler state, the grid table with its free list, both solution buffers (and, in
 * 3D, the aux block) of every grid, and the gauge samples so far. path == NULL: fort.chkNNNNN
 * (NNNNN = coarse steps taken) in the output directory, or fort.chkaaaaa / fort.chkbbbbb
 * alternately when checkpt_style < 0. A run continues from it when claw.data sets
 * restart = T and restart_file (restrt.f: amrgpu_init reads it in place of the initial
 * grids); continuing gives the same results as the run that was not interrupted.
 * checkpt_style 2 (at checkpt_times) and 3 (every checkpt_interval coarse steps) write
 * them during amrgpu_run, and any style but 0 writes one at the end (tick.f:322-368).
 * The layout is this library's own, not the reference's fort.chk (one layout for 2D
 * runs, one for 3D). */
int amrgpu_checkpoint(amrgpu_ctx* ctx, const char* path);

/* Sweep schedule of the batched 3D path. 1 (default): one launch per sweep direction (a
 * block per tile of 128 interfaces); 2: one persistent work-queue launch in which resident
 * blocks take the tiles of all three directions from an atomic counter; 0: autotune per
 * level (the level's first substeps alternate the two, timed with CUDA events per
 * cell-update, and the faster is kept). Results are identical under every schedule.
 * 2D contexts accept only 0. No counterpart in the reference. */
int amrgpu_set_schedule(amrgpu_ctx* ctx, int schedule);

/* Selects the Riemann solver plugin of the run by registry name and sets its problem
 * constants (params[0..n), n = 0 keeps the current ones). Replaces the reference's
 * plugin binding: the rpn2/rpt2 (2D) or rpn3/rpt3/rptt3 (3D) routines linked into the
 * program and called at src/2d/flux2.f:125,202,219, src/2d/qad.f:129 and
 * src/3d/flux3.f:220-226,302-365,411-422, with their constants in setprob's /cparam/
 * common block (examples/advection_2d_square/setprob.f:4, examples/euler_2d_quadrants/
 * setprob.f:7). Registered device plugins (their per-interface contract is declared in
 * include/amrgpu_riemann.cuh):
 *   2D  "advection"       params u, v            (num_eqn 1, num_waves 1)
 *       "acoustics"       params rho, bulk       (num_eqn 3, num_waves 2)
 *       "euler_roe_efix"  params gamma[, efix]   (num_eqn 4, num_waves 4)
 *       "vc_advection"    no params; face velocities in aux 1..2 (num_eqn 1)
 *   3D  "euler_roe_efix"  params gamma[, efix]   (num_eqn 5, num_waves 3)
 *       "vc_advection"    no params; face velocities in aux 1..3 (num_eqn 1, num_aux 3)
 * Unknown names, a wrong count or invalid constants, and solvers whose equations do not
 * match the run return AMRGPU_EINVAL and leave the run unchanged. The choice applies to
 * every later substep (and, in 3D Euler, to the pressure of the flagging). The problem
 * named in setprob.data still sets the initial data and the default solver. */
int amrgpu_set_solver(amrgpu_ctx* ctx, const char* name, const double* params, int n);

/* Caps the context's device pools (patch storage and fill scratch, flux registers) at
 * `bytes` in all; 0 removes the cap. No counterpart in the reference, whose storage is one
 * growable array (igetsp.f calls resize_storage, src/2d/resize_alloc.f90, when it runs
 * out): a serving loop that admits solves by an HBM budget caps each at its share.
 * A later call that would grow a pool past the cap returns AMRGPU_ENOMEM and the solve
 * stops there (destroy the context). A cap below what the pools already hold returns
 * AMRGPU_EINVAL and changes nothing. */
int amrgpu_set_pool_limit(amrgpu_ctx* ctx, long long bytes);

/* Cross-request batching of the level step, for serving loops that run several solves
 * at once in one process (each on its own host thread). window_us > 0: each batched level
 * step of this (2D) context is handed to the process's step batcher, which launches the
 * steps that contexts of the same Riemann plugin and precision submit within window_us
 * microseconds as one kernel over all their tiles; window_us = 0: the context launches
 * its steps alone (the default). Results do not depend on the batching. No counterpart in
 * the reference (one solve per program). AMRGPU_EINVAL for a negative window or a 3D
 * context. Captured-graph replay and dimensionally split steps launch alone. */
int amrgpu_set_step_batching(amrgpu_ctx* ctx, int window_us);

/* 1: record CUDA events around every patch-step launch (kernel time is then
 * reported by amrgpu_info); 0: no per-launch events. */
int amrgpu_set_profile(amrgpu_ctx* ctx, int on);

/* The whole time integration: Berger-Oliger subcycling, regridding cadence,
 * output times. Replaces tick (src/2d/tick.f:4-391). max_cycles > 0 stops after
 * that many coarse steps; a later call continues from there. */
int amrgpu_run(amrgpu_ctx* ctx, int max_cycles);

/* One substep of every patch of `level`: ghost fill, coarse-value save for the
 * finer level, coarse/fine Riemann fix-up, patch step and flux registers.
 * Replaces advanc (src/2d/advanc.f:10-142) and par_advanc (advanc.f:170-291).
 * dtnew_out receives the level's suggested next dt (stepgrid.f:206-212). */
int amrgpu_level_advance(amrgpu_ctx* ctx, int level, double* dtnew_out, double* cfl_out);

/* amrgpu_level_advance without any device allocation. No counterpart in the
 * reference (its level advance allocates per call from the alloc heap).
 * 2D, FP64 contexts only: 3D and FP32 contexts return AMRGPU_EINVAL, and so does a
 * call made while another device than the context's is current.
 * The ghost-fill and saved-coarse-value programs stage their coarse scratch
 * rectangles in one file-scope device array of 4194304 doubles (32 MiB)
 * instead of the context's device pool; a level whose programs need more
 * returns AMRGPU_EINVAL with a message. The first call on a device looks up
 * the array's address (cudaGetSymbolAddress) with that device current; make
 * that first call before anything that must not see set-up work. The array is
 * shared by every context on the device and keeps the last call's contents:
 * nothing in it needs to start at zero (every scratch cell is written before
 * it is read), but calls that overlap in time, from any context, race on it.
 * Gauges are not sampled and no profiling events are recorded. */
int amrgpu_level_advance_noalloc(amrgpu_ctx* ctx, int level, double* dtnew_out, double* cfl_out);

/* Fine-to-coarse averaging and flux-register fix-up of `level` from level+1.
 * Replaces update (src/2d/update.f:16-189) and upbnd (src/2d/upbnd.f:18-127). */
int amrgpu_update(amrgpu_ctx* ctx, int level);

/* Regrid levels lbase+1 and finer. Replaces regrid (src/2d/regrid.f:4-122). */
int amrgpu_regrid(amrgpu_ctx* ctx, int lbase);

/* Write fort.qNNNN / fort.tNNNN into dir (ASCII form of src/2d/valout.f90:8-397). */
int amrgpu_valout(amrgpu_ctx* ctx, const char* dir);

/* Total of q(1)*dx*dy (3D: *dz) over level 1 (src/2d/conck.f:6-73, src/3d/conck.f). */
int amrgpu_mass(amrgpu_ctx* ctx, double* mass_out);

/* Run statistics: out[0..n) = time, cell updates, coarse steps, finest level,
 * stepping seconds, regrid seconds, initial mass, max Courant number, kernels
 * launched, peak pool bytes, level substeps, patch-step kernel milliseconds
 * (profiling on), cells of those launches, device milliseconds of the last
 * amrgpu_run call, cell updates of that call, 1 when tfinal was reached,
 * bytes of initial data copied host to device, then regrid seconds spent in:
 * device flagging, host flag processing, clustering, new-grid fill, register
 * and list set-up, device-program compilation, then the number of space dimensions,
 * the precision in bits (64 or 32), the CUDA graphs captured and replayed, and (3D)
 * the number of levels whose autotuned sweep schedule is the work queue, and the number
 * whose is per direction, then the bytes the device pools hold now (what
 * amrgpu_set_pool_limit counts). */
int amrgpu_info(amrgpu_ctx* ctx, double* out, int n);

/* Hierarchy rows in output order (valout.f90 loop order): (grid_number, level,
 * ilo, ihi, jlo, jhi) in 2D, (..., klo, khi) appended in 3D, i.e. 2 + 2*num_dim
 * ints per row; *n_out receives the row count. */
int amrgpu_grids(amrgpu_ctx* ctx, int* out, int cap, int* n_out);

/* Interior cell values of every grid in amrgpu_grids order, [m][j][i] per grid
 * in 2D and [m][k][j][i] in 3D (one [m][i] row per grid in 1D). *n_out receives
 * the number of values. out == NULL is a size query and gathers nothing; a buffer
 * with room for all of them (cap >= *n_out) receives them straight from the
 * device, a smaller one the first cap. */
int amrgpu_values(amrgpu_ctx* ctx, double* out, long long cap, long long* n_out);

/* Gauge samples as rows (gauge number, level, time, q1..qmeqn), grouped by gauge
 * (src/2d/gauges_module.f90:313-500). */
int amrgpu_gauges(amrgpu_ctx* ctx, double* out, int cap_rows, int* n_out);

/* 2 or 3: the dimension of the context's run (0 for a null context). No
 * counterpart in the reference, whose 2D and 3D programs are separate builds. */
int amrgpu_num_dim(amrgpu_ctx* ctx);

/* Release the context and its device memory. */
int amrgpu_destroy(amrgpu_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* AMRCLAW_B200_H */
