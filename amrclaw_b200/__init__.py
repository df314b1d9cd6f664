"""amrclaw_b200: B200-native patch-advance path of AMRClaw.

Python side of the drop-in boundary: ``ClawRunData`` mirrors the reference's
``setrun.py`` objects and writes the same data files; ``Solver`` drives the CUDA
library through its C ABI (``include/amrclaw_b200.h``). There is no CPU
fallback: without the built library on a CUDA device the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

from .data import ClawRunData  # noqa: F401
from . import _lib

__all__ = ["ClawRunData", "Solver", "AmrError"]


class AmrError(RuntimeError):
    """A failed C-ABI call; ``code`` is its status (1 AMRGPU_ERROR, 2 AMRGPU_EINVAL,
    3 AMRGPU_ENOMEM: a capped device pool would have grown past its cap)."""

    def __init__(self, msg: str, code: int = 1):
        super().__init__(msg)
        self.code = code


def _check(lib, rc: int, what: str) -> None:
    if rc != 0:
        msg = lib.amrgpu_last_error()
        raise AmrError("%s failed: %s" % (what, msg.decode() if msg else "error %d" % rc), rc)


class Solver:
    """One AMR run on the GPU (the reference's ``amr2`` program from init to tfinal)."""

    def __init__(self, rundata_or_dir, outdir: str | None = None, write_output: bool = False, batched: bool = True,
                 precision: str = "fp64", graphs: bool = False, schedule: int | None = None,
                 pool_limit: int = 0, step_batching_us: int = 0):
        self._lib = _lib.load()
        if isinstance(rundata_or_dir, ClawRunData):
            self._tmp = tempfile.TemporaryDirectory(prefix="amrgpu_")
            rundir = rundata_or_dir.write(self._tmp.name)
        else:
            self._tmp = None
            rundir = str(rundata_or_dir)
        self.rundir = rundir
        self.outdir = outdir or rundir
        if write_output:
            os.makedirs(self.outdir, exist_ok=True)
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        h = ctypes.c_void_p()
        _check(self._lib, self._lib.amrgpu_init_precision(rundir.encode(), self.outdir.encode(), int(write_output),
                                                          64 if precision == "fp64" else 32, ctypes.byref(h)),
               "amrgpu_init")
        self._h = h
        self.set_batched(batched)
        if schedule is not None:
            self.set_schedule(schedule)
        if graphs:
            self.set_graphs(True)
        if pool_limit:
            self.set_pool_limit(pool_limit)
        if step_batching_us:
            self.set_step_batching(step_batching_us)

    def set_batched(self, batched: bool) -> None:
        _check(self._lib, self._lib.amrgpu_set_batched(self._h, int(batched)), "amrgpu_set_batched")

    def set_graphs(self, on: bool) -> None:
        """Replay each level substep from captured CUDA graphs (3D path)."""
        _check(self._lib, self._lib.amrgpu_set_graphs(self._h, int(on)), "amrgpu_set_graphs")

    def checkpoint(self, path: str | None = None) -> None:
        """Write a checkpoint of the run at its current coarse-step boundary (3D); a run
        whose claw.data sets restart / restart_file continues from it."""
        _check(self._lib, self._lib.amrgpu_checkpoint(self._h, path.encode() if path else None), "amrgpu_checkpoint")

    def set_schedule(self, schedule: int) -> None:
        """Sweep schedule of the batched 3D path: 1 per direction (the default), 2 work queue,
        0 autotune per level. 2D runs accept only 0 (they have a single schedule)."""
        _check(self._lib, self._lib.amrgpu_set_schedule(self._h, int(schedule)), "amrgpu_set_schedule")

    def set_solver(self, name: str, params=()) -> None:
        """The Riemann solver plugin by name, with its problem constants (amrgpu_set_solver)."""
        vals = (ctypes.c_double * max(1, len(params)))(*[float(x) for x in params])
        _check(self._lib, self._lib.amrgpu_set_solver(self._h, name.encode(), vals, len(params)), "amrgpu_set_solver")

    def set_pool_limit(self, nbytes: int) -> None:
        """Cap the context's device pools at nbytes (0: no cap); growth past it raises
        AmrError with code 3 (amrgpu_set_pool_limit)."""
        _check(self._lib, self._lib.amrgpu_set_pool_limit(self._h, int(nbytes)), "amrgpu_set_pool_limit")

    def set_step_batching(self, window_us: int) -> None:
        """Launch this (2D) solve's level steps together with those of other solves of the same
        plugin and precision running at the same time in this process, waiting at most
        window_us microseconds for them (amrgpu_set_step_batching); 0 launches them alone."""
        _check(self._lib, self._lib.amrgpu_set_step_batching(self._h, int(window_us)), "amrgpu_set_step_batching")

    def set_profile(self, on: bool) -> None:
        _check(self._lib, self._lib.amrgpu_set_profile(self._h, int(on)), "amrgpu_set_profile")

    def run(self, max_cycles: int = 0) -> None:
        _check(self._lib, self._lib.amrgpu_run(self._h, int(max_cycles)), "amrgpu_run")

    def level_advance(self, level: int):
        dt = ctypes.c_double(); cfl = ctypes.c_double()
        _check(self._lib, self._lib.amrgpu_level_advance(self._h, level, ctypes.byref(dt), ctypes.byref(cfl)),
               "amrgpu_level_advance")
        return dt.value, cfl.value

    def level_advance_noalloc(self, level: int):
        """amrgpu_level_advance with the ghost-fill scratch in a fixed device array (no allocation)."""
        dt = ctypes.c_double(); cfl = ctypes.c_double()
        _check(self._lib, self._lib.amrgpu_level_advance_noalloc(self._h, level, ctypes.byref(dt), ctypes.byref(cfl)),
               "amrgpu_level_advance_noalloc")
        return dt.value, cfl.value

    def update(self, level: int) -> None:
        _check(self._lib, self._lib.amrgpu_update(self._h, level), "amrgpu_update")

    def regrid(self, lbase: int) -> None:
        _check(self._lib, self._lib.amrgpu_regrid(self._h, lbase), "amrgpu_regrid")

    def valout(self, outdir: str) -> None:
        os.makedirs(outdir, exist_ok=True)
        _check(self._lib, self._lib.amrgpu_valout(self._h, outdir.encode()), "amrgpu_valout")

    def mass(self) -> float:
        m = ctypes.c_double()
        _check(self._lib, self._lib.amrgpu_mass(self._h, ctypes.byref(m)), "amrgpu_mass")
        return m.value

    def info(self) -> dict:
        keys = ["time", "cell_updates", "coarse_steps", "lfine", "step_seconds", "regrid_seconds", "mass0",
                "cflmax", "kernels", "pool_peak_bytes", "substeps", "step_kernel_ms", "step_kernel_cells",
                "last_run_ms", "last_run_cells", "finished", "h2d_bytes",
                "regrid_flags_s", "regrid_hostflags_s", "regrid_cluster_s", "regrid_fill_s", "regrid_prep_s", "regrid_compile_s",
                "num_dim", "precision_bits", "graph_captures", "graph_replays", "levels_tuned_queue",
                "levels_tuned_per_direction", "pool_bytes", "step_batch_submits", "step_batch_shared",
                "step_batch_members"]
        out = (ctypes.c_double * len(keys))()
        _check(self._lib, self._lib.amrgpu_info(self._h, out, len(keys)), "amrgpu_info")
        return dict(zip(keys, list(out)))

    @property
    def num_dim(self) -> int:
        """2 or 3: the dimension of the run's data files."""
        d = self._lib.amrgpu_num_dim(self._h)
        if d < 0:
            _check(self._lib, d, "amrgpu_num_dim")
        return d

    def grids(self) -> np.ndarray:
        """Rows (grid_number, level, ilo, ihi, jlo, jhi[, klo, khi]) in output order."""
        n = ctypes.c_int()
        _check(self._lib, self._lib.amrgpu_grids(self._h, None, 0, ctypes.byref(n)), "amrgpu_grids")
        a = np.zeros((n.value, 2 + 2 * self.num_dim), dtype=np.int32)
        _check(self._lib, self._lib.amrgpu_grids(self._h, a.ctypes.data_as(_lib.c_int_p), n.value, ctypes.byref(n)),
               "amrgpu_grids")
        return a

    def values(self) -> np.ndarray:
        n = ctypes.c_longlong()
        _check(self._lib, self._lib.amrgpu_values(self._h, None, 0, ctypes.byref(n)), "amrgpu_values")
        a = np.empty(n.value, dtype=np.float64)
        _check(self._lib, self._lib.amrgpu_values(self._h, a.ctypes.data_as(_lib.c_double_p), n.value, ctypes.byref(n)),
               "amrgpu_values")
        return a

    def gauges(self, nvar: int) -> np.ndarray:
        n = ctypes.c_int()
        _check(self._lib, self._lib.amrgpu_gauges(self._h, None, 0, ctypes.byref(n)), "amrgpu_gauges")
        a = np.zeros((n.value, 3 + nvar), dtype=np.float64)
        _check(self._lib, self._lib.amrgpu_gauges(self._h, a.ctypes.data_as(_lib.c_double_p), n.value, ctypes.byref(n)),
               "amrgpu_gauges")
        return a

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.amrgpu_destroy(self._h)
            self._h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
