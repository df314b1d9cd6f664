"""ctypes wrapper of the CPU oracle (test infrastructure only; see oracle/amr2d.cpp, oracle/amr3d.cpp)."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".cpp", ".hpp"))]
    if force or not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        lib.oracle2d_create.restype = vp
        lib.oracle2d_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        lib.oracle2d_destroy.argtypes = [vp]
        lib.oracle2d_run.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        for n in ("oracle2d_time", "oracle2d_cell_updates", "oracle2d_mass", "oracle2d_mass0"):
            getattr(lib, n).restype = ctypes.c_double
            getattr(lib, n).argtypes = [vp]
        for n in ("oracle2d_lfine", "oracle2d_ncycle"):
            getattr(lib, n).argtypes = [vp]
        lib.oracle2d_grids.argtypes = [vp, vp, ctypes.c_int]
        lib.oracle2d_values.restype = ctypes.c_long
        lib.oracle2d_values.argtypes = [vp, vp, ctypes.c_long]
        lib.oracle2d_gauges.argtypes = [vp, vp, ctypes.c_int]
        lib.oracle3d_create.restype = vp
        lib.oracle3d_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int]
        lib.oracle3d_destroy.argtypes = [vp]
        lib.oracle3d_run.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        for n in ("oracle3d_time", "oracle3d_cell_updates", "oracle3d_mass", "oracle3d_mass0"):
            getattr(lib, n).restype = ctypes.c_double
            getattr(lib, n).argtypes = [vp]
        for n in ("oracle3d_lfine", "oracle3d_ncycle"):
            getattr(lib, n).argtypes = [vp]
        lib.oracle3d_grids.argtypes = [vp, vp, ctypes.c_int]
        lib.oracle3d_values.restype = ctypes.c_long
        lib.oracle3d_values.argtypes = [vp, vp, ctypes.c_long]
        lib.oracle3d_gauges.argtypes = [vp, vp, ctypes.c_int]
        lib.oracle1d_create.restype = vp
        lib.oracle1d_create.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        lib.oracle1d_destroy.argtypes = [vp]
        lib.oracle1d_run.argtypes = [vp, ctypes.c_int]
        for n in ("oracle1d_time", "oracle1d_cell_updates", "oracle1d_mass"):
            getattr(lib, n).restype = ctypes.c_double
            getattr(lib, n).argtypes = [vp]
        lib.oracle1d_grids.argtypes = [vp, vp, ctypes.c_int]
        lib.oracle1d_values.restype = ctypes.c_long
        lib.oracle1d_values.argtypes = [vp, vp, ctypes.c_long]
        lib.oracle1d_gauges.argtypes = [vp, vp, ctypes.c_int]
        _lib = lib
    return _lib


class Oracle2D:
    def __init__(self, rundir: str, outdir: str | None = None, write_output: bool = False, threads: int = 1):
        self.lib = load()
        self.h = self.lib.oracle2d_create(rundir.encode(), (outdir or rundir).encode(), int(write_output), threads)
        if not self.h:
            raise RuntimeError("oracle2d_create failed for %s" % rundir)

    def run(self, max_cycles: int = 0) -> float:
        sec = ctypes.c_double()
        if self.lib.oracle2d_run(self.h, max_cycles, ctypes.byref(sec)) != 0:
            raise RuntimeError("oracle run failed")
        return sec.value

    def time(self) -> float:
        return self.lib.oracle2d_time(self.h)

    def cell_updates(self) -> float:
        return self.lib.oracle2d_cell_updates(self.h)

    def mass(self) -> float:
        return self.lib.oracle2d_mass(self.h)

    def grids(self) -> np.ndarray:
        n = self.lib.oracle2d_grids(self.h, None, 0)
        a = np.zeros((n, 6), dtype=np.int32)
        self.lib.oracle2d_grids(self.h, a.ctypes.data, n)
        return a

    def values(self) -> np.ndarray:
        n = self.lib.oracle2d_values(self.h, None, 0)
        a = np.zeros(n, dtype=np.float64)
        self.lib.oracle2d_values(self.h, a.ctypes.data, n)
        return a

    def gauges(self, nvar: int) -> np.ndarray:
        n = self.lib.oracle2d_gauges(self.h, None, 0)
        a = np.zeros((n, 3 + nvar), dtype=np.float64)
        self.lib.oracle2d_gauges(self.h, a.ctypes.data, n)
        return a

    def close(self) -> None:
        if self.h:
            self.lib.oracle2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Oracle3D(Oracle2D):
    """The 3D restatement (oracle/amr3d.cpp) behind the same interface; grid rows have 8 columns."""

    def __init__(self, rundir: str, outdir: str | None = None, write_output: bool = False, threads: int = 1):
        self.lib = load()
        self.h = self.lib.oracle3d_create(rundir.encode(), (outdir or rundir).encode(), int(write_output), threads)
        if not self.h:
            raise RuntimeError("oracle3d_create failed for %s" % rundir)

    def run(self, max_cycles: int = 0) -> float:
        sec = ctypes.c_double()
        if self.lib.oracle3d_run(self.h, max_cycles, ctypes.byref(sec)) != 0:
            raise RuntimeError("oracle run failed")
        return sec.value

    def time(self) -> float:
        return self.lib.oracle3d_time(self.h)

    def cell_updates(self) -> float:
        return self.lib.oracle3d_cell_updates(self.h)

    def mass(self) -> float:
        return self.lib.oracle3d_mass(self.h)

    def grids(self) -> np.ndarray:
        n = self.lib.oracle3d_grids(self.h, None, 0)
        a = np.zeros((n, 8), dtype=np.int32)
        self.lib.oracle3d_grids(self.h, a.ctypes.data, n)
        return a

    def values(self) -> np.ndarray:
        n = self.lib.oracle3d_values(self.h, None, 0)
        a = np.zeros(n, dtype=np.float64)
        self.lib.oracle3d_values(self.h, a.ctypes.data, n)
        return a

    def gauges(self, nvar: int) -> np.ndarray:
        n = self.lib.oracle3d_gauges(self.h, None, 0)
        a = np.zeros((n, 3 + nvar), dtype=np.float64)
        self.lib.oracle3d_gauges(self.h, a.ctypes.data, n)
        return a

    def close(self) -> None:
        if self.h:
            self.lib.oracle3d_destroy(self.h)
            self.h = None


class Oracle1D:
    """The 1D restatement (oracle/amr1d.cpp)."""

    def __init__(self, rundir: str, outdir: str | None = None, write_output: bool = False):
        self.lib = load()
        self.h = self.lib.oracle1d_create(rundir.encode(), (outdir or rundir).encode(), int(write_output))
        if not self.h:
            raise RuntimeError("oracle1d_create failed for %s" % rundir)
        self.nvar = None

    def run(self, max_cycles: int = 0) -> None:
        if self.lib.oracle1d_run(self.h, max_cycles) != 0:
            raise RuntimeError("oracle run failed")

    def time(self) -> float:
        return self.lib.oracle1d_time(self.h)

    def cell_updates(self) -> float:
        return self.lib.oracle1d_cell_updates(self.h)

    def mass(self) -> float:
        return self.lib.oracle1d_mass(self.h)

    def grids(self) -> np.ndarray:
        n = self.lib.oracle1d_grids(self.h, None, 0)
        a = np.zeros((n, 4), dtype=np.int32)
        self.lib.oracle1d_grids(self.h, a.ctypes.data, n)
        return a

    def values(self) -> np.ndarray:
        n = self.lib.oracle1d_values(self.h, None, 0)
        a = np.zeros(n, dtype=np.float64)
        self.lib.oracle1d_values(self.h, a.ctypes.data, n)
        return a

    def gauges(self, nvar: int) -> np.ndarray:
        n = self.lib.oracle1d_gauges(self.h, None, 0)
        a = np.zeros((n, 3 + nvar), dtype=np.float64)
        self.lib.oracle1d_gauges(self.h, a.ctypes.data, n)
        return a

    def close(self) -> None:
        if self.h:
            self.lib.oracle1d_destroy(self.h)
            self.h = None
