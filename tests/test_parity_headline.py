"""GPU path versus the CPU oracle at the full size of the benchmark configurations.

The smaller parity tests cannot reach hierarchies that only appear at full size: a
single flag that flips (a `dq > tol` comparison one ulp apart) changes every later grid.
These tests run the FP64 device path and the oracle on the benchmark workloads
themselves and require the same hierarchy (boxes, grid numbers, order), bit-identical
cell values, the same time and cell-update count, and level-1 mass within 1e-13:

- 3D Euler blast: 64^3, 3 levels, ratio 2, max1d 68, the first 12 coarse steps (six
  regrids of levels 2-3);
- 2D Euler quadrants: 100^2, 4 levels, ratio 2, the whole run to t = 0.8;
- 2D constant advection of the square: 50^2, 3 levels, periodic, the whole run to t = 2.0;
- 3D advection in the time-modulated swirl field (FP64): 32^3, 4 levels, the whole
  period to t = 1.5.
"""
import os
import tempfile

import numpy as np
import pytest

import configs
from amrclaw_b200 import problems
from oracle.pyoracle import Oracle2D, Oracle3D

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8


def _compare(rd, ndim, cycles=0):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            assert s.num_dim == ndim
            s.run(cycles)
            gpu = dict(grids=s.grids(), values=s.values(), info=s.info(), mass=s.mass())
        o = (Oracle3D if ndim == 3 else Oracle2D)(d, threads=THREADS)
        o.run(cycles)
        ref = dict(grids=o.grids(), values=o.values(), time=o.time(), mass=o.mass(), cells=o.cell_updates())
        o.close()
    np.testing.assert_array_equal(gpu["grids"], ref["grids"])
    assert gpu["values"].shape == ref["values"].shape
    diff = np.nonzero(gpu["values"] != ref["values"])[0]
    assert diff.size == 0, "values differ at %d of %d cells, first %s: gpu %r oracle %r" % (
        diff.size, gpu["values"].size, diff[:3], gpu["values"][diff[:3]], ref["values"][diff[:3]])
    assert gpu["info"]["time"] == ref["time"]
    assert gpu["info"]["cell_updates"] == ref["cells"]
    np.testing.assert_allclose(gpu["mass"], ref["mass"], rtol=1e-13)
    return gpu, ref


def test_euler3d_blast_full_size_twelve_coarse_steps():
    rd = configs.euler_blast(n=64, levels=3, tfinal=0.5, seed=0, max1d=68)
    gpu, ref = _compare(rd, 3, cycles=12)
    assert gpu["info"]["coarse_steps"] == 12
    levels = ref["grids"][:, 1]
    assert (levels == 2).any() and (levels == 3).sum() > 1


def test_euler2d_quadrants_full_size_whole_run():
    rd = configs.euler_quadrants(n=100, levels=4, tfinal=0.8)
    gpu, ref = _compare(rd, 2)
    assert gpu["info"]["finished"] and (ref["grids"][:, 1] == 4).any()


def test_advection2d_square_full_size_whole_run():
    rd = configs.advection_square_bench(n=50, tfinal=2.0, levels=3)
    gpu, ref = _compare(rd, 2)
    assert gpu["info"]["finished"] and (ref["grids"][:, 1] == 3).any()


def test_swirl3d_fp64_full_size_whole_period():
    rd = problems.advection_swirl3d(n=32, levels=4, tfinal=1.5)
    gpu, ref = _compare(rd, 3)
    assert gpu["info"]["finished"] and (ref["grids"][:, 1] == 4).any()
