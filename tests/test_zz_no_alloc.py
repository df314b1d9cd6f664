"""amrgpu_level_advance_noalloc against amrgpu_level_advance (collected last).

The no-allocation entry point runs the same level substep with the ghost-fill
scratch in a fixed device array. Two substeps in a row through each entry
point, from the same initial hierarchy, must give the same cell values, the
same suggested dt and the same Courant number. Tolerance: exact equality (the
two paths do the same FP64 operations in the same order). The substeps must
also leave the context's device pool and the device's free memory unchanged,
and a level whose scratch does not fit the fixed array must be refused.
"""
import tempfile

import numpy as np
import pytest

import configs

pytestmark = pytest.mark.gpu

EINVAL = 2


def _advance_twice(d, level, noalloc):
    from amrclaw_b200 import Solver
    with Solver(d) as s:
        step = s.level_advance_noalloc if noalloc else s.level_advance
        out = [step(level), step(level)]
        return s.grids(), s.values(), out


@pytest.mark.parametrize("level", [1, 2])
def test_noalloc_level_advance_matches_level_advance(level):
    rd = configs.euler_quadrants(n=40, levels=3, tfinal=0.1)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        g0, v0, o0 = _advance_twice(d, level, noalloc=False)
        g1, v1, o1 = _advance_twice(d, level, noalloc=True)
    np.testing.assert_array_equal(g1, g0)
    assert len(g0) > 1 and (g0[:, 1] == level).any()
    np.testing.assert_array_equal(v1, v0)
    assert o1 == o0


@pytest.mark.parametrize("level", [1, 2])
def test_noalloc_level_advance_with_aux_and_capacity(level):
    """The annulus: the step reads the patches' aux and the saved coarse rings' aux."""
    rd = configs.advection_annulus_regression()
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        g0, v0, o0 = _advance_twice(d, level, noalloc=False)
        g1, v1, o1 = _advance_twice(d, level, noalloc=True)
    np.testing.assert_array_equal(g1, g0)
    assert (g0[:, 1] == level).any()
    np.testing.assert_array_equal(v1, v0)
    assert o1 == o0


def test_noalloc_substeps_allocate_nothing():
    """After the first call (which looks up the array's address and may load the kernels),
    further substeps change neither the context's peak pool bytes nor the device's free memory."""
    import torch
    from amrclaw_b200 import Solver
    rd = configs.euler_quadrants(n=40, levels=3, tfinal=0.1)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            s.level_advance_noalloc(2)
            torch.cuda.synchronize()
            peak0 = s.info()["pool_peak_bytes"]
            free0 = torch.cuda.mem_get_info()[0]
            s.level_advance_noalloc(2)
            s.level_advance_noalloc(1)
            torch.cuda.synchronize()
            assert s.info()["pool_peak_bytes"] == peak0
            assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_a_missing_level():
    from amrclaw_b200 import AmrError, Solver
    rd = configs.euler_quadrants(n=40, levels=3, tfinal=0.1)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            with pytest.raises(AmrError) as e:
                s.level_advance_noalloc(7)
            assert e.value.code == EINVAL


def test_noalloc_rejects_scratch_beyond_the_fixed_array():
    """Level 2 covering the whole 1024^2 domain: level 1's saved-coarse-value program needs
    a coarse rectangle per fine grid, over 1024^2 cells x 4 equations in all, more than the
    fixed array holds; the substep is refused before any launch and the regular entry
    point still advances the level."""
    from amrclaw_b200 import AmrError, Solver
    rd = configs.euler_quadrants(n=1024, levels=2, tfinal=0.1)
    rd.amrdata.flag2refine_tol = -1.0  # every cell flagged: level 2 covers the domain
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            g = s.grids()
            fine = g[g[:, 1] == 2]
            assert ((fine[:, 3] - fine[:, 2] + 1) * (fine[:, 5] - fine[:, 4] + 1)).sum() == 2048 * 2048
            v0 = s.values()
            with pytest.raises(AmrError) as e:
                s.level_advance_noalloc(1)
            assert e.value.code == EINVAL and "exceeds the fixed array" in str(e.value)
            np.testing.assert_array_equal(s.values(), v0)
            dt, cfl = s.level_advance(1)
            assert cfl > 0
