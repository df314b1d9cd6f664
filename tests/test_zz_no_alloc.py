"""amrgpu_level_advance_noalloc against amrgpu_level_advance (collected last).

The no-allocation entry point runs the same level substep with the ghost-fill
scratch in a fixed device array. Two substeps in a row through each entry
point, from the same initial hierarchy, must give the same cell values, the
same suggested dt and the same Courant number. Tolerance: exact equality (the
two paths do the same FP64 operations in the same order).
"""
import tempfile

import numpy as np
import pytest

import configs

pytestmark = pytest.mark.gpu


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


def test_noalloc_rejects_a_missing_level():
    from amrclaw_b200 import AmrError, Solver
    rd = configs.euler_quadrants(n=40, levels=3, tfinal=0.1)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            with pytest.raises(AmrError):
                s.level_advance_noalloc(7)
