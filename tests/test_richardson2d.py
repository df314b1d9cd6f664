"""Richardson error estimation (errest.f, errf1.f, coarsen.f, prepbigstep.f, prepregstep.f)
as a flagging option of the 2D path.

The device path runs the big step (2*dt on the old values coarsened by 2, ghost ring of
twice the width filled at the previous time) and the regular step as virtual patches of
the level step kernel, and merges errf1's flags on the host. FP64 results must equal the
oracle's bit for bit: hierarchy, values, time and cell-update count. The reference's own
tests do not run this option, so the oracle's restatement is checked here by properties
(an unreachable tolerance changes nothing, a small one refines more).
"""
import tempfile

import numpy as np
import pytest

import configs
from oracle.pyoracle import Oracle2D


def _rich(rd, tol, gradient=True):
    rd.amrdata.flag_richardson = True
    rd.amrdata.flag_richardson_tol = tol
    rd.amrdata.flag2refine = gradient
    return rd


def _oracle(rd):
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle2D(d)
        o.run(0)
        out = dict(grids=o.grids(), values=o.values(), time=o.time(), cells=o.cell_updates())
        o.close()
    return out


def _gpu(rd, **kw):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d, **kw) as s:
            s.run(0)
            return dict(grids=s.grids(), values=s.values(), info=s.info())


def _assert_identical(ref, gpu):
    np.testing.assert_array_equal(gpu["grids"], ref["grids"])
    assert gpu["values"].shape == ref["values"].shape
    diff = np.nonzero(gpu["values"] != ref["values"])[0]
    assert diff.size == 0, "values differ at %d cells" % diff.size
    assert gpu["info"]["time"] == ref["time"]
    assert gpu["info"]["cell_updates"] == ref["cells"]


# ---------------------------------------------------------------- oracle properties (CPU)

def test_oracle_unreachable_tolerance_changes_nothing():
    base = _oracle(configs.euler_quadrants(n=32, levels=3, tfinal=0.15))
    rich = _oracle(_rich(configs.euler_quadrants(n=32, levels=3, tfinal=0.15), 1e30))
    np.testing.assert_array_equal(rich["grids"], base["grids"])
    np.testing.assert_array_equal(rich["values"], base["values"])


def test_oracle_small_tolerance_refines_more():
    grad = _oracle(configs.euler_quadrants(n=32, levels=3, tfinal=0.15))
    rich = _oracle(_rich(configs.euler_quadrants(n=32, levels=3, tfinal=0.15), 1e-5))
    only = _oracle(_rich(configs.euler_quadrants(n=32, levels=3, tfinal=0.15), 1e-5, gradient=False))
    assert rich["cells"] > grad["cells"]
    assert only["cells"] > _oracle(_rich(configs.euler_quadrants(n=32, levels=3, tfinal=0.15), 1e30, gradient=False))["cells"]


# ---------------------------------------------------------------- device vs oracle (GPU)

@pytest.mark.gpu
@pytest.mark.parametrize("batched", [True, False])
def test_euler_richardson_and_gradient_matches_oracle(batched):
    # regrid_buffer_width 2: errf1's flags sit one cell off the blocks they test
    mk = lambda: _rich(configs.euler_quadrants(n=40, levels=3, tfinal=0.25), 1e-3)
    _assert_identical(_oracle(mk()), _gpu(mk(), batched=batched))


@pytest.mark.gpu
def test_euler_richardson_only_matches_oracle():
    mk = lambda: _rich(configs.euler_quadrants(n=40, levels=3, tfinal=0.25), 1e-5, gradient=False)
    ref = _oracle(mk())
    assert len(ref["grids"]) > 1
    _assert_identical(ref, _gpu(mk()))


@pytest.mark.gpu
def test_periodic_advection_richardson_matches_oracle():
    # periodic domain (prefilrecur.f with twice the ghost width) and regrid_buffer_width 3
    mk = lambda: _rich(configs.advection_square_regression(), 1e-4)
    ref = _oracle(mk())
    assert len(ref["grids"]) > 1
    _assert_identical(ref, _gpu(mk()))


@pytest.mark.gpu
def test_acoustics_richardson_four_levels_matches_oracle():
    from amrclaw_b200 import problems
    mk = lambda: _rich(problems.acoustics_pulse(48, levels=4, ratio=2, tfinal=0.3), 1e-4)
    _assert_identical(_oracle(mk()), _gpu(mk()))


@pytest.mark.gpu
def test_fp32_richardson_runs_and_refines():
    mk = lambda: _rich(configs.euler_quadrants(n=40, levels=3, tfinal=0.25), 1e-5, gradient=False)
    g32 = _gpu(mk(), precision="fp32")
    assert len(g32["grids"]) > 1
    assert np.isfinite(g32["values"]).all()
