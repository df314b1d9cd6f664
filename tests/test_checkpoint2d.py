"""Checkpoint and restart of the 2D path (check.f / restrt.f).

A run checkpointed after some coarse steps and continued from the checkpoint in a new
context (claw.data restart = T, restart_file) must give the same hierarchy, cell values,
gauge series, time and cell-update count as the run that was not interrupted.
"""
import os
import tempfile

import numpy as np
import pytest

import configs
from amrclaw_b200 import problems

pytestmark = pytest.mark.gpu


def _solve(rd, d, precision="fp64"):
    from amrclaw_b200 import Solver
    rd.write(d)
    with Solver(d, precision=precision) as s:
        s.run(0)
        return dict(grids=s.grids(), values=s.values(), gauges=s.gauges(rd.clawdata.num_eqn), info=s.info())


def _interrupted(rd, d, after, precision="fp64"):
    from amrclaw_b200 import Solver
    rd.write(d)
    with Solver(d, precision=precision) as s:
        s.run(after)
        s.checkpoint(os.path.join(d, "mid.chk"))
    rd.clawdata.restart = True
    rd.clawdata.restart_file = "mid.chk"
    try:
        return _solve(rd, d, precision)
    finally:
        rd.clawdata.restart = False


def _assert_same(a, b):
    np.testing.assert_array_equal(a["grids"], b["grids"])
    np.testing.assert_array_equal(a["values"], b["values"])
    np.testing.assert_array_equal(a["gauges"], b["gauges"])
    assert a["info"]["time"] == b["info"]["time"]
    assert a["info"]["cell_updates"] == b["info"]["cell_updates"]
    assert a["info"]["coarse_steps"] == b["info"]["coarse_steps"]


def _quadrants():
    rd = problems.euler_quadrants(48, levels=3, ratio=2, tfinal=0.2)
    rd.gaugedata.gauges = [[1, 0.3, 0.4, 0.0, 1e9], [2, 0.75, 0.8, 0.0, 1e9]]
    return rd


@pytest.mark.parametrize("after", [1, 6])
def test_quadrants_restart_is_identical(after):
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        full = _solve(_quadrants(), d1)
        cont = _interrupted(_quadrants(), d2, after)
    _assert_same(full, cont)


def test_fp32_acoustics_restart_is_identical():
    mk = lambda: problems.acoustics_pulse(48, levels=3, ratio=2, tfinal=0.2)
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        full = _solve(mk(), d1, "fp32")
        cont = _interrupted(mk(), d2, 4, "fp32")
    _assert_same(full, cont)


def test_periodic_advection_restart_is_identical():
    mk = lambda: configs.advection_square_bench(n=32, tfinal=0.3, levels=3)
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        full = _solve(mk(), d1)
        cont = _interrupted(mk(), d2, 5)
    _assert_same(full, cont)


def test_annulus_restart_is_identical():
    """aux arrays (face velocities, capacity) are set again by setaux on the restored grids."""
    mk = configs.advection_annulus_regression
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        full = _solve(mk(), d1)
        cont = _interrupted(mk(), d2, 7)
    _assert_same(full, cont)


def test_checkpoint_cadence_and_final_checkpoint():
    from amrclaw_b200 import Solver
    rd = problems.advection_square(32, levels=2, tfinal=0.1)
    rd.clawdata.checkpt_style = 3
    rd.clawdata.checkpt_interval = 3
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d, outdir=d) as s:
            s.run(0)
            nsteps = int(s.info()["coarse_steps"])
            v_end = s.values()
        names = {f for f in os.listdir(d) if f.startswith("fort.chk")}
        assert names == {"fort.chk%05d" % k for k in range(3, nsteps + 1, 3)} | {"fort.chk%05d" % nsteps}, (names, nsteps)
        rd.clawdata.checkpt_style = 0
        rd.clawdata.restart = True
        rd.clawdata.restart_file = "fort.chk%05d" % nsteps
        rd.write(d)
        with Solver(d) as s:
            np.testing.assert_array_equal(s.values(), v_end)
