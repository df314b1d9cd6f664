"""Checkpoint and restart of the 3D path (check.f / restrt.f).

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


def _solve(rd, d, precision="fp64", steps=0):
    from amrclaw_b200 import Solver
    rd.write(d)
    with Solver(d, precision=precision) as s:
        s.run(steps)
        return dict(grids=s.grids(), values=s.values(), gauges=s.gauges(rd.clawdata.num_eqn), info=s.info())


def _interrupted(rd, d, after, precision="fp64"):
    from amrclaw_b200 import Solver
    rd.write(d)
    chk = os.path.join(d, "mid.chk")
    with Solver(d, precision=precision) as s:
        s.run(after)
        s.checkpoint(chk)
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


def _blast():
    rd = configs.euler_blast(n=16, levels=3, tfinal=0.3, max1d=16)
    rd.gaugedata.gauges = [[1, 0.05, -0.02, 0.03, 0.0, 1e9], [2, 0.31, 0.12, -0.27, 0.0, 1e9]]
    return rd


@pytest.mark.parametrize("after", [1, 5])
def test_blast_restart_is_identical(after):
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        full = _solve(_blast(), d1)
        cont = _interrupted(_blast(), d2, after)
    _assert_same(full, cont)


def test_modulated_swirl_restart_is_identical():
    """The aux block (scaled by the last b4step3) is part of the checkpoint."""
    mk = lambda: problems.advection_swirl3d(n=16, levels=3, tfinal=0.3, max1d=16)
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        full = _solve(mk(), d1)
        cont = _interrupted(mk(), d2, 4)
    _assert_same(full, cont)


def test_fp32_restart_is_identical():
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        full = _solve(_blast(), d1, "fp32")
        cont = _interrupted(_blast(), d2, 3, "fp32")
    _assert_same(full, cont)


def test_checkpoint_cadence_and_final_checkpoint():
    """checkpt_style 3 writes fort.chkNNNNN every checkpt_interval coarse steps, and one
    at the end; the last one restarts into the finished state."""
    from amrclaw_b200 import Solver
    rd = configs.euler_blast(n=16, levels=2, tfinal=0.1, max1d=16)
    rd.clawdata.checkpt_style = 3
    rd.clawdata.checkpt_interval = 2
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d, outdir=d) as s:
            s.run(0)
            nsteps = int(s.info()["coarse_steps"])
            t_end, v_end = s.info()["time"], s.values()
        names = sorted(f for f in os.listdir(d) if f.startswith("fort.chk"))
        want = {"fort.chk%05d" % k for k in range(2, nsteps + 1, 2)} | {"fort.chk%05d" % nsteps}
        assert set(names) == want, (names, nsteps)
        rd.clawdata.checkpt_style = 0
        rd.clawdata.restart = True
        rd.clawdata.restart_file = "fort.chk%05d" % nsteps
        rd.write(d)
        with Solver(d) as s:
            assert s.info()["time"] == t_end
            np.testing.assert_array_equal(s.values(), v_end)
            s.run(0)
            assert s.info()["coarse_steps"] == nsteps
