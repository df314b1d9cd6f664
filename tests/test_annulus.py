"""Aux arrays and a capacity function in 2D: the reference's tests/advection_2d_annulus.

Advection on the mapped annulus 0.2 <= r <= 1 (computational (r, theta), periodic in
theta) with aux(1) = u on the left face, aux(2) = v on the bottom face and aux(3) = kappa,
the capacity (capa_index 3). The capacity enters the step (dtdx1d = dt/(dx kappa),
stepgrid.f's update divides by kappa), filval (fixcapaq.f), upbnd, update and conck; the
face velocities enter rpn2/rpt2 and qad.f's coarse/fine Riemann problems. The oracle is
pinned to the reference's regression gauges (test_oracle2d.py); here the device path is
held bit-identical to the oracle and to those gauges.
"""
import tempfile

import numpy as np
import pytest

import configs
from golden_io import assert_gauges_match, gauge_rows
from oracle.pyoracle import Oracle2D


def _oracle(rd, cycles=0):
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle2D(d, threads=4)
        o.run(cycles)
        out = dict(grids=o.grids(), values=o.values(), gauges=o.gauges(1), time=o.time(), mass=o.mass(),
                   cells=o.cell_updates())
        o.close()
    return out


def _device(rd, cycles=0, **kw):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d, **kw) as s:
            s.run(cycles)
            return dict(grids=s.grids(), values=s.values(), gauges=s.gauges(1), time=s.info()["time"],
                        cells=s.info()["cell_updates"], mass=s.mass(), info=s.info())


def _same(gpu, ref):
    np.testing.assert_array_equal(gpu["grids"], ref["grids"])
    diff = np.nonzero(gpu["values"] != ref["values"])[0]
    assert diff.size == 0, "values differ at %d cells, first %s: gpu %r oracle %r" % (
        diff.size, diff[:3], gpu["values"][diff[:3]], ref["values"][diff[:3]])
    assert gpu["time"] == ref["time"] and gpu["cells"] == ref["cells"]
    # the two Gaussians have opposite signs: the total (about 1e-5) is a cancellation of
    # terms near 1e-1, summed in another order on the device, so the bound is absolute
    np.testing.assert_allclose(gpu["mass"], ref["mass"], rtol=0, atol=1e-15)


# ------------------------------------------------------------------------- CPU
def test_single_level_conserves_kappa_q():
    """conck.f with a capacity sums q kappa dx dy. On one level the flow is along theta
    (periodic) and the radial face velocities vanish to rounding, so that total is kept."""
    rd = configs.advection_annulus_regression()
    rd.amrdata.amr_levels_max = 1
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle2D(d)
        m0 = o.mass()
        o.run(0)
        m1 = o.mass()
        o.close()
    assert abs(m1 - m0) <= 1e-13


def test_aux_needs_a_problem_with_setaux():
    rd = configs.advection_square_regression()
    rd.clawdata.num_aux = 1
    rd.amrdata.aux_type = ["center"]
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with pytest.raises(RuntimeError):
            Oracle2D(d)


# ------------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_device_annulus_matches_oracle_and_reference_gauges():
    rd = configs.advection_annulus_regression()
    ref = _oracle(rd)
    gpu = _device(rd)
    _same(gpu, ref)
    np.testing.assert_array_equal(gpu["gauges"], ref["gauges"])
    assert_gauges_match(gpu["gauges"], gauge_rows("advection_2d_annulus"))
    assert (gpu["grids"][:, 1] == 3).any()


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(batched=False), dict(graphs=True)], ids=["plain", "graphs"])
def test_device_annulus_other_schedules_match_oracle(kw):
    rd = configs.advection_annulus_regression()
    _same(_device(rd, **kw), _oracle(rd))


@pytest.mark.gpu
def test_device_annulus_finer_run_matches_oracle():
    # more regrids and more coarse/fine boundaries than the regression case
    rd = configs.advection_annulus_regression()
    rd.clawdata.num_cells = [40, 240]
    rd.clawdata.tfinal = 0.3
    rd.amrdata.flag2refine_tol = 0.01
    _same(_device(rd), _oracle(rd))


@pytest.mark.gpu
def test_device_annulus_dimensional_split_matches_oracle():
    rd = configs.advection_annulus_regression()
    rd.clawdata.dimensional_split = "godunov"
    _same(_device(rd), _oracle(rd))


@pytest.mark.gpu
def test_device_vc_advection_plugin():
    from amrclaw_b200 import AmrError, Solver
    rd = configs.advection_annulus_regression()
    ref = _oracle(rd)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            s.set_solver("vc_advection", [])
            with pytest.raises(AmrError) as e:
                s.set_solver("advection", [0.5, 1.0])  # a different equation set than the run's
            assert e.value.code == 2
            s.run(0)
            got = dict(grids=s.grids(), values=s.values(), time=s.info()["time"], cells=s.info()["cell_updates"],
                       mass=s.mass())
    _same(got, ref)
