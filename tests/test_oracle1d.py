"""The 1D CPU oracle against the reference's 1D regression data (no GPU needed).

tests/acoustics_1d_homogeneous (40 cells, 3 levels, extrapolation, van Leer) and
tests/advection_1d_example1 (40 cells, 3 levels, periodic, MC) of the reference: their
gauges (printed e15.7) are reproduced to 7 digits, row for row.

tests/euler_1d_wcblast cannot pin anything: its flag2refine1.f90 takes two arguments
(DONTFLAG, DOFLAG) that the current src/1d/flagger.f does not pass, so the reference's own
build of that test reads undefined memory, and its regression data (2017) refines at t = 0
where the density, the only flagged quantity, is uniform. The oracle runs it as its source
states it (density differences), checked here by properties.
"""
import tempfile

import numpy as np

import configs
from golden_io import assert_gauges_match, gauge_rows
from oracle.pyoracle import Oracle1D


def _run(rd, nvar):
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle1D(d)
        m0 = o.mass()
        o.run(0)
        out = dict(gauges=o.gauges(nvar), grids=o.grids(), time=o.time(), mass0=m0, mass=o.mass(), values=o.values(),
                   cells=o.cell_updates())
        o.close()
    return out


def test_acoustics_1d_regression_gauges():
    r = _run(configs.acoustics_1d_regression(), 2)
    assert abs(r["time"] - 0.2) < 1e-12
    assert (r["grids"][:, 1] == 3).any()
    assert_gauges_match(r["gauges"], gauge_rows("acoustics_1d_homogeneous"))


def test_advection_1d_periodic_regression_gauges():
    r = _run(configs.advection_1d_regression(), 1)
    assert abs(r["time"] - 0.2) < 1e-12
    assert_gauges_match(r["gauges"], gauge_rows("advection_1d_example1"))
    # Nothing leaves a periodic domain, but the reference's prepc.f registers a coarse
    # cell for a fine grid's periodic image on one side only (its other branch calls
    # setuse with the 2D argument list and adds nothing), so the level-1 mass drifts by
    # the missing flux correction; the gauges above pin that behaviour
    assert abs(r["mass"] - r["mass0"]) < 1e-4 * abs(r["mass0"])


def test_euler_1d_blast_between_walls_conserves_mass():
    rd = configs.euler_1d_regression()
    rd.clawdata.tfinal = 0.004
    rd.clawdata.num_output_times = 1
    r = _run(rd, 3)
    assert abs(r["time"] - 0.004) < 1e-15
    assert (r["grids"][:, 1] == 4).any()
    np.testing.assert_allclose(r["mass"], r["mass0"], rtol=1e-13)
    v = r["values"]
    assert np.isfinite(v).all()
