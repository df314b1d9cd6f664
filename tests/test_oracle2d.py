"""The CPU oracle reproduces the reference's own regression data (the oracle pin)."""
import tempfile

import configs
from golden_io import assert_gauges_match, gauge_rows
from oracle.pyoracle import Oracle2D


def _run(rd, nvar):
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle2D(d)
        o.run()
        g = o.gauges(nvar)
        o.close()
    return g


def test_advection_square_gauges_match_reference():
    # tests/advection_2d_square/regression_data/gauge0000{1,2}.txt of the reference
    g = _run(configs.advection_square_regression(), 1)
    assert_gauges_match(g, gauge_rows("advection_2d_square"))


def test_acoustics_radial_gauges_match_reference():
    # tests/acoustics_2d_radial/regression_data/gauge0000{0,1,2}.txt of the reference
    g = _run(configs.acoustics_radial_regression(), 3)
    assert_gauges_match(g, gauge_rows("acoustics_2d_radial"))


def test_advection_annulus_gauges_match_reference():
    # tests/advection_2d_annulus/regression_data/gauge0000{1,2}.txt of the reference: a mapped
    # grid with face velocities and the capacity kappa in aux (capa_index 3), periodic in theta
    g = _run(configs.advection_annulus_regression(), 1)
    assert_gauges_match(g, gauge_rows("advection_2d_annulus"))


def test_oracle_detects_a_planted_mistake():
    # A planted change of the limiter must break the pin (the comparison has teeth).
    rd = configs.advection_square_regression()
    rd.clawdata.limiter = ["minmod"]
    g = _run(rd, 1)
    try:
        assert_gauges_match(g, gauge_rows("advection_2d_square"))
    except AssertionError:
        return
    raise AssertionError("a different limiter still matched the regression data")
