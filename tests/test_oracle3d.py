"""The 3D CPU oracle against the reference's regression data (no GPU needed).

tests/advection_3d_swirl of the reference: 40^3, 2 levels, face-centred swirl
velocities (3 aux), CTU with transverse_waves = 22, MC limiter. Its two gauges
(20 samples each, printed e15.7) must be reproduced to 7 digits.
"""
import tempfile

import numpy as np

import configs
from golden_io import assert_gauges_match, gauge_rows
from oracle.pyoracle import Oracle3D


def test_swirl_regression_gauges():
    rd = configs.advection_swirl_regression()
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle3D(d, threads=4)
        o.run(0)
        g = o.gauges(1)
        assert abs(o.time() - 0.1) < 1e-12
        o.close()
    assert_gauges_match(g, gauge_rows("advection_3d_swirl"))


def test_euler_blast_small_runs_and_conserves_mass():
    rd = configs.euler_blast(n=16, levels=2, tfinal=0.05, max1d=20)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle3D(d, threads=4)
        m0 = o.mass()
        o.run(0)
        grids = o.grids()
        assert o.time() > 0.0499
        assert (grids[:, 1] == 2).any()
        # extrapolation boundaries: nothing has reached the boundary yet, so level-1 mass is conserved
        np.testing.assert_allclose(o.mass(), m0, rtol=1e-13)
        o.close()
