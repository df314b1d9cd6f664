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


def _periodic_blast(n, levels, tfinal, max1d, bc=("periodic", "periodic", "periodic"), centre=(0.8, -0.85, 0.9)):
    """The blast with its centre near a corner of the domain, so that it crosses the periodic faces early."""
    rd = configs.euler_blast(n=n, levels=levels, tfinal=tfinal, max1d=max1d)
    for k, name in enumerate(("x0", "y0", "z0")):
        rd.probdata.add_param(name, centre[k])
    rd.clawdata.bc_lower = list(bc)
    rd.clawdata.bc_upper = list(bc)
    return rd


def test_euler_blast_periodic_conserves_mass():
    """With every direction periodic nothing leaves the domain: the level-1 mass after each
    coarse step (conck.f) stays at its initial value while the blast wraps across the faces
    and refined grids meet their periodic images (prefilp.f, preicall.f, prepc.f)."""
    rd = _periodic_blast(n=12, levels=2, tfinal=0.3, max1d=16)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle3D(d, threads=4)
        m0 = o.mass()
        o.run(0)
        grids = o.grids()
        assert o.time() > 0.2999
        lev2 = grids[grids[:, 1] == 2]
        # refined grids on both sides of the x faces (the blast wrapped around)
        assert (lev2[:, 2] == 0).any() and (lev2[:, 3] == 2 * 12 - 1).any()
        np.testing.assert_allclose(o.mass(), m0, rtol=1e-13)
        v = o.values()
        assert np.isfinite(v).all()
        o.close()


def test_euler_blast_one_periodic_direction_runs():
    """x periodic, y wall, z extrapolation: the ghost fill mixes the periodic pieces with the
    physical boundary conditions; the solve stays finite with positive density."""
    rd = _periodic_blast(n=12, levels=2, tfinal=0.3, max1d=16, bc=("periodic", "wall", "extrap"))
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle3D(d, threads=4)
        o.run(0)
        assert o.time() > 0.2999
        v = o.values()
        g = o.grids()
        assert np.isfinite(v).all()
        o.close()
