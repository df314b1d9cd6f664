"""The FP32 form against the FP64 oracle (2D and 3D).

FP32 storage, ghost values, Riemann solves and flux differencing; FP64 flux registers,
register corrections, averages, totals and time steps. Its error is stated, not zero:
on the acoustic pulse (64^2, 4 levels, t = 0.4) the level-1 L1 error relative to the
FP64 oracle must stay below 1e-5 in every component and the level-1 mass within 1e-7
of the oracle's. Both runs share the base level, where the comparison is made. On the
3D blast (16^3, 3 levels, t = 0.2) the bound is 1e-5 per component and 1e-7 on the mass.
"""
import tempfile

import numpy as np
import pytest

from amrclaw_b200 import fields, problems
from oracle.pyoracle import Oracle2D, Oracle3D

import configs

pytestmark = pytest.mark.gpu

L1_REL_TOL = 1e-5
MASS_REL_TOL = 1e-7


def _fp32_vs_oracle(rd, nvar, n, width, ndim=2):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = (Oracle2D if ndim == 2 else Oracle3D)(d, threads=8)
        o.run(0)
        g64, v64, m64 = o.grids(), o.values(), o.mass()
        o.close()
        with Solver(d, precision="fp32") as s:
            s.run(0)
            g32, v32, m32, inf = s.grids(), s.values(), s.mass(), s.info()
    assert inf["precision_bits"] == 32
    dx = width / n
    ref = fields.level_array(g64, v64, nvar, 1, (n,) * ndim)
    got = fields.level_array(g32, v32, nvar, 1, (n,) * ndim)
    assert not np.isnan(got).any()
    _, rel = fields.l1_error(got, ref, dx ** ndim)
    return rel, abs(m32 - m64) / abs(m64)


def test_acoustics_pulse_fp32_within_stated_error():
    rel, mass = _fp32_vs_oracle(problems.acoustics_pulse(64, levels=4, ratio=2, tfinal=0.4), 3, 64, 2.0)
    assert (rel < L1_REL_TOL).all(), rel
    assert mass < MASS_REL_TOL
    assert rel.max() > 0.0  # it is FP32: not bit-identical


def test_euler_quadrants_fp32_within_stated_error():
    rel, mass = _fp32_vs_oracle(problems.euler_quadrants(48, levels=3, ratio=2, tfinal=0.2), 4, 48, 1.0)
    assert (rel < 1e-4).all(), rel
    assert mass < 1e-6


def test_fp32_context_rejects_the_fixed_scratch_entry_point():
    from amrclaw_b200 import AmrError, Solver
    with Solver(problems.advection_square(32, levels=2, tfinal=0.05), precision="fp32") as s:
        with pytest.raises(AmrError):
            s.level_advance_noalloc(1)


def test_euler_blast3d_fp32_within_stated_error():
    rel, mass = _fp32_vs_oracle(configs.euler_blast(n=16, levels=3, tfinal=0.2, max1d=16), 5, 16, 2.0, ndim=3)
    assert (rel < L1_REL_TOL).all(), rel
    assert mass < MASS_REL_TOL
    assert rel.max() > 0.0


def test_euler_blast3d_fp32_plain_path_matches_batched():
    """The per-grid (plain) path runs the same FP32 kernels one patch at a time: its results
    equal the batched path's bit for bit, as in FP64."""
    from amrclaw_b200 import Solver
    rd = configs.euler_blast(n=16, levels=2, tfinal=0.05, max1d=12)
    out = []
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        for batched in (True, False):
            with Solver(d, batched=batched, precision="fp32") as s:
                s.run(0)
                out.append((s.grids(), s.values()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
