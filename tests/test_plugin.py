"""The Riemann-solver plugin boundary: amrgpu_set_solver.

In the reference the solver is the rpn2/rpt2 (rpn3/rpt3/rptt3) pair linked into the
program, with its constants in setprob's /cparam/ block. Here a registered device plugin
is chosen by name through the C ABI and its constants are passed in. A run whose plugin
and constants are set through the ABI must give the oracle's result for a run whose
setprob.data carries those constants; bad names, counts, constants and plugins that do
not match the run's equations return AMRGPU_EINVAL and change nothing.
"""
import ctypes
import tempfile

import numpy as np
import pytest

import configs

pytestmark = pytest.mark.gpu

EINVAL = 2


def _oracle(rd, ndim, cycles):
    from oracle.pyoracle import Oracle2D, Oracle3D
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = (Oracle3D if ndim == 3 else Oracle2D)(d, threads=8)
        o.run(cycles)
        out = o.grids(), o.values(), o.time()
        o.close()
    return out


def _device(rd, cycles, name, params):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            s.set_solver(name, params)
            s.run(cycles)
            return s.grids(), s.values(), s.info()["time"]


def _same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2] == b[2]


def _set_prob(rd, **kw):
    for k, v in kw.items():
        rd.probdata.add_param(k, v)


def test_advection_velocity_set_through_the_abi():
    """Initial data and flags do not depend on (u, v): the run with the solver's velocity
    set through the ABI equals the oracle run whose setprob carries that velocity."""
    rd = configs.advection_square_bench(n=32, tfinal=0.4, levels=3)
    _set_prob(rd, u=-0.25, v=0.75)
    ref = _oracle(rd, 2, 0)
    rd0 = configs.advection_square_bench(n=32, tfinal=0.4, levels=3)  # setprob u = 0.5, v = 1.0
    got = _device(rd0, 0, "advection", [-0.25, 0.75])
    _same(got, ref)


def test_acoustics_constants_set_through_the_abi():
    rd = configs.acoustics_radial_regression()
    _set_prob(rd, rho=2.0, bulk=3.0)
    ref = _oracle(rd, 2, 6)
    got = _device(configs.acoustics_radial_regression(), 6, "acoustics", [2.0, 3.0])
    _same(got, ref)


def test_euler2d_entropy_fix_off_through_the_abi():
    rd = configs.euler_quadrants(n=40, levels=3, tfinal=0.2)
    _set_prob(rd, efix=0)
    ref = _oracle(rd, 2, 0)
    got = _device(configs.euler_quadrants(n=40, levels=3, tfinal=0.2), 0, "euler_roe_efix", [1.4, 0])
    _same(got, ref)


def test_euler3d_entropy_fix_off_through_the_abi():
    rd = configs.euler_blast(n=16, levels=2, tfinal=0.05, max1d=12)
    _set_prob(rd, efix=0)
    ref = _oracle(rd, 3, 0)
    got = _device(configs.euler_blast(n=16, levels=2, tfinal=0.05, max1d=12), 0, "euler_roe_efix", [1.4, 0])
    _same(got, ref)


def test_bad_plugin_requests_return_einval_and_change_nothing():
    from amrclaw_b200 import AmrError, Solver, _lib
    lib = _lib.load()
    cases2 = [("roe_hllc", [1.4]), ("acoustics", [1.0, 4.0]), ("euler_roe_efix", [1.4, 1, 3]),
              ("euler_roe_efix", [0.5]), ("vc_advection", [])]
    cases3 = [("euler", [1.4]), ("vc_advection", []), ("euler_roe_efix", [1.4, 1, 2])]
    for rd, cases in ((configs.euler_quadrants(n=24, levels=2, tfinal=0.05), cases2),
                      (configs.euler_blast(n=8, levels=2, tfinal=0.02, max1d=12), cases3)):
        with tempfile.TemporaryDirectory() as d:
            rd.write(d)
            with Solver(d) as s, Solver(d) as t:
                for name, params in cases:
                    with pytest.raises(AmrError) as e:
                        s.set_solver(name, params)
                    assert e.value.code == EINVAL, (name, params)
                assert lib.amrgpu_set_solver(s._h, None, None, 0) == EINVAL
                assert lib.amrgpu_set_solver(s._h, b"euler_roe_efix", None, 1) == EINVAL
                s.run(2)
                t.run(2)
                np.testing.assert_array_equal(s.values(), t.values())
