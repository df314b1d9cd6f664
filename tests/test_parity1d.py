"""The 1D device path against the 1D CPU oracle (and the reference's 1D regression data).

FP64 results must be bit-identical: the same hierarchy (grid numbers, levels, boxes), the
same cell values, the same gauge samples, time and cell-update count. The oracle itself is
pinned to the reference's 1D regression gauges in test_oracle1d.py; the device's gauges
are checked against them here too.
"""
import os
import tempfile

import numpy as np
import pytest

import configs
from golden_io import assert_gauges_match, gauge_rows
from oracle.pyoracle import Oracle1D

pytestmark = pytest.mark.gpu


def _both(rd, nvar, max_cycles=0, outdirs=None):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        od = outdirs[0] if outdirs else None
        o = Oracle1D(d, outdir=od, write_output=od is not None)
        o.run(max_cycles)
        ref = dict(grids=o.grids(), values=o.values(), gauges=o.gauges(nvar), time=o.time(), cells=o.cell_updates(), mass=o.mass())
        o.close()
        od = outdirs[1] if outdirs else None
        with Solver(d, outdir=od, write_output=od is not None) as s:
            assert s.num_dim == 1
            s.run(max_cycles)
            gpu = dict(grids=s.grids(), values=s.values(), gauges=s.gauges(nvar), info=s.info(), mass=s.mass())
    return ref, gpu


def _assert_identical(ref, gpu):
    np.testing.assert_array_equal(gpu["grids"], ref["grids"])
    assert gpu["values"].shape == ref["values"].shape
    diff = np.nonzero(gpu["values"] != ref["values"])[0]
    assert diff.size == 0, "values differ at %d cells, first %s" % (diff.size, diff[:3])
    assert gpu["info"]["time"] == ref["time"]
    assert gpu["info"]["cell_updates"] == ref["cells"]
    assert gpu["info"]["num_dim"] == 1.0
    np.testing.assert_array_equal(gpu["gauges"], ref["gauges"])
    assert gpu["mass"] == ref["mass"]


def test_acoustics_1d_regression_matches_oracle_and_reference_gauges():
    ref, gpu = _both(configs.acoustics_1d_regression(), 2)
    _assert_identical(ref, gpu)
    assert (gpu["grids"][:, 1] == 3).any()
    assert_gauges_match(gpu["gauges"], gauge_rows("acoustics_1d_homogeneous"))


def test_advection_1d_periodic_regression_matches_oracle_and_reference_gauges():
    ref, gpu = _both(configs.advection_1d_regression(), 1)
    _assert_identical(ref, gpu)
    assert_gauges_match(gpu["gauges"], gauge_rows("advection_1d_example1"))


def test_euler_1d_blast_between_walls_matches_oracle():
    rd = configs.euler_1d_regression()
    rd.clawdata.tfinal = 0.004
    rd.clawdata.num_output_times = 1
    ref, gpu = _both(rd, 3)
    assert (ref["grids"][:, 1] == 4).any()
    _assert_identical(ref, gpu)


def test_euler_1d_plugin_through_the_c_abi():
    """The Euler plugin chosen and parametrised through amrgpu_set_solver (gamma) gives the
    oracle's result for the same gamma; a wrong constant count is refused."""
    from amrclaw_b200 import AmrError, Solver
    rd = configs.euler_1d_regression()
    rd.clawdata.tfinal = 0.002
    rd.probdata.add_param("gamma", 1.4)
    ref, _ = _both(rd, 3)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        with Solver(d) as s:
            with pytest.raises(AmrError) as e:
                s.set_solver("euler_roe_efix", [1.4, 1.0])
            assert e.value.code == 2
            s.set_solver("euler_roe_efix", [1.4])
            s.run(0)
            np.testing.assert_array_equal(s.grids(), ref["grids"])
            np.testing.assert_array_equal(s.values(), ref["values"])


@pytest.mark.parametrize("fmt", ["ascii", "binary"])
def test_output_files_1d_identical_to_oracle(fmt):
    rd = configs.acoustics_1d_regression()
    rd.clawdata.num_output_times = 2
    rd.clawdata.output_format = fmt
    with tempfile.TemporaryDirectory() as a, tempfile.TemporaryDirectory() as b:
        _both(rd, 2, outdirs=(a, b))
        names = sorted(f for f in os.listdir(a) if f.startswith("fort."))
        assert names == sorted(f for f in os.listdir(b) if f.startswith("fort."))
        assert any(n.startswith("fort.q") for n in names) and any(n.startswith("fort.t") for n in names)
        for n in names:
            with open(os.path.join(a, n), "rb") as fa, open(os.path.join(b, n), "rb") as fb:
                assert fa.read() == fb.read(), n
