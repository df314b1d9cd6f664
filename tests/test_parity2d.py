"""GPU path versus the CPU oracle on the same inputs (2D).

FP64 results must be bit-identical: the same hierarchy (rectangles, grid numbers,
order), the same cell values and the same gauge samples. The reference pins the
oracle through its regression gauges (test_oracle2d.py); here the GPU path is held
to the oracle.
"""
import tempfile

import numpy as np
import pytest

import configs
from golden_io import assert_gauges_match, gauge_rows
from oracle.pyoracle import Oracle2D

pytestmark = pytest.mark.gpu


def _both(rd, nvar, batched=True, max_cycles=0, graphs=False):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle2D(d)
        o.run(max_cycles)
        ref = dict(grids=o.grids(), values=o.values(), gauges=o.gauges(nvar), time=o.time(), mass=o.mass(),
                   cells=o.cell_updates())
        o.close()
        with Solver(d, batched=batched, graphs=graphs) as s:
            s.run(max_cycles)
            gpu = dict(grids=s.grids(), values=s.values(), gauges=s.gauges(nvar), info=s.info(), mass=s.mass())
    return ref, gpu


def _assert_identical(ref, gpu):
    np.testing.assert_array_equal(gpu["grids"], ref["grids"])
    assert gpu["values"].shape == ref["values"].shape
    diff = np.nonzero(gpu["values"] != ref["values"])[0]
    assert diff.size == 0, "values differ at %d cells, first %s: gpu %r oracle %r" % (
        diff.size, diff[:3], gpu["values"][diff[:3]], ref["values"][diff[:3]])
    assert gpu["info"]["time"] == ref["time"]
    assert gpu["info"]["cell_updates"] == ref["cells"]
    np.testing.assert_allclose(gpu["mass"], ref["mass"], rtol=1e-13)


def test_advection_square_matches_oracle_and_reference_gauges():
    ref, gpu = _both(configs.advection_square_regression(), 1)
    _assert_identical(ref, gpu)
    np.testing.assert_array_equal(gpu["gauges"], ref["gauges"])
    assert_gauges_match(gpu["gauges"], gauge_rows("advection_2d_square"))


def test_acoustics_radial_matches_oracle_and_reference_gauges():
    ref, gpu = _both(configs.acoustics_radial_regression(), 3)
    _assert_identical(ref, gpu)
    np.testing.assert_array_equal(gpu["gauges"], ref["gauges"])
    assert_gauges_match(gpu["gauges"], gauge_rows("acoustics_2d_radial"))


def test_plain_per_patch_path_matches_batched():
    ref, gpu = _both(configs.acoustics_radial_regression(), 3, batched=False)
    _assert_identical(ref, gpu)


def test_euler_quadrants_matches_oracle():
    rd = configs.euler_quadrants(n=40, levels=3, tfinal=0.25)
    ref, gpu = _both(rd, 4)
    _assert_identical(ref, gpu)


def test_advection_bench_config_short_run():
    rd = configs.advection_square_bench(n=50, tfinal=2.0, levels=3)
    ref, gpu = _both(rd, 1, max_cycles=12)
    _assert_identical(ref, gpu)


def test_four_levels_wave_leaving_the_domain():
    # a new fine grid whose coarse neighbourhood is not covered by the coarser level
    # (filval/saveqc read the reference's initial zeros there), at an outflow boundary
    from amrclaw_b200 import problems
    ref, gpu = _both(problems.acoustics_pulse(64, levels=4, ratio=2, tfinal=0.4), 3)
    _assert_identical(ref, gpu)


def test_split_run_equals_one_run():
    from amrclaw_b200 import Solver, problems
    rd = problems.euler_quadrants(32, levels=3, ratio=2, tfinal=0.2)
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle2D(d)
        o.run(0)
        ref = dict(grids=o.grids(), values=o.values(), gauges=o.gauges(4), time=o.time(), mass=o.mass(), cells=o.cell_updates())
        o.close()
        with Solver(d) as s:
            while not s.info()["finished"]:
                s.run(3)
            gpu = dict(grids=s.grids(), values=s.values(), info=s.info(), mass=s.mass())
    _assert_identical(ref, gpu)


@pytest.mark.parametrize("batched", [True, False])
def test_cuda_graph_replay_is_identical(batched):
    """Level substeps replayed from captured CUDA graphs (dt and the fill weights read from
    device memory) give the oracle's results; graphs are re-captured after regrids and
    reused in between."""
    ref, gpu = _both(configs.acoustics_radial_regression(), 3, batched=batched, graphs=True)
    _assert_identical(ref, gpu)
    assert_gauges_match(gpu["gauges"], gauge_rows("acoustics_2d_radial"))
    assert gpu["info"]["graph_captures"] > 0
    assert gpu["info"]["graph_replays"] > 2 * gpu["info"]["graph_captures"]


def test_cuda_graph_replay_fp32_periodic():
    """The FP32 form and periodic boundaries under graph replay match direct launches."""
    from amrclaw_b200 import Solver
    rd = configs.advection_square_bench(n=32, tfinal=0.3, levels=3)
    out = []
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        for graphs in (False, True):
            with Solver(d, precision="fp32", graphs=graphs) as s:
                s.run(0)
                out.append((s.grids(), s.values()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
