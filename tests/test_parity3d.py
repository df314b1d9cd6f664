"""GPU path versus the CPU oracle on the same inputs (3D Euler).

FP64 results must be bit-identical: the same hierarchy (boxes, grid numbers,
order), the same cell values, the same gauge samples and the same cell-update
count. The oracle itself is pinned to the reference's 3D regression gauges in
test_oracle3d.py.
"""
import tempfile

import numpy as np
import pytest

import configs
from oracle.pyoracle import Oracle3D

pytestmark = pytest.mark.gpu


def _both(rd, batched=True, max_cycles=0, split=None, graphs=False, schedule=0):
    from amrclaw_b200 import Solver
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle3D(d, threads=8)
        o.run(max_cycles)
        ref = dict(grids=o.grids(), values=o.values(), gauges=o.gauges(5), time=o.time(), mass=o.mass(),
                   cells=o.cell_updates())
        o.close()
        with Solver(d, batched=batched, graphs=graphs, schedule=schedule) as s:
            assert s.num_dim == 3
            if split:
                for _ in range(max_cycles // split):
                    s.run(split)
            else:
                s.run(max_cycles)
            gpu = dict(grids=s.grids(), values=s.values(), gauges=s.gauges(5), info=s.info(), mass=s.mass())
    return ref, gpu


def _assert_identical(ref, gpu):
    assert gpu["grids"].shape[1] == 8
    np.testing.assert_array_equal(gpu["grids"], ref["grids"])
    assert gpu["values"].shape == ref["values"].shape
    diff = np.nonzero(gpu["values"] != ref["values"])[0]
    assert diff.size == 0, "values differ at %d cells, first %s: gpu %r oracle %r" % (
        diff.size, diff[:3], gpu["values"][diff[:3]], ref["values"][diff[:3]])
    assert gpu["info"]["time"] == ref["time"]
    assert gpu["info"]["cell_updates"] == ref["cells"]
    assert gpu["info"]["num_dim"] == 3.0
    np.testing.assert_allclose(gpu["mass"], ref["mass"], rtol=1e-13)
    np.testing.assert_array_equal(gpu["gauges"], ref["gauges"])


def _with_gauges(rd):
    rd.gaugedata.gauges.append([1, 0.05, -0.02, 0.03, 0.0, 1e9])
    rd.gaugedata.gauges.append([2, 0.31, 0.12, -0.27, 0.0, 1e9])
    return rd


def test_blast_two_levels_many_patches():
    rd = _with_gauges(configs.euler_blast(n=16, levels=2, tfinal=0.05, max1d=12))
    ref, gpu = _both(rd)
    assert (ref["grids"][:, 1] == 2).sum() > 1
    _assert_identical(ref, gpu)
    assert len(gpu["gauges"]) > 0


def test_blast_three_levels_regrids():
    rd = _with_gauges(configs.euler_blast(n=16, levels=3, tfinal=0.1, max1d=16))
    ref, gpu = _both(rd)
    assert (ref["grids"][:, 1] == 3).any()
    _assert_identical(ref, gpu)


def test_blast_wall_boundaries_reach_the_wall():
    rd = configs.euler_blast(n=12, levels=2, tfinal=0.6, max1d=16)
    rd.clawdata.bc_lower = ["wall"] * 3
    rd.clawdata.bc_upper = ["extrap", "wall", "extrap"]
    ref, gpu = _both(rd)
    _assert_identical(ref, gpu)


def test_plain_per_patch_path_matches_batched():
    rd = configs.euler_blast(n=16, levels=2, tfinal=0.05, max1d=12)
    ref, gpu = _both(rd, batched=False)
    _assert_identical(ref, gpu)


def test_split_run_equals_one_run():
    rd = configs.euler_blast(n=16, levels=3, tfinal=10.0, max1d=20)
    ref, gpu = _both(rd, max_cycles=6, split=2)
    _assert_identical(ref, gpu)


@pytest.mark.parametrize("batched", [True, False])
def test_cuda_graph_replay_is_identical(batched):
    """Level substeps replayed from captured CUDA graphs (scalars read from device memory)
    give the same results as direct launches; graphs are re-captured after regrids and
    reused in between."""
    rd = _with_gauges(configs.euler_blast(n=16, levels=3, tfinal=0.1, max1d=16))
    ref, gpu = _both(rd, batched=batched, graphs=True, schedule=1)
    _assert_identical(ref, gpu)
    assert gpu["info"]["graph_captures"] > 0
    assert gpu["info"]["graph_replays"] > 2 * gpu["info"]["graph_captures"]


def test_autotuned_schedule_then_graphs_is_identical():
    """Levels launch directly while the sweep schedule is tuned, then replay graphs."""
    rd = configs.euler_blast(n=16, levels=3, tfinal=0.1, max1d=16)
    ref, gpu = _both(rd, graphs=True)
    _assert_identical(ref, gpu)
    assert gpu["info"]["levels_tuned_queue"] + gpu["info"]["levels_tuned_per_direction"] >= 2
    assert gpu["info"]["graph_replays"] > 0


@pytest.mark.parametrize("schedule", [1, 2])
def test_sweep_schedules_are_identical(schedule):
    """Per-direction sweep launches (1) and the persistent work-queue launch (2) give the
    oracle's results; the default (0) autotunes between them per level."""
    rd = _with_gauges(configs.euler_blast(n=16, levels=3, tfinal=0.1, max1d=16))
    ref, gpu = _both(rd, schedule=schedule)
    _assert_identical(ref, gpu)


def _periodic_blast(n, levels, tfinal, max1d, bc, centre=(0.8, -0.85, 0.9)):
    """The blast centred near a corner, so that it crosses the periodic faces early."""
    rd = configs.euler_blast(n=n, levels=levels, tfinal=tfinal, max1d=max1d)
    for k, name in enumerate(("x0", "y0", "z0")):
        rd.probdata.add_param(name, centre[k])
    rd.clawdata.bc_lower = list(bc)
    rd.clawdata.bc_upper = list(bc)
    return rd


@pytest.mark.parametrize("bc", [("periodic", "periodic", "periodic"), ("periodic", "wall", "extrap"),
                                ("extrap", "periodic", "periodic")])
def test_blast_periodic_boundaries(bc):
    """Periodic faces (prefilp.f pieces in bound and filpatch, preicall.f in saveqc and
    filval, prepc.f register images, periodic domain-flag rings), alone and mixed with wall
    and extrapolation faces, on three levels with regrids."""
    rd = _with_gauges(_periodic_blast(n=12, levels=3, tfinal=0.15, max1d=16, bc=bc))
    ref, gpu = _both(rd)
    lev2 = ref["grids"][ref["grids"][:, 1] == 2]
    per = [k for k in range(3) if bc[k] == "periodic"]
    # refined grids touch both faces of a periodic direction: the blast wrapped around
    assert any((lev2[:, 2 + 2 * k] == 0).any() and (lev2[:, 3 + 2 * k] == 2 * 12 - 1).any() for k in per)
    _assert_identical(ref, gpu)


def test_blast_periodic_plain_path_and_richardson():
    """The per-patch path with Richardson estimation on a periodic domain (the big step's
    wide ghost ring is filled through the periodic pieces too)."""
    rd = _periodic_blast(n=12, levels=2, tfinal=0.1, max1d=16, bc=("periodic",) * 3)
    rd.amrdata.flag_richardson = True
    rd.amrdata.flag_richardson_tol = 2e-3
    ref, gpu = _both(rd, batched=False)
    _assert_identical(ref, gpu)


@pytest.mark.parametrize("ratios", [((3,), (3,), (3,)), ((4,), (2,), (3,)), ((2, 4), (2, 4), (2, 4))])
@pytest.mark.parametrize("batched", [True, False])
def test_blast_other_refinement_ratios(ratios, batched):
    """Refinement ratios other than 2, isotropic and anisotropic: a coarse face of a fine
    patch then holds 9 to 16 coarse-fine Riemann problems (qad.f), so the device's register
    groups sum them over several rounds, and the last round of a 3 x 3 face is partial."""
    levels = len(ratios[0]) + 1
    rd = configs.euler_blast(n=12, levels=levels, tfinal=0.1, seed=3, max1d=40)
    a = rd.amrdata
    rx, ry, rz = (list(r) for r in ratios)
    a.refinement_ratios_x = rx; a.refinement_ratios_y = ry; a.refinement_ratios_z = rz
    a.refinement_ratios_t = [max(x, y, z) for x, y, z in zip(rx, ry, rz)]
    ref, gpu = _both(rd, batched=batched)
    _assert_identical(ref, gpu)
    assert ref["grids"][:, 1].max() == levels  # the finest level exists
