"""Run configurations used by the parity tests and the benchmark.

Each builder returns an ``amrclaw_b200.data.ClawRunData`` exactly like a
reference ``setrun.py`` would: the regression-test setups restate
``tests/advection_2d_square/setrun.py`` and ``tests/acoustics_2d_radial/setrun.py``
of the reference; the benchmark workloads restate the configurations the
benchmark is quoted on (2D advection, 2D Euler quadrants, 3D Euler blast,
2D acoustics pulse, 3D swirl), with optional down-scaling for fast tests.
"""
from __future__ import annotations

import math

from amrclaw_b200.data import ClawRunData


def advection_square_regression() -> ClawRunData:
    """tests/advection_2d_square/setrun.py of the reference (gauges 1, 2 pinned)."""
    rd = ClawRunData(num_dim=2)
    p = rd.probdata
    p.add_param("problem", "advection_square")
    p.add_param("u", 0.5)
    p.add_param("v", 1.0)
    c = rd.clawdata
    c.lower = [0.0, 0.0]; c.upper = [1.0, 1.0]; c.num_cells = [50, 50]
    c.num_eqn = 1; c.num_waves = 1; c.num_aux = 0
    c.output_style = 1; c.num_output_times = 1; c.tfinal = 0.4; c.output_t0 = True
    c.dt_variable = True; c.dt_initial = 0.016; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = 100000; c.order = 2; c.transverse_waves = "all"; c.limiter = ["vanleer"]
    c.bc_lower = ["periodic", "periodic"]; c.bc_upper = ["periodic", "periodic"]
    rd.gaugedata.gauges = [[1, 0.65, 0.4, 0.0, 10.0], [2, 0.2, 0.8, 0.0, 10.0]]
    a = rd.amrdata
    a.amr_levels_max = 3; a.refinement_ratios_x = [2, 2]; a.refinement_ratios_y = [2, 2]; a.refinement_ratios_t = [2, 2]
    a.flag2refine = True; a.flag2refine_tol = 0.05; a.regrid_interval = 2; a.regrid_buffer_width = 3
    a.clustering_cutoff = 0.7
    rd.regiondata.regions = [[1, 1, 0, 1e10, 0., 1., 0., 1.], [1, 3, 0, 1e10, 0., 1., 0., 0.7]]
    return rd


def acoustics_radial_regression() -> ClawRunData:
    """tests/acoustics_2d_radial/setrun.py of the reference (gauges 0, 1, 2 pinned)."""
    rd = ClawRunData(num_dim=2)
    p = rd.probdata
    p.add_param("problem", "acoustics_cosine")
    p.add_param("rho", 1.0)
    p.add_param("bulk", 4.0)
    c = rd.clawdata
    c.lower = [-1.0, -1.0]; c.upper = [1.0, 1.0]; c.num_cells = [50, 50]
    c.num_eqn = 3; c.num_waves = 2; c.num_aux = 0
    c.output_style = 1; c.num_output_times = 1; c.tfinal = 0.2; c.output_t0 = True
    c.dt_variable = True; c.dt_initial = 1e-2; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = 50000; c.order = 2; c.transverse_waves = 2; c.limiter = ["vanleer", "vanleer"]
    c.bc_lower = ["extrap", "extrap"]; c.bc_upper = ["extrap", "extrap"]
    rd.gaugedata.gauges = [[0, 0.0, 0.0, 0., 10.], [1, 0.7, 0.0, 0., 10.],
                           [2, 0.7 / math.sqrt(2.), 0.7 / math.sqrt(2.), 0., 10.]]
    a = rd.amrdata
    a.amr_levels_max = 3; a.refinement_ratios_x = [2, 2]; a.refinement_ratios_y = [2, 2]; a.refinement_ratios_t = [2, 2]
    a.flag2refine = True; a.flag2refine_tol = 0.2; a.regrid_interval = 2; a.regrid_buffer_width = 2
    a.clustering_cutoff = 0.7
    rd.regiondata.regions = [[1, 1, 0, 1e10, -1., 1., -1., 1.], [1, 3, 0, 1e10, -1., 1., -.2, .2]]
    return rd


def advection_square_bench(n: int = 50, tfinal: float = 2.0, levels: int = 3) -> ClawRunData:
    """2D constant advection, periodic, u=(0.5,1), square IC, MC limiter, buffer 2, tol 0.05."""
    rd = advection_square_regression()
    c = rd.clawdata
    c.num_cells = [n, n]; c.tfinal = tfinal; c.limiter = ["mc"]
    rd.gaugedata.gauges = []
    rd.regiondata.regions = []
    a = rd.amrdata
    a.amr_levels_max = levels; a.regrid_buffer_width = 2
    a.refinement_ratios_x = [2] * max(1, levels - 1); a.refinement_ratios_y = [2] * max(1, levels - 1)
    a.refinement_ratios_t = [2] * max(1, levels - 1)
    return rd


def euler_quadrants(n: int = 100, levels: int = 4, tfinal: float = 0.8, ratio: int = 2) -> ClawRunData:
    """2D Euler four-quadrant Riemann problem, Roe + entropy fix, density flagging at 0.1."""
    rd = ClawRunData(num_dim=2)
    p = rd.probdata
    p.add_param("problem", "euler_quadrants")
    p.add_param("gamma", 1.4)
    p.add_param("efix", 1)
    p.add_param("flag_component", 1)
    c = rd.clawdata
    c.lower = [0.0, 0.0]; c.upper = [1.0, 1.0]; c.num_cells = [n, n]
    c.num_eqn = 4; c.num_waves = 4; c.num_aux = 0
    c.output_style = 1; c.num_output_times = 1; c.tfinal = tfinal; c.output_t0 = False
    c.dt_variable = True; c.dt_initial = 5e-4; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.order = 2; c.transverse_waves = 2; c.limiter = ["mc"] * 4
    c.bc_lower = ["extrap", "extrap"]; c.bc_upper = ["extrap", "extrap"]
    a = rd.amrdata
    a.amr_levels_max = levels
    a.refinement_ratios_x = [ratio] * max(1, levels - 1); a.refinement_ratios_y = [ratio] * max(1, levels - 1)
    a.refinement_ratios_t = [ratio] * max(1, levels - 1)
    a.flag2refine = True; a.flag2refine_tol = 0.1; a.regrid_interval = 2; a.regrid_buffer_width = 2
    a.clustering_cutoff = 0.7
    return rd


def advection_annulus_regression() -> ClawRunData:
    """tests/advection_2d_annulus/setrun.py of the reference (gauges 1, 2 pinned): advection
    on the mapped annulus 0.2 <= r <= 1, with face velocities and the capacity kappa in aux."""
    rd = ClawRunData(num_dim=2)
    p = rd.probdata
    p.add_param("problem", "advection_annulus")
    for name, val in (("A1", 1.0), ("beta1", 40.0), ("x1", -0.5), ("y1", 0.0),
                      ("A2", -1.0), ("beta2", 40.0), ("x2", 0.5), ("y2", 0.0)):
        p.add_param(name, val)
    c = rd.clawdata
    c.lower = [0.2, 0.0]; c.upper = [1.0, 2.0 * math.pi]; c.num_cells = [20, 120]
    c.num_eqn = 1; c.num_waves = 1; c.num_aux = 3; c.capa_index = 3
    c.output_style = 1; c.num_output_times = 1; c.tfinal = 0.5; c.output_t0 = True
    c.output_aux_components = "none"; c.output_aux_onlyonce = True
    c.dt_variable = True; c.dt_initial = 0.005; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = 1000; c.order = 2; c.transverse_waves = 2; c.limiter = ["vanleer"]
    c.bc_lower = ["extrap", "periodic"]; c.bc_upper = ["extrap", "periodic"]
    rd.gaugedata.gauges = [[1, 0.5, 0.5 * math.pi, 0., 10.], [2, 0.5, 1.5 * math.pi, 0., 10.]]
    a = rd.amrdata
    a.amr_levels_max = 3; a.refinement_ratios_x = [2, 2]; a.refinement_ratios_y = [2, 2]; a.refinement_ratios_t = [2, 2]
    a.aux_type = ["xleft", "yleft", "capacity"]
    a.flag2refine = True; a.flag2refine_tol = 0.02; a.regrid_interval = 2; a.regrid_buffer_width = 3
    a.clustering_cutoff = 0.7
    rd.regiondata.regions = [[1, 2, 0., 10., 0.2, 1., 0., 2. * math.pi], [3, 3, 0., 10., 0.5, 1., 0., 0.5 * math.pi]]
    return rd


def advection_swirl_regression() -> ClawRunData:
    """tests/advection_3d_swirl/setrun.py of the reference (gauges 1, 2 pinned)."""
    rd = ClawRunData(num_dim=3)
    rd.probdata.add_param("problem", "advection_swirl")
    c = rd.clawdata
    c.lower = [0.0, 0.0, 0.0]; c.upper = [1.0, 1.0, 1.0]; c.num_cells = [40, 40, 40]
    c.num_eqn = 1; c.num_waves = 1; c.num_aux = 3; c.capa_index = 0
    c.output_style = 1; c.num_output_times = 2; c.tfinal = 0.1; c.output_t0 = True
    c.dt_variable = True; c.dt_initial = 0.01; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = 5000; c.order = 2; c.transverse_waves = 22; c.limiter = ["mc"]
    c.bc_lower = ["extrap"] * 3; c.bc_upper = ["extrap"] * 3
    rd.gaugedata.gauges = [[1, 0.55, 0.4, 0.4, 0., 1e9], [2, 0.45, 0.6, 0.4, 0., 1e9]]
    a = rd.amrdata
    a.amr_levels_max = 2
    a.refinement_ratios_x = [2, 2, 2, 2]; a.refinement_ratios_y = [2, 2, 2, 2]
    a.refinement_ratios_z = [2, 2, 2, 2]; a.refinement_ratios_t = [2, 2, 2, 2]
    a.aux_type = ["xleft", "yleft", "zleft"]
    a.flag2refine = True; a.flag2refine_tol = 0.5; a.regrid_interval = 2; a.regrid_buffer_width = 3
    a.clustering_cutoff = 0.7
    a.max1d = 32
    return rd


def euler_blast(n: int = 64, levels: int = 3, tfinal: float = 0.5, seed: int = 0, max1d: int = 68) -> ClawRunData:
    """3D Euler radial blast on [-1,1]^3: rho = 1, p = 5 within r < 0.2 of a centre drawn
    uniformly from [-0.1,0.1]^3 (numpy default_rng(seed)), p = 1 outside, u = 0; Roe +
    entropy fix, pressure-difference flagging at 0.2, extrapolation boundaries."""
    import numpy as np
    cx, cy, cz = np.random.default_rng(seed).uniform(-0.1, 0.1, 3)
    rd = ClawRunData(num_dim=3)
    p = rd.probdata
    p.add_param("problem", "euler_blast")
    p.add_param("gamma", 1.4)
    p.add_param("x0", float(cx)); p.add_param("y0", float(cy)); p.add_param("z0", float(cz))
    p.add_param("r0", 0.2); p.add_param("pin", 5.0); p.add_param("pout", 1.0)
    p.add_param("flag_pressure", 1)
    c = rd.clawdata
    c.lower = [-1.0, -1.0, -1.0]; c.upper = [1.0, 1.0, 1.0]; c.num_cells = [n, n, n]
    c.num_eqn = 5; c.num_waves = 3; c.num_aux = 0
    c.output_style = 1; c.num_output_times = 1; c.tfinal = tfinal; c.output_t0 = False
    c.dt_variable = True; c.dt_initial = 0.2 / n; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = 100000; c.order = 2; c.transverse_waves = 22; c.limiter = ["mc", "mc", "mc"]
    c.bc_lower = ["extrap"] * 3; c.bc_upper = ["extrap"] * 3
    a = rd.amrdata
    a.amr_levels_max = levels
    r = [2] * max(1, levels - 1)
    a.refinement_ratios_x = list(r); a.refinement_ratios_y = list(r); a.refinement_ratios_z = list(r); a.refinement_ratios_t = list(r)
    a.flag2refine = True; a.flag2refine_tol = 0.2; a.regrid_interval = 2; a.regrid_buffer_width = 2
    a.clustering_cutoff = 0.7
    a.max1d = max1d
    return rd


def _regression_1d(problem: str, params: dict, lower: float, upper: float, n: int, meqn: int, mwaves: int, tfinal: float,
                   nout: int, dt_initial: float, steps_max: int, limiter: list, bc: str, gauges: list, levels: int,
                   ratios: list, tol: float, ibuff: int) -> ClawRunData:
    rd = ClawRunData(num_dim=1)
    rd.probdata.add_param("problem", problem)
    for k, v in params.items():
        rd.probdata.add_param(k, v)
    c = rd.clawdata
    c.lower = [lower]; c.upper = [upper]; c.num_cells = [n]
    c.num_eqn = meqn; c.num_waves = mwaves; c.num_aux = 0
    c.output_style = 1; c.num_output_times = nout; c.tfinal = tfinal; c.output_t0 = True
    c.dt_variable = True; c.dt_initial = dt_initial; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = steps_max; c.order = 2; c.limiter = limiter
    c.bc_lower = [bc]; c.bc_upper = [bc]
    rd.gaugedata.gauges = gauges
    a = rd.amrdata
    a.amr_levels_max = levels; a.refinement_ratios_x = ratios; a.refinement_ratios_t = ratios
    a.flag2refine = True; a.flag2refine_tol = tol; a.regrid_interval = 2; a.regrid_buffer_width = ibuff
    a.clustering_cutoff = 0.7
    return rd


def acoustics_1d_regression() -> ClawRunData:
    """tests/acoustics_1d_homogeneous/setrun.py of the reference (gauges 0, 1 pinned)."""
    return _regression_1d("acoustics_1d", {"rho": 1.0, "bulk": 4.0, "beta": 200.0}, -1.0, 1.0, 40, 2, 2, 0.2, 1, 1e-2, 500,
                          ["vanleer", "vanleer"], "extrap", [[0, 0.0, 0.0, 0.8], [1, 0.6, 0.0, 0.8]], 3, [2, 2], 0.1, 2)


def advection_1d_regression() -> ClawRunData:
    """tests/advection_1d_example1/setrun.py of the reference (gauges 0, 1 pinned)."""
    return _regression_1d("advection_1d", {"u": 1.0, "beta": 400.0}, 0.0, 1.0, 40, 1, 1, 0.2, 1, 0.01, 500, ["mc"],
                          "periodic", [[0, 0.2, 0.0, 1e9], [1, 0.9, 0.0, 1e9]], 3, [2, 2], 0.1, 2)


def euler_1d_regression() -> ClawRunData:
    """tests/euler_1d_wcblast/setrun.py of the reference (gauges 1, 2 pinned): the Woodward-Colella
    blast waves between walls, 4 levels with ratios 2, 6, 10."""
    return _regression_1d("euler_1d_wcblast", {"gamma": 1.4}, 0.0, 1.0, 50, 3, 3, 0.015, 2, 1e-6, 5000,
                          ["minmod"] * 3, "wall", [[1, 0.3, 0.0, 1e9], [2, 0.85, 0.0, 1e9]], 4, [2, 6, 10], 0.1, 3)
