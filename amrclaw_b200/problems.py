"""Run-data builders for the problems the device path ships (the reference's example
applications, as a setrun.py would write them).

Each returns a ClawRunData for the given base grid, number of levels, refinement ratio
and final time; the keyword arguments set the problem's parameters (setprob.data).
"""
from __future__ import annotations

from .data import ClawRunData


def _amr(rd: ClawRunData, levels: int, ratio: int, tol: float, buffer: int = 2) -> None:
    a = rd.amrdata
    r = [ratio] * max(1, levels - 1)
    a.amr_levels_max = levels
    a.refinement_ratios_x = list(r); a.refinement_ratios_y = list(r); a.refinement_ratios_t = list(r)
    a.flag2refine = True; a.flag2refine_tol = tol; a.regrid_interval = 2; a.regrid_buffer_width = buffer
    a.clustering_cutoff = 0.7


def _claw(rd: ClawRunData, lower, upper, n: int, meqn: int, mwaves: int, tfinal: float, dt0: float, limiter, bc) -> None:
    c = rd.clawdata
    c.lower = list(lower); c.upper = list(upper); c.num_cells = [n, n]
    c.num_eqn = meqn; c.num_waves = mwaves; c.num_aux = 0
    c.output_style = 1; c.num_output_times = 1; c.tfinal = tfinal; c.output_t0 = False
    c.dt_variable = True; c.dt_initial = dt0; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = 1000000; c.order = 2; c.transverse_waves = 2; c.limiter = [limiter] * mwaves
    c.bc_lower = [bc, bc]; c.bc_upper = [bc, bc]


def advection_square(n: int, levels: int = 3, ratio: int = 2, tfinal: float = 1.0, u: float = 0.5, v: float = 1.0,
                     x0: float = 0.1, x1: float = 0.6, y0: float = 0.1, y1: float = 0.6) -> ClawRunData:
    """Constant advection of a square on the periodic unit square (examples/advection_2d_square)."""
    rd = ClawRunData(num_dim=2)
    p = rd.probdata
    p.add_param("problem", "advection_square")
    for k, val in (("u", u), ("v", v), ("x0", x0), ("x1", x1), ("y0", y0), ("y1", y1)):
        p.add_param(k, val)
    _claw(rd, (0.0, 0.0), (1.0, 1.0), n, 1, 1, tfinal, 0.4 / n, "mc", "periodic")
    _amr(rd, levels, ratio, 0.05)
    return rd


def euler_quadrants(n: int, levels: int = 3, ratio: int = 2, tfinal: float = 0.8, xs: float = 0.8,
                    ys: float = 0.8) -> ClawRunData:
    """2D Euler four-quadrant Riemann problem (examples/euler_2d_quadrants), density flag 0.1."""
    rd = ClawRunData(num_dim=2)
    p = rd.probdata
    p.add_param("problem", "euler_quadrants")
    p.add_param("gamma", 1.4); p.add_param("efix", 1); p.add_param("flag_component", 1)
    p.add_param("xs", xs); p.add_param("ys", ys)
    _claw(rd, (0.0, 0.0), (1.0, 1.0), n, 4, 4, tfinal, 0.05 / n, "mc", "extrap")
    _amr(rd, levels, ratio, 0.1)
    return rd


def acoustics_pulse(n: int, levels: int = 3, ratio: int = 2, tfinal: float = 0.4, r0: float = 0.3, width: float = 0.05,
                    rho: float = 1.0, bulk: float = 4.0) -> ClawRunData:
    """2D acoustics on [-1,1]^2 with a radial Gaussian pressure pulse p = exp(-((r-r0)/width)^2)."""
    rd = ClawRunData(num_dim=2)
    p = rd.probdata
    p.add_param("problem", "acoustics_gauss")
    p.add_param("rho", rho); p.add_param("bulk", bulk); p.add_param("r0", r0); p.add_param("width", width)
    _claw(rd, (-1.0, -1.0), (1.0, 1.0), n, 3, 2, tfinal, 0.5 / n, "mc", "extrap")
    _amr(rd, levels, ratio, 0.05)
    return rd


def advection_swirl3d(n: int = 32, levels: int = 4, ratio: int = 2, tfinal: float = 1.5, sphere: bool = True,
                      vel_period: float = 1.5, x0: float = 0.5, y0: float = 0.25, z0: float = 0.5, r0: float = 0.15,
                      tol: float = 0.1, max1d: int = 32) -> ClawRunData:
    """3D advection in the swirling field u = 2 sin^2(pi x) sin(2 pi y) sin(2 pi z), v and w
    permuted likewise, on [0,1]^3 (examples/advection_3d_swirl), face-centred velocities in
    aux 1..3. sphere: q = 1 within r0 of (x0, y0, z0), else the example's half space x < 0.5;
    vel_period > 0 scales the field by cos(pi t / vel_period) before every step (b4step3)."""
    rd = ClawRunData(num_dim=3)
    p = rd.probdata
    p.add_param("problem", "advection_swirl")
    p.add_param("ic", "sphere" if sphere else "halfspace")
    for k, val in (("x0", x0), ("y0", y0), ("z0", z0), ("r0", r0), ("vel_period", vel_period)):
        p.add_param(k, val)
    c = rd.clawdata
    c.lower = [0.0, 0.0, 0.0]; c.upper = [1.0, 1.0, 1.0]; c.num_cells = [n, n, n]
    c.num_eqn = 1; c.num_waves = 1; c.num_aux = 3; c.capa_index = 0
    c.output_style = 1; c.num_output_times = 1; c.tfinal = tfinal; c.output_t0 = False
    c.dt_variable = True; c.dt_initial = 0.4 / n; c.dt_max = 1e99; c.cfl_desired = 0.9; c.cfl_max = 1.0
    c.steps_max = 1000000; c.order = 2; c.transverse_waves = 22; c.limiter = ["mc"]
    c.bc_lower = ["extrap"] * 3; c.bc_upper = ["extrap"] * 3
    a = rd.amrdata
    r = [ratio] * max(1, levels - 1)
    a.amr_levels_max = levels
    a.refinement_ratios_x = list(r); a.refinement_ratios_y = list(r); a.refinement_ratios_z = list(r)
    a.refinement_ratios_t = list(r)
    a.aux_type = ["xleft", "yleft", "zleft"]
    a.flag2refine = True; a.flag2refine_tol = tol; a.regrid_interval = 2; a.regrid_buffer_width = 2
    a.clustering_cutoff = 0.7
    a.max1d = max1d
    return rd
