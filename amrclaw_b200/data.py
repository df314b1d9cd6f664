"""Run-parameter objects and data-file writers (the setrun.py / clawdata boundary).

AMRClaw reads its run parameters positionally from text files written by
``setrun.py`` (``claw.data``, ``amr.data``, ``regions.data``, ``gauges.data``,
``setprob.data``). The read order is fixed by ``src/2d/amr2.f90:148-394`` (and
``src/3d/amr3.f90`` for 3D), ``src/python/amrclaw/data.py:62-123`` (amr.data),
``src/2d/regions_module.f90:50-60`` and ``src/2d/gauges_module.f90:92``.
clawpack's own ``ClawInputData`` writer is not part of the reference
(clawpack/clawutil is not vendored), so this module restates it: every line is
``values =: name`` and lines come in the reference's read order, so the same
files drive the reference's Fortran reader and this package's C++ reader.

Usage mirrors a reference ``setrun.py``::

    rundata = ClawRunData(num_dim=2)
    c = rundata.clawdata
    c.lower[:] = [0., 0.]; c.upper[:] = [1., 1.]; c.num_cells[:] = [50, 50]
    ...
    rundata.write(outdir)
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Any, Dict, List

_LIMITERS = {"none": 0, "minmod": 1, "superbee": 2, "vanleer": 3, "van leer": 3, "mc": 4,
             "beam_warming": 5, "bw": 5}
_BCS = {"user": 0, "extrap": 1, "periodic": 2, "wall": 3}
_TRANSVERSE = {"none": 0, "increment": 1, "all": 2}
_SPLIT = {"unsplit": 0, "godunov": 1, "strang": 2}
_SOURCE = {"none": 0, "godunov": 1, "strang": 2}
_FORMATS = {"ascii": 1, "netcdf": 2, "binary": 3}


def _code(table: Dict[str, int], v: Any) -> int:
    if isinstance(v, str):
        key = v.lower()
        if key not in table:
            raise ValueError("unknown option %r (expected one of %s)" % (v, sorted(table)))
        return table[key]
    return int(v)


def _fmt(v: Any) -> str:
    if isinstance(v, bool):
        return "T" if v else "F"
    if isinstance(v, int):
        return "%d" % v
    if isinstance(v, float):
        return "%.16e" % v
    if isinstance(v, str):
        return "'%s'" % v
    if isinstance(v, (list, tuple)):
        return "   ".join(_fmt(x) for x in v)
    return str(v)


class _Writer:
    def __init__(self, path: str):
        self.f = open(path, "w")
        self.f.write("# Written by amrclaw_b200.data (setrun.py boundary)\n\n")

    def put(self, name: str, value: Any) -> None:
        self.f.write("%-40s =: %s\n" % (_fmt(value), name))

    def blank(self) -> None:
        self.f.write("\n")

    def row(self, text: str) -> None:
        self.f.write(text + "\n")

    def close(self) -> None:
        self.f.close()


@dataclass
class ClawData:
    num_dim: int = 2
    lower: List[float] = field(default_factory=lambda: [0.0, 0.0])
    upper: List[float] = field(default_factory=lambda: [1.0, 1.0])
    num_cells: List[int] = field(default_factory=lambda: [50, 50])
    num_eqn: int = 1
    num_waves: int = 1
    num_aux: int = 0
    capa_index: int = 0
    t0: float = 0.0
    output_style: int = 1
    num_output_times: int = 1
    tfinal: float = 1.0
    output_t0: bool = True
    output_times: List[float] = field(default_factory=list)
    output_step_interval: int = 1
    total_steps: int = 1
    output_format: Any = "ascii"
    output_q_components: Any = "all"
    output_aux_components: Any = "none"
    output_aux_onlyonce: bool = True
    dt_initial: float = 1e-3
    dt_max: float = 1e99
    cfl_max: float = 1.0
    cfl_desired: float = 0.9
    steps_max: int = 100000
    dt_variable: bool = True
    order: int = 2
    transverse_waves: Any = "all"
    dimensional_split: Any = "unsplit"
    verbosity: int = 0
    source_split: Any = "none"
    use_fwaves: bool = False
    limiter: List[Any] = field(default_factory=lambda: ["mc"])
    num_ghost: int = 2
    bc_lower: List[Any] = field(default_factory=lambda: ["extrap", "extrap"])
    bc_upper: List[Any] = field(default_factory=lambda: ["extrap", "extrap"])
    restart: bool = False
    restart_file: str = "fort.chk00000"
    checkpt_style: int = 0
    checkpt_times: List[float] = field(default_factory=list)
    checkpt_interval: int = 1

    def write(self, path: str) -> None:
        # order follows src/2d/amr2.f90:148-335 (3D: src/3d/amr3.f90)
        w = _Writer(path)
        nd = self.num_dim
        w.put("num_dim", nd)
        w.put("lower", [float(x) for x in self.lower[:nd]])
        w.put("upper", [float(x) for x in self.upper[:nd]])
        w.put("num_cells", [int(x) for x in self.num_cells[:nd]])
        w.blank()
        w.put("num_eqn", int(self.num_eqn))
        w.put("num_waves", int(self.num_waves))
        w.put("num_aux", int(self.num_aux))
        w.blank()
        w.put("t0", float(self.t0))
        w.blank()
        w.put("output_style", int(self.output_style))
        if self.output_style == 1:
            w.put("num_output_times", int(self.num_output_times))
            w.put("tfinal", float(self.tfinal))
            w.put("output_t0", bool(self.output_t0))
        elif self.output_style == 2:
            w.put("output_times", [float(x) for x in self.output_times])
        elif self.output_style == 3:
            w.put("output_step_interval", int(self.output_step_interval))
            w.put("total_steps", int(self.total_steps))
            w.put("output_t0", bool(self.output_t0))
        else:
            raise ValueError("output_style must be 1, 2 or 3")
        w.blank()
        w.put("output_format", _code(_FORMATS, self.output_format))
        qc = [1] * self.num_eqn if self.output_q_components == "all" else [int(bool(x)) for x in self.output_q_components]
        w.put("output_q_components", qc)
        if self.num_aux > 0:
            if self.output_aux_components == "all":
                ac = [1] * self.num_aux
            elif self.output_aux_components == "none":
                ac = [0] * self.num_aux
            else:
                ac = [int(bool(x)) for x in self.output_aux_components]
            w.put("output_aux_components", ac)
            w.put("output_aux_onlyonce", bool(self.output_aux_onlyonce))
        w.blank()
        w.put("dt_initial", float(self.dt_initial))
        w.put("dt_max", float(self.dt_max))
        w.put("cfl_max", float(self.cfl_max))
        w.put("cfl_desired", float(self.cfl_desired))
        w.put("steps_max", int(self.steps_max))
        w.blank()
        w.put("dt_variable", bool(self.dt_variable))
        w.put("order", int(self.order))
        if nd > 1:  # src/1d/amr1.f90 reads order, verbosity, source_split, capa_index, use_fwaves
            w.put("transverse_waves", _code(_TRANSVERSE, self.transverse_waves))
            w.put("dimensional_split", _code(_SPLIT, self.dimensional_split))
        w.put("verbosity", int(self.verbosity))
        w.put("source_split", _code(_SOURCE, self.source_split))
        w.put("capa_index", int(self.capa_index))
        w.put("use_fwaves", bool(self.use_fwaves))
        w.put("limiter", [_code(_LIMITERS, x) for x in self.limiter])
        w.blank()
        w.put("num_ghost", int(self.num_ghost))
        w.put("bc_lower", [_code(_BCS, x) for x in self.bc_lower[:nd]])
        w.put("bc_upper", [_code(_BCS, x) for x in self.bc_upper[:nd]])
        w.blank()
        w.put("restart", bool(self.restart))
        w.put("restart_file", str(self.restart_file))
        w.put("checkpt_style", int(self.checkpt_style))
        if abs(int(self.checkpt_style)) == 2:
            w.put("num_checkpt_times", len(self.checkpt_times))
            w.put("checkpt_times", [float(t) for t in self.checkpt_times])
        elif abs(int(self.checkpt_style)) == 3:
            w.put("checkpt_interval", int(self.checkpt_interval))
        w.close()


@dataclass
class AmrData:
    amr_levels_max: int = 1
    refinement_ratios_x: List[int] = field(default_factory=lambda: [2])
    refinement_ratios_y: List[int] = field(default_factory=lambda: [2])
    refinement_ratios_z: List[int] = field(default_factory=lambda: [2])
    refinement_ratios_t: List[int] = field(default_factory=lambda: [2])
    aux_type: List[str] = field(default_factory=list)
    flag_richardson: bool = False
    flag_richardson_tol: float = -1.0
    flag2refine: bool = True
    flag2refine_tol: float = 0.05
    regrid_interval: int = 2
    regrid_buffer_width: int = 3
    clustering_cutoff: float = 0.7
    verbosity_regrid: int = 0
    # Largest patch extent (cells incl. ghosts) before bisection (birect.f).
    # The reference fixes it at compile time (max1d = 60 in 2D, 32 in 3D).
    max1d: int = 0

    def write(self, path: str, num_dim: int, num_aux: int) -> None:
        # order follows src/python/amrclaw/data.py:62-123
        w = _Writer(path)
        w.put("amr_levels_max", int(self.amr_levels_max))
        n = max(abs(self.amr_levels_max) - 1, 1)
        names = ("refinement_ratios_x",) + (("refinement_ratios_y",) if num_dim > 1 else ()) + \
            (("refinement_ratios_z",) if num_dim == 3 else ()) + ("refinement_ratios_t",)
        for name in names:
            v = list(getattr(self, name))
            if len(v) < n:
                raise ValueError("require len(%s) >= %d" % (name, n))
            w.put(name, [int(x) for x in v[:n]])
        w.blank()
        if num_aux > 0:
            if len(self.aux_type) < num_aux:
                raise ValueError("aux_type must list num_aux entries")
            w.put("aux_type", [str(x) for x in self.aux_type[:num_aux]])
        w.blank()
        w.put("flag_richardson", bool(self.flag_richardson))
        w.put("flag_richardson_tol", float(self.flag_richardson_tol) if self.flag_richardson else -1.0)
        w.put("flag2refine", bool(self.flag2refine))
        w.put("flag2refine_tol", float(self.flag2refine_tol))
        w.put("regrid_interval", int(self.regrid_interval))
        w.put("regrid_buffer_width", int(self.regrid_buffer_width))
        w.put("clustering_cutoff", float(self.clustering_cutoff))
        w.put("verbosity_regrid", int(self.verbosity_regrid))
        w.blank()
        for name in ("dprint", "eprint", "edebug", "gprint", "nprint", "pprint", "rprint", "sprint", "tprint", "uprint"):
            w.put(name, False)
        w.blank()
        w.put("max1d", int(self.max1d if self.max1d else {1: 500, 2: 60}.get(num_dim, 32)))
        w.close()


@dataclass
class RegionData:
    regions: List[List[float]] = field(default_factory=list)

    def write(self, path: str) -> None:
        # regions_module.f90:50-60: minlevel maxlevel t1 t2 x1 x2 y1 y2 [z1 z2]
        w = _Writer(path)
        w.put("num_regions", len(self.regions))
        for r in self.regions:
            w.row("%i  %i " % (int(r[0]), int(r[1])) + "".join("%20.14e  " % float(x) for x in r[2:]))
        w.close()


@dataclass
class GaugeData:
    gauges: List[List[float]] = field(default_factory=list)
    min_time_increment: float = 0.0

    def write(self, path: str) -> None:
        # gauges_module.f90:92: gauge_num x y [z] t_start t_end (+ min_time_increment). The
        # location and times carry the digits the reference's writer gives them
        # (src/python/amrclaw/data.py:246: %17.10e and %13.6e): a gauge on a cell edge lands
        # in the same grid as it does there.
        w = _Writer(path)
        w.put("num_gauges", len(self.gauges))
        for g in self.gauges:
            w.row("%4i" % int(g[0]) + "".join("  %17.10e" % float(x) for x in g[1:-2]) +
                  "".join("  %13.6e" % float(x) for x in g[-2:]) + "  %20.14e" % float(self.min_time_increment))
        w.close()


@dataclass
class ProbData:
    """setprob.data: the problem plugin (qinit / Riemann solver / flagging) and its constants."""
    params: Dict[str, Any] = field(default_factory=dict)

    def add_param(self, name: str, value: Any, descr: str = "") -> None:
        self.params[name] = value

    def write(self, path: str) -> None:
        w = _Writer(path)
        for k, v in self.params.items():
            w.put(k, v)
        w.close()


class ClawRunData:
    """The object a reference ``setrun.py`` builds: clawdata + amrdata + regions + gauges + probdata."""

    def __init__(self, num_dim: int = 2):
        self.clawdata = ClawData(num_dim=num_dim)
        if num_dim == 1:
            self.clawdata.lower = [0.0]
            self.clawdata.upper = [1.0]
            self.clawdata.num_cells = [100]
            self.clawdata.bc_lower = ["extrap"]
            self.clawdata.bc_upper = ["extrap"]
        if num_dim == 3:
            self.clawdata.lower = [0.0, 0.0, 0.0]
            self.clawdata.upper = [1.0, 1.0, 1.0]
            self.clawdata.num_cells = [32, 32, 32]
            self.clawdata.bc_lower = ["extrap"] * 3
            self.clawdata.bc_upper = ["extrap"] * 3
        self.amrdata = AmrData()
        self.regiondata = RegionData()
        self.gaugedata = GaugeData()
        self.probdata = ProbData()

    def write(self, outdir: str = ".") -> str:
        os.makedirs(outdir, exist_ok=True)
        c = self.clawdata
        c.write(os.path.join(outdir, "claw.data"))
        self.amrdata.write(os.path.join(outdir, "amr.data"), c.num_dim, c.num_aux)
        self.regiondata.write(os.path.join(outdir, "regions.data"))
        self.gaugedata.write(os.path.join(outdir, "gauges.data"))
        self.probdata.write(os.path.join(outdir, "setprob.data"))
        return outdir
