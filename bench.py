#!/usr/bin/env python
"""Benchmark of the B200 AMRClaw patch-advance path.

One "step" is one coarse time step of the AMR hierarchy (tick.f cycle): every
level substep (ghost fill, saved coarse values, patch steps, flux registers),
the level syncs and the regrids that fall in it. The metric is cell-updates/s,
counted as the reference counts them (src/2d/advanc.f:223-224: interior cells per
patch per level substep). ``value`` is the batched path (one launch per level)
with the hierarchy resident in HBM; ``plain`` is the per-patch launch path on
the same steps; ``e2e`` is the whole solve through the C ABI from host input
files to host results.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Under torchrun each rank runs an independent replica of the workload (replicas
only: one AMR hierarchy per GPU, no exchange); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "cell-updates/s batched vs plain GPU at stated L1 err vs FP64; p50/p99 solve latency"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def workload(name: str):
    """(run data, config record, meqn, naux, num_dim) of a named workload."""
    import configs
    if name == "euler3d_blast":
        rd = configs.euler_blast(n=64, levels=3, tfinal=0.5, seed=0, max1d=68)
        return rd, dict(workload=name, base_grid="64x64x64", levels=3, ratio=2, solver="Roe+entropy fix, CTU 3D (22)",
                        meqn=5, naux=0, tfinal=0.5, seed=0, max1d=68, flag="pressure difference > 0.2",
                        bc="extrapolation", precision="fp64"), 5, 0, 3
    if name == "euler3d_blast_48":
        # the same blast on a 48^3 base grid with 2 levels: the profiling case (its level-1 step
        # staging is larger than L2, its device memory a few hundred MB)
        rd = configs.euler_blast(n=48, levels=2, tfinal=0.5, seed=0, max1d=68)
        return rd, dict(workload=name, base_grid="48x48x48", levels=2, ratio=2, solver="Roe+entropy fix, CTU 3D (22)",
                        meqn=5, naux=0, tfinal=0.5, seed=0, max1d=68, flag="pressure difference > 0.2",
                        bc="extrapolation", precision="fp64"), 5, 0, 3
    if name == "euler2d_quadrants":
        rd = configs.euler_quadrants(n=100, levels=4, tfinal=0.8)
        return rd, dict(workload=name, base_grid="100x100", levels=4, ratio=2, solver="Roe+entropy fix", meqn=4,
                        naux=0, tfinal=0.8, precision="fp64"), 4, 0, 2
    if name == "advection2d_square":
        rd = configs.advection_square_bench(n=50, tfinal=2.0, levels=3)
        return rd, dict(workload=name, base_grid="50x50", levels=3, ratio=2, solver="constant advection (0.5, 1.0)",
                        meqn=1, naux=0, tfinal=2.0, bc="periodic", limiter="MC", precision="fp64"), 1, 0, 2
    if name == "acoustics2d_pulse_fp32":
        from amrclaw_b200 import problems
        rd = problems.acoustics_pulse(64, levels=4, ratio=2, tfinal=0.4)
        return rd, dict(workload=name, base_grid="64x64", levels=4, ratio=2, solver="acoustics rho=1 K=4", meqn=3,
                        naux=0, tfinal=0.4, precision="fp32"), 3, 0, 2
    if name == "swirl3d_fp32":
        from amrclaw_b200 import problems
        rd = problems.advection_swirl3d(n=32, levels=4, tfinal=1.5)
        return rd, dict(workload=name, base_grid="32x32x32", levels=4, ratio=2,
                        solver="advection in the swirl field x cos(pi t / 1.5), sphere r=0.15", meqn=1, naux=3,
                        tfinal=1.5, precision="fp32"), 1, 3, 3
    raise SystemExit("unknown workload %s" % name)


# FP64 operations per cell-update of the 3D Euler CTU (transverse_waves 22) step kernels:
# dadd + dmul + 2*dfma thread instructions of the three sweeps of a level-1 step, divided by
# its cells (ncu instruction counts; the count does not depend on the patch sizes)
FLOPS_PER_CELL_UPDATE_3D = 10.4e3
# DRAM bytes per cell-update of the same kernels (sweeps, face gather, update): ncu
# dram__bytes_read.sum + dram__bytes_write.sum of a level-1 substep of the 64^3 blast,
# 1,070 MB over 262,144 cell-updates
DRAM_BYTES_PER_CELL_UPDATE_3D = 1070.2e6 / 262144


def fp64_peak_tflops() -> float:
    """Measured FP64 peak of this GPU: a 4096^3 DGEMM (2*N^3 flops), best of 5."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def oracle_cls(ndim):
    from oracle.pyoracle import Oracle2D, Oracle3D
    return Oracle3D if ndim == 3 else Oracle2D


def peaks():
    try:
        with open(PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self):
        self.rows = []
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + q, "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        dev = os.environ.get("LOCAL_RANK", "0")
        rows = [r for r in self.rows if len(r) >= 9 and r[0] == dev] or [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, n in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows)}


def flush_l2(buf):
    buf.fill_(1.0)
    import torch
    torch.cuda.synchronize()


def fp32_leg(cpu_threads: int, rd3=None, cfg3=None) -> dict:
    """The FP32 form. 2D acoustic pulse (64^2 base grid, 4 levels, ratio 2, t = 0.4): device
    throughput of the FP32 and FP64 runs, and the FP32 run's level-1 L1 error and mass
    against the FP64 oracle (the reference's arithmetic). 3D (rd3, the headline workload):
    FP32 and FP64 device throughput over the whole solve and the FP32 level-1 L1 error
    against the FP64 device run, which the parity tests hold bit-identical to the oracle
    (the oracle itself would take minutes at this size)."""
    from amrclaw_b200 import Solver, fields, problems
    from oracle.pyoracle import Oracle2D
    rd = problems.acoustics_pulse(64, levels=4, ratio=2, tfinal=0.4)
    out = {"workload": "acoustics2d_pulse", "base_grid": "64x64", "levels": 4, "ratio": 2, "tfinal": 0.4}
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = Oracle2D(d, threads=cpu_threads)
        o.run(0)
        g64, v64, m64 = o.grids(), o.values(), o.mass()
        o.close()
        res = {}
        for prec in ("fp64", "fp32"):
            with Solver(d, precision=prec) as s:
                s.run(0)
                inf = s.info()
                res[prec] = (s.grids(), s.values(), s.mass(), inf["cell_updates"] / (inf["last_run_ms"] * 1e-3))
    ref = fields.level_array(g64, v64, 3, 1, (64, 64))
    for prec, (g, v, m, cups) in res.items():
        _, rel = fields.l1_error(fields.level_array(g, v, 3, 1, (64, 64)), ref, (2.0 / 64) ** 2)
        out[prec] = {"value": cups, "unit": "cell-updates/s", "l1_rel_err_vs_fp64_oracle": [float(x) for x in rel],
                     "mass_rel_diff_vs_fp64_oracle": abs(m - m64) / abs(m64)}
    if rd3 is not None:
        n = cfg3["base_grid"]
        n = int(str(n).split("x")[0]) if not isinstance(n, int) else n
        o3 = {"workload": cfg3["workload"], "base_grid": cfg3["base_grid"], "levels": cfg3.get("levels")}
        with tempfile.TemporaryDirectory() as d:
            rd3.write(d)
            res = {}
            for prec in ("fp64", "fp32"):
                with Solver(d, precision=prec) as s:
                    s.run(0)
                    inf = s.info()
                    res[prec] = (s.grids(), s.values(), s.mass(), inf["cell_updates"], inf["last_run_ms"])
        g, v, m, _, _ = res["fp64"]
        ref = fields.level_array(g, v, 5, 1, (n, n, n))
        for prec, (g, v, mm, cells, ms) in res.items():
            _, rel = fields.l1_error(fields.level_array(g, v, 5, 1, (n, n, n)), ref, (2.0 / n) ** 3)
            o3[prec] = {"value": cells / (ms * 1e-3), "unit": "cell-updates/s", "solve_ms": ms, "cell_updates": cells,
                        "l1_rel_err_vs_fp64": [float(x) for x in rel], "mass_rel_diff_vs_fp64": abs(mm - m) / abs(m)}
        out["blast3d"] = o3
    out["swirl3d"] = swirl_fp32_leg(cpu_threads)
    return out


def swirl_fp32_leg(cpu_threads: int) -> dict:
    """The FP32 form on the 3D swirl (sphere r = 0.15 at (0.5, 0.25, 0.5), velocity field
    scaled by cos(pi t / 1.5), 32^3 base grid, 4 levels, ratio 2): level-1 L1 error and mass
    against the FP64 oracle at t = 0.1 (an oracle run of seconds), and against the FP64
    device path, which the parity tests hold bit-identical to the oracle, over the whole
    period to t = 1.5; mass drift is the relative change of the level-1 mass over the run."""
    from amrclaw_b200 import Solver, fields, problems
    from oracle.pyoracle import Oracle3D
    n = 32
    out = {"workload": "swirl3d_sphere_modulated", "base_grid": "32x32x32", "levels": 4, "ratio": 2,
           "velocity": "swirl x cos(pi t / 1.5)", "ic": "sphere r=0.15 at (0.5,0.25,0.5)"}

    def run(tfinal, precisions, with_oracle):
        rd = problems.advection_swirl3d(n=n, levels=4, tfinal=tfinal)
        res = {}
        with tempfile.TemporaryDirectory() as d:
            rd.write(d)
            if with_oracle:
                o = Oracle3D(d, threads=cpu_threads)
                o.run(0)
                res["oracle"] = (o.grids(), o.values(), o.mass(), None, None, None)
                o.close()
            for prec in precisions:
                with Solver(d, precision=prec) as s:
                    m0 = s.mass()
                    s.run(0)
                    inf = s.info()
                    res[prec] = (s.grids(), s.values(), s.mass(), m0, inf["cell_updates"], inf["last_run_ms"])
        return res

    def compare(res, ref_key, key):
        g, v, m, _, _, _ = res[ref_key]
        ref = fields.level_array(g, v, 1, 1, (n, n, n))
        g2, v2, m2, m0, cells, ms = res[key]
        _, rel = fields.l1_error(fields.level_array(g2, v2, 1, 1, (n, n, n)), ref, (1.0 / n) ** 3)
        return float(rel[0]), abs(m2 - m) / abs(m), (m2 - m0) / m0, cells / (ms * 1e-3)

    short = run(0.1, ("fp64", "fp32"), True)
    full = run(1.5, ("fp64", "fp32"), False)
    for prec in ("fp64", "fp32"):
        l1o, mo, drift_s, _ = compare(short, "oracle", prec)
        l1f, mf, drift, cups = compare(full, "fp64", prec)
        out[prec] = {"value": cups, "unit": "cell-updates/s", "tfinal": 1.5,
                     "l1_rel_err_vs_fp64_oracle_t0.1": l1o, "mass_rel_diff_vs_fp64_oracle_t0.1": mo,
                     "l1_rel_err_vs_fp64_t1.5": l1f, "mass_rel_diff_vs_fp64_t1.5": mf, "mass_drift_t1.5": drift}
    return out


def serving_leg(scale: str = "small", n_requests: int = 64, batch_us: int = 0) -> dict:
    """A seeded Poisson stream (200 requests/s) of 2D solves, FP64/FP32 mixed.

    "small" is 64 shrunken requests under a 16 GiB budget and 16 slots; "full" is the
    serving configuration itself: requests at the full 2D problem sizes under a 160 GiB
    budget and 32 slots, with level steps of concurrent solves batched across requests
    when batch_us > 0."""
    from amrclaw_b200 import serve
    if scale == "full":
        reqs = serve.synthetic_requests(n_requests, rate=200.0, seed=1, scale="full")
        out = serve.serve(reqs, budget_bytes=160 << 30, slots=32, batch_us=batch_us)["summary"]
    else:
        reqs = serve.synthetic_requests(n_requests, rate=200.0, seed=1, scale="small")
        out = serve.serve(reqs, budget_bytes=16 << 30, slots=16, batch_us=batch_us)["summary"]
    out["scale"] = scale
    return out


def parity_record(state: dict, o, prec: str) -> dict:
    """The value leg's final state against the oracle after the same coarse steps."""
    g, v = o.grids(), o.values()
    same_grids = g.shape == state["grids"].shape and bool(np.array_equal(g, state["grids"]))
    rec = {"against": "oracle (FP64 CPU restatement), same workload, same coarse steps",
           "grids": int(len(state["grids"])), "cells": int(state["values"].size),
           "hierarchy_identical": same_grids, "time_identical": state["time"] == o.time(),
           "cell_updates_identical": state["cells"] == o.cell_updates()}
    if same_grids and v.shape == state["values"].shape:
        diff = int(np.count_nonzero(v != state["values"]))
        rec["values_differing"] = diff
        if prec == "fp32":
            rec["max_rel_err"] = float(np.max(np.abs(v - state["values"]) / np.maximum(np.abs(v), 1e-300)))
    ok = same_grids and rec.get("values_differing") == 0 and rec["time_identical"] and rec["cell_updates_identical"]
    rec["result"] = "bit-identical" if ok else ("hierarchy differs" if not same_grids else "values differ")
    return rec


REFERENCE_BUDGET_S = 120


def run_reference(args, rank):
    """The reference's CPU path: the CPU restatement (the reference Fortran cannot be built here)."""
    if rank != 0:
        return
    rd, cfg, nvar, _, ndim = workload(args.workload)
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        o = oracle_cls(ndim)(d, threads=threads)
        o.run(args.warmup)
        c0 = o.cell_updates()
        # coarse steps one at a time, at most REFERENCE_BUDGET_S of timed host work (the
        # later steps of the hierarchy cost several times the early ones)
        sec, done = 0.0, 0
        while done < args.steps and sec < REFERENCE_BUDGET_S:
            sec += o.run(1)
            done += 1
        cells = o.cell_updates() - c0
        o.close()
    v = cells / sec
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded initial conditions",
            "config": cfg,
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                             "sample": "coarse steps %d..%d of the workload (%d of the %d requested, at most %d s of "
                                       "timed host work), all host threads (OpenMP over patches)" % (
                                 args.warmup, args.warmup + done, done, args.steps, REFERENCE_BUDGET_S)},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="euler3d_blast")
    ap.add_argument("--cpu-steps", type=int, default=0, help="oracle coarse steps timed (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving", default="small", choices=["small", "full", "none"],
                    help="serving leg: 64 shrunken requests (small) or the full-size stream (full)")
    ap.add_argument("--serving-requests", type=int, default=0, help="requests in the serving leg (default 64 small, 512 full)")
    ap.add_argument("--serving-batch-us", type=int, default=0, help="cross-request step batching window of the serving leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    os.environ.setdefault("CUDA_VISIBLE_DEVICES", os.environ.get("CUDA_VISIBLE_DEVICES", ""))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from amrclaw_b200 import Solver, replicas
    rd, cfg, nvar, naux, ndim = workload(args.workload)
    prec = cfg["precision"]
    headline = args.workload == "euler3d_blast"  # the workload the FP64 roof and traffic figures were measured on
    bytes_per_update = (2 * nvar + naux) * (4 if prec == "fp32" else 8)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    with tempfile.TemporaryDirectory() as d:
        rd.write(d)
        # ---------------- process warm-up: one untimed solve over the same coarse steps, so
        # that the timed legs find the device memory pool grown and the kernel modules
        # loaded, as a long-running process does (the first solve of a process otherwise
        # pays page mapping and lazy module loads inside its steps)
        w = Solver(d, batched=True, precision=prec)
        w.run(args.warmup + args.steps)
        w.close()
        # ---------------- batched path (the value)
        s = Solver(d, batched=True, precision=prec)
        s.run(args.warmup)
        s.set_profile(True)
        i0 = s.info()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = Clocks()
        clocks.start()
        ms = 0.0
        cells = 0.0
        torch.cuda.nvtx.range_push("batched_timed")  # the range a launch-list capture selects
        for _ in range(args.steps):
            flush_l2(flush)
            s.run(1)
            inf = s.info()
            ms += inf["last_run_ms"]
            cells += inf["last_run_cells"]
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        i1 = s.info()
        # the state after the timed steps, compared with the oracle over the same steps
        value_state = dict(grids=s.grids(), values=s.values(), time=i1["time"], cells=i1["cell_updates"])
        s.close()
        batched_regrid_ms = 1e3 * (i1["regrid_seconds"] - i0["regrid_seconds"]) / args.steps
        batched_advance_ms = 1e3 * (i1["step_seconds"] - i0["step_seconds"]) / args.steps - batched_regrid_ms
        ms, cells = replicas.combine(ms, cells, dist, device="cuda")
        value = cells / (ms * 1e-3)
        kern_ms = i1["step_kernel_ms"] - i0["step_kernel_ms"]
        kern_cells = i1["step_kernel_cells"] - i0["step_kernel_cells"]
        launches = int(i1["kernels"] - i0["kernels"])
        step_launches = int(i1["substeps"] - i0["substeps"])

        # ---------------- plain per-patch path on the same steps, and both paths replayed
        # from captured CUDA graphs (3D)
        def leg(batched, graphs, schedule=None):
            p = Solver(d, batched=batched, graphs=graphs, schedule=schedule, precision=prec)
            p.run(args.warmup)
            j0 = p.info()
            pms = 0.0
            pcells = 0.0
            for _ in range(args.steps):
                flush_l2(flush)
                p.run(1)
                inf = p.info()
                pms += inf["last_run_ms"]
                pcells += inf["last_run_cells"]
            inf = p.info()
            p.close()
            # host wall time of the steps, split into regrid and the rest (the level substeps)
            inf["regrid_ms_per_step"] = 1e3 * (inf["regrid_seconds"] - j0["regrid_seconds"]) / args.steps
            inf["advance_ms_per_step"] = (1e3 * (inf["step_seconds"] - j0["step_seconds"]) / args.steps
                                          - inf["regrid_ms_per_step"])
            return pcells / (pms * 1e-3), pms / args.steps, inf

        plain_value, plain_ms, plain_inf = leg(False, False)
        graph_legs = {}
        for name, b in (("plain_graphs", False), ("batched_graphs", True)):
            v, m, inf = leg(b, True)
            graph_legs[name] = {"value": v, "unit": "cell-updates/s", "ms_per_step": m,
                                "advance_ms_per_step": inf["advance_ms_per_step"],
                                "graph_captures": inf["graph_captures"], "graph_replays": inf["graph_replays"]}
        if ndim == 3:
            # the other sweep schedules of the batched path (the value leg launches per
            # direction): the persistent work queue, and the per-level autotuner
            tuned = None
            for name, sch in (("batched_work_queue", 2), ("batched_autotune", 0)):
                v, m, inf = leg(True, False, sch)
                graph_legs[name] = {"value": v, "unit": "cell-updates/s", "ms_per_step": m}
                if sch == 0:
                    tuned = {"work_queue": inf["levels_tuned_queue"], "per_direction": inf["levels_tuned_per_direction"]}
            graph_legs["autotune_leg_levels_tuned"] = tuned

        # the clock record spans the timed steps of the value leg and of the legs above (the
        # value leg alone is shorter than nvidia-smi's sampling period)
        clk = clocks.stop()
        clk["span"] = "timed steps of the value, plain, graph and schedule legs"
        # ---------------- end to end through the C ABI: data files in, the whole solve to tfinal,
        # level-1 mass read back after every coarse step, final cell values read back. The
        # process first makes one untimed whole solve, as a long-running one has: the device
        # memory pool then already holds the late steps' level sizes (growing it maps pages,
        # milliseconds per reallocation on some hosts)
        w = Solver(d, batched=True, precision=prec)
        w.run(0)
        w.close()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e = Solver(d, batched=True, precision=prec)
        nstep = 0
        while not e.info()["finished"]:
            e.run(1)
            e.mass()
            nstep += 1
        vals = e.values()
        t1 = time.perf_counter()
        einf = e.info()
        egrids = e.grids()
        e.close()
        e2e_value = einf["cell_updates"] / (t1 - t0)
        h2d = einf["h2d_bytes"]
        d2h = vals.nbytes + 8 * nstep
        # the FP32 form's level-1 L1 error against the FP64 path (bit-identical to the oracle
        # in the parity tests) over the same whole solve
        l1_err = 0.0
        if prec == "fp32":
            from amrclaw_b200 import fields
            dims = tuple(int(x) for x in cfg["base_grid"].split("x"))
            with Solver(d, batched=True) as f64:
                f64.run(0)
                ref = fields.level_array(f64.grids(), f64.values(), nvar, 1, dims)
            got = fields.level_array(egrids, vals, nvar, 1, dims)
            width = [rd.clawdata.upper[k] - rd.clawdata.lower[k] for k in range(ndim)]
            vol = float(np.prod([width[k] / dims[k] for k in range(ndim)]))
            _, rel = fields.l1_error(got, ref, vol)
            l1_err = float(rel.max())

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peak, peak_kind = peaks()
    # the FP32-form and serving legs run with the headline workload (they solve fixed problems of their own)
    fp32 = None
    if headline and not args.no_cpu_baseline:
        rd3, cfg3, _, _, nd3 = workload(args.workload)
        fp32 = fp32_leg(os.cpu_count() or 1, rd3 if nd3 == 3 else None, cfg3)
    os.environ.setdefault("AMRGPU_HOST_THREADS", "2")
    serving = None
    if headline and not args.no_cpu_baseline and args.serving != "none":
        nreq = args.serving_requests or (512 if args.serving == "full" else 64)
        serving = serving_leg(args.serving, nreq, args.serving_batch_us)
    achieved = kern_cells * bytes_per_update / (kern_ms * 1e-3) / 1e9 if kern_ms > 0 else 0.0
    fp64_roof = None
    if headline and kern_ms > 0:
        # the roof that binds this step: FP64 arithmetic, against a DGEMM measured here
        fpk = fp64_peak_tflops()
        ach = kern_cells * FLOPS_PER_CELL_UPDATE_3D / (kern_ms * 1e-3) / 1e12
        fp64_roof = {"achieved": ach, "peak": fpk, "unit": "TFLOP/s", "frac": ach / fpk,
                     "flops_per_cell_update": FLOPS_PER_CELL_UPDATE_3D,
                     "peak_kind": "measured here: FP64 DGEMM 4096^3, best of 5",
                     "note": "built without FMA contraction for bit-exact FP64, so dadd/dmul issue at the dfma rate"}
    cpu = None
    parity = None
    if not args.no_cpu_baseline:
        # the oracle over the value leg's coarse steps: untimed up to the first timed step,
        # then timed over the same steps; its state afterwards is the parity check of the
        # value leg (FP64: bit-identical hierarchy and cell values required)
        threads = os.cpu_count() or 1
        cpu_steps = args.cpu_steps if args.cpu_steps > 0 else args.steps
        with tempfile.TemporaryDirectory() as d:
            rd.write(d)
            o = oracle_cls(ndim)(d, threads=threads)
            o.run(args.warmup)
            c0 = o.cell_updates()
            sec = o.run(cpu_steps)
            cpu_v = (o.cell_updates() - c0) / sec
            if cpu_steps == args.steps:
                parity = parity_record(value_state, o, prec)
            o.close()
        cpu = {"value": cpu_v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
               "sample": "coarse steps %d..%d of the same workload (the value leg's timed steps) on the CPU "
                         "restatement (OpenMP over patches)" % (args.warmup, args.warmup + cpu_steps)}
    line = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if prec == "fp32" else "f64",
        "data": "synthetic: seeded initial conditions of the workload",
        "config": dict(cfg, l2="flushed between steps (256 MB write)", parallelism="replicas" if world > 1 else "single",
                       process_warmup="one untimed solve of the same %d coarse steps before the timed legs" % (args.warmup + args.steps)),
        "advance_ms_per_step": batched_advance_ms, "regrid_ms_per_step": batched_regrid_ms,
        "l1_err_vs_fp64": l1_err,
        "fp32_form": fp32,
        "serving": serving,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": (DRAM_BYTES_PER_CELL_UPDATE_3D * kern_cells / step_launches
                                 if headline and step_launches else None),
                     "traffic_note": "DRAM bytes per level substep of the step kernels: ncu bytes per cell-update "
                                     "of a level-1 substep times the average cells of a timed substep",
                     "kernel": "sweep3<1..3> + face3 + update3" if ndim == 3 else "step2 sweeps + update",
                     "peak_kind": peak_kind,
                     "bytes_per_cell_update": bytes_per_update,
                     "algorithmic_bytes_per_launch": (bytes_per_update * kern_cells / step_launches
                                                      if step_launches else None),
                     "fp64": fp64_roof},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": int(h2d) // max(1, nstep),
                "d2h_bytes_per_step": d2h // max(1, nstep), "seconds": t1 - t0, "coarse_steps": nstep,
                "cell_updates": einf["cell_updates"],
                "includes": "init from data files, initial upload, all %d coarse steps to tfinal with a mass read-back "
                            "after each, final values download; the process made one untimed whole solve "
                            "before it" % nstep},
        "gpu_launches": launches,
        "level_substeps": step_launches,
        "clocks": clk,
        "parity": parity,
        # last, so that a reader that keeps only the tail of the line still sees them
        "schedules": graph_legs or None,
        "plain": {"value": plain_value, "unit": "cell-updates/s", "ms_per_step": plain_ms,
                  "speedup_batched_over_plain": value / plain_value if plain_value else None,
                  "advance_ms_per_step": plain_inf["advance_ms_per_step"],
                  "regrid_ms_per_step": plain_inf["regrid_ms_per_step"],
                  "advance_speedup_batched_over_plain": (plain_inf["advance_ms_per_step"] / batched_advance_ms
                                                         if batched_advance_ms > 0 else None)},
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
