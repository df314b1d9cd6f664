"""Serving loop: independent AMR solves admitted by HBM budget, run concurrently.

Each admitted request gets its own context (device pool, CUDA stream) driven by its own
host thread; the C library releases the interpreter while it works, so the level steps
of all admitted solves are in flight on the device together and overlap there. A
request waits in arrival order until both a slot and its reserved device memory are
free; finished solves release both. Each context's pools are capped at the request's
reservation (amrgpu_set_pool_limit), so the budget holds: a solve that would outgrow
its reservation stops with AMRGPU_ENOMEM, gives its reservation back and waits again,
first in line, with twice the reservation (at most the whole budget). Latency is
completion time minus arrival time.

    python -m amrclaw_b200.serve [--requests N] [--rate R] [--budget-gb G] [--slots S] [--scale small|full] [--batch-us W]

prints one JSON line: p50/p99 latency, aggregate cell-updates/s, makespan, admissions.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import problems
from .replicas import percentiles

KINDS = ("advection", "euler", "acoustics")
ENOMEM = 3  # AMRGPU_ENOMEM


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the stream
    kind: str               # advection | euler | acoustics
    n: int                  # base grid n x n
    levels: int
    ratio: int
    tfinal: float
    precision: str          # "fp64" or "fp32" (the FP32 form)
    params: dict = field(default_factory=dict)
    reserve: int = 0        # device bytes reserved at admission (0: est_bytes())
    retries: int = 0        # admissions after a pool-cap stop

    def rundata(self):
        if self.kind == "advection":
            return problems.advection_square(self.n, self.levels, self.ratio, self.tfinal, **self.params)
        if self.kind == "euler":
            return problems.euler_quadrants(self.n, self.levels, self.ratio, self.tfinal, **self.params)
        return problems.acoustics_pulse(self.n, self.levels, self.ratio, self.tfinal, **self.params)

    def nvar(self) -> int:
        return {"advection": 1, "euler": 4, "acoustics": 3}[self.kind]

    def est_bytes(self) -> int:
        """Device memory reserved for admission: the context's initial patch pool (sized in
        doubles in both precisions: eight arrays of the enlarged base grid per level, and
        4 Mi doubles), its register pool (1 Mi doubles) and room for growth."""
        pool = 8 * (self.nvar() * (self.n + 4) ** 2 * 8 * self.levels + (1 << 22))
        return int(pool + 8 * (1 << 20) + (24 << 20))

    def reservation(self) -> int:
        return self.reserve or self.est_bytes()


def synthetic_requests(n: int = 512, rate: float = 200.0, seed: int = 1, scale: str = "small") -> List[Request]:
    """A seeded Poisson stream of independent solves.

    scale "full": base grids 32^2-256^2 (log-uniform), 2-4 levels, ratio 2 or 4, final
    times 0.1-1.0 (the serving configuration as stated). scale "small": 32^2-96^2, 2-3
    levels, ratio 2, final times 0.05-0.2, for runs that finish in seconds. Problems are
    drawn uniformly from advection, Euler quadrants and acoustics, each with a seeded
    perturbation of its parameters; precision is fp64/fp32 with equal odds."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        kind = KINDS[int(rng.integers(0, 3))]
        if scale == "full":
            nb = int(round(math.exp(rng.uniform(math.log(32), math.log(256))) / 2)) * 2
            levels = int(rng.integers(2, 5)); ratio = int(rng.choice([2, 4])); tfinal = float(rng.uniform(0.1, 1.0))
        else:
            nb = int(round(math.exp(rng.uniform(math.log(32), math.log(96))) / 2)) * 2
            levels = int(rng.integers(2, 4)); ratio = 2; tfinal = float(rng.uniform(0.05, 0.2))
        prec = "fp32" if rng.uniform() < 0.5 else "fp64"
        if kind == "advection":
            x0 = float(rng.uniform(0.05, 0.3)); y0 = float(rng.uniform(0.05, 0.3))
            params = dict(u=float(rng.uniform(0.3, 0.7)), v=float(rng.uniform(0.7, 1.2)), x0=x0, x1=x0 + 0.4, y0=y0, y1=y0 + 0.4)
        elif kind == "euler":
            params = dict(xs=float(rng.uniform(0.6, 0.85)), ys=float(rng.uniform(0.6, 0.85)))
        else:
            params = dict(r0=float(rng.uniform(0.2, 0.4)), width=float(rng.uniform(0.04, 0.08)))
        out.append(Request(rid, t, kind, nb, levels, ratio, tfinal, prec, params))
    return out


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    done: float
    cell_updates: float
    mass: float
    values: Optional[np.ndarray]
    device_ms: float
    pool_peak_bytes: float
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def run_one(req: Request, keep_values: bool = False, batch_us: int = 0):
    """One solve from start to tfinal on the current device, in the request's precision, its
    pools capped at the request's reservation: (cell updates, mass, values, device ms, pool
    peak). batch_us > 0: its level steps go out in shared launches with those of the other
    solves of the same plugin and precision running meanwhile (amrgpu_set_step_batching)."""
    from . import AmrError, Solver
    with Solver(req.rundata(), batched=True, precision=req.precision, step_batching_us=batch_us) as s:
        # the pools a new context starts with can already exceed a small reservation: that
        # is the same outcome as outgrowing it (readmission with twice the reservation)
        held = int(s.info()["pool_bytes"])
        if req.reservation() < held:
            raise AmrError("reservation of %d bytes is below the %d bytes the new context's pools hold"
                           % (req.reservation(), held), ENOMEM)
        s.set_pool_limit(req.reservation())
        s.run(0)
        inf = s.info()
        vals = s.values() if keep_values else None
        STEP_BATCH_STATS.add(inf)
        return inf["cell_updates"], s.mass(), vals, inf["last_run_ms"], inf["pool_peak_bytes"]


class _BatchStats:
    """Level steps the solves of this process submitted to the step batcher, how many of
    them shared their launch with another solve, and the members those launches carried."""

    def __init__(self):
        self.mu = threading.Lock()
        self.reset()

    def reset(self):
        self.submits = self.shared = self.members = 0.0

    def add(self, inf: dict):
        with self.mu:
            self.submits += inf.get("step_batch_submits", 0.0)
            self.shared += inf.get("step_batch_shared", 0.0)
            self.members += inf.get("step_batch_members", 0.0)

    def summary(self) -> dict:
        with self.mu:
            return {"level_steps_submitted": int(self.submits), "level_steps_in_shared_launches": int(self.shared),
                    "mean_solves_per_launch": self.members / self.submits if self.submits else 0.0}


STEP_BATCH_STATS = _BatchStats()


def serve(requests: List[Request], budget_bytes: int, slots: int, keep_values: bool = False,
          clock: Callable[[], float] = time.perf_counter, runner: Optional[Callable] = None,
          batch_us: int = 0) -> dict:
    """Admit the requests as they arrive (arrival times relative to the call), run them
    concurrently, return the per-request results and the summary. `runner(req, keep_values)`
    performs one solve (default run_one: the device path in the request's precision, with
    cross-request step batching when batch_us > 0)."""
    if runner is None:
        STEP_BATCH_STATS.reset()
        runner = lambda req, keep: run_one(req, keep, batch_us)  # noqa: E731
    pending = sorted(requests, key=lambda r: r.arrival)
    waiting: List[Request] = []
    results: List[Result] = []
    lock = threading.Condition()
    state = {"used": 0, "active": 0, "peak_active": 0, "peak_used": 0, "pool_retries": 0}
    t0 = clock()

    def worker(req: Request, admitted: float, est: int):
        err = None
        cells = mass = dev_ms = peak = 0.0
        vals = None
        retry = False
        try:
            cells, mass, vals, dev_ms, peak = runner(req, keep_values)
        except Exception as e:  # reported per request; the server keeps going
            err = str(e)
            # AMRGPU_ENOMEM: the solve outgrew its reservation; readmit with twice as much
            retry = getattr(e, "code", None) == ENOMEM and est < budget_bytes
        done = clock() - t0
        with lock:
            state["used"] -= est
            state["active"] -= 1
            if retry:
                req.reserve = min(2 * est, budget_bytes)
                req.retries += 1
                state["pool_retries"] += 1
                waiting.insert(0, req)
            else:
                results.append(Result(req.rid, req.arrival, admitted, done, cells, mass, vals, dev_ms, peak, err))
            lock.notify_all()

    threads = []
    with lock:
        while pending or waiting or state["active"]:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.pop(0))
            # FIFO admission: the oldest waiting request first, while slot and memory allow
            while waiting and state["active"] < slots:
                est = waiting[0].reservation()
                if state["used"] + est > budget_bytes and state["active"] > 0:
                    break
                req = waiting.pop(0)
                state["used"] += est
                state["active"] += 1
                state["peak_active"] = max(state["peak_active"], state["active"])
                state["peak_used"] = max(state["peak_used"], state["used"])
                th = threading.Thread(target=worker, args=(req, now, est), daemon=True)
                th.start()
                threads.append(th)
            wait = 0.05
            if pending:
                wait = max(0.0, min(wait, pending[0].arrival - (clock() - t0)))
            lock.wait(timeout=wait)
    for th in threads:
        th.join()
    makespan = clock() - t0
    ok = [r for r in results if r.error is None]
    lat = [r.latency for r in ok]
    p50, p99 = percentiles(lat, (50, 99))
    cells = sum(r.cell_updates for r in ok)
    summary = {
        "requests": len(requests), "completed": len(ok), "failed": len(results) - len(ok),
        "p50_latency_ms": 1e3 * p50, "p99_latency_ms": 1e3 * p99, "makespan_s": makespan,
        "cell_updates": cells, "throughput_cell_updates_per_s": cells / makespan if makespan > 0 else 0.0,
        "peak_concurrent": state["peak_active"], "peak_reserved_bytes": state["peak_used"],
        "budget_bytes": budget_bytes, "slots": slots, "pool_retries": state["pool_retries"],
        "fp32_requests": sum(1 for r in requests if r.precision == "fp32"),
        "step_batching_window_us": batch_us,
    }
    if batch_us:
        summary["step_batching"] = STEP_BATCH_STATS.summary()
    return {"summary": summary, "results": sorted(results, key=lambda r: r.rid)}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--scale", default="small", choices=["small", "full"])
    ap.add_argument("--budget-gb", type=float, default=16.0)
    ap.add_argument("--slots", type=int, default=16)
    ap.add_argument("--batch-us", type=int, default=0,
                    help="cross-request step batching window in microseconds (0: each solve launches alone)")
    args = ap.parse_args(argv)
    os.environ.setdefault("AMRGPU_HOST_THREADS", "2")
    reqs = synthetic_requests(args.requests, args.rate, args.seed, args.scale)
    out = serve(reqs, int(args.budget_gb * (1 << 30)), args.slots, batch_us=args.batch_us)
    s = out["summary"]
    s.update({"scale": args.scale, "rate_per_s": args.rate, "seed": args.seed,
              "mix": {k: sum(1 for r in reqs if r.kind == k) for k in KINDS}})
    print(json.dumps(s), flush=True)


if __name__ == "__main__":
    main()
