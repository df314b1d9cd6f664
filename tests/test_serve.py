"""Serving loop: admission by slots and HBM budget (CPU, fake solves), and on the GPU the
same result for a solve alone and in a concurrent mix (bit-identical, FP64)."""
import threading
import time

import numpy as np
import pytest

from amrclaw_b200 import serve


def test_synthetic_stream_is_seeded_and_shaped():
    a = serve.synthetic_requests(40, rate=200.0, seed=3, scale="full")
    b = serve.synthetic_requests(40, rate=200.0, seed=3, scale="full")
    assert [(r.kind, r.n, r.levels, r.ratio, r.tfinal, r.precision) for r in a] == \
           [(r.kind, r.n, r.levels, r.ratio, r.tfinal, r.precision) for r in b]
    assert all(32 <= r.n <= 256 and r.n % 2 == 0 and 2 <= r.levels <= 4 and r.ratio in (2, 4) for r in a)
    assert all(0.1 <= r.tfinal <= 1.0 for r in a)
    arr = [r.arrival for r in a]
    assert arr == sorted(arr) and 0.05 < arr[-1] < 0.6  # 40 arrivals at 200/s
    assert {r.kind for r in a} == {"advection", "euler", "acoustics"}


def test_admission_respects_slots_and_budget():
    reqs = serve.synthetic_requests(24, rate=2000.0, seed=5, scale="small")
    live = {"n": 0, "max": 0, "bytes": 0, "max_bytes": 0}
    mu = threading.Lock()

    def fake(req, keep):
        with mu:
            live["n"] += 1; live["max"] = max(live["max"], live["n"])
            live["bytes"] += req.est_bytes(); live["max_bytes"] = max(live["max_bytes"], live["bytes"])
        time.sleep(0.02)
        with mu:
            live["n"] -= 1; live["bytes"] -= req.est_bytes()
        return float(req.n * req.n), 1.0, None, 1.0, 0.0

    budget = 3 * max(r.est_bytes() for r in reqs)
    out = serve.serve(reqs, budget_bytes=budget, slots=4, runner=fake)
    s = out["summary"]
    assert s["completed"] == 24 and s["failed"] == 0
    assert live["max"] <= 4 and s["peak_concurrent"] <= 4
    assert live["max_bytes"] <= budget
    assert s["p99_latency_ms"] >= s["p50_latency_ms"] > 0
    assert [r.rid for r in out["results"]] == list(range(24))


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix():
    reqs = serve.synthetic_requests(6, rate=1000.0, seed=7, scale="small")
    for r in reqs:
        r.n = min(r.n, 40); r.n -= r.n % 2; r.tfinal = min(r.tfinal, 0.08)
    alone = {r.rid: serve.run_one(r, keep_values=True) for r in reqs}
    out = serve.serve(reqs, budget_bytes=1 << 34, slots=6, keep_values=True)
    assert out["summary"]["completed"] == len(reqs)
    assert out["summary"]["peak_concurrent"] >= 2
    for res in out["results"]:
        cells, mass, vals, _, _ = alone[res.rid]
        assert res.cell_updates == cells
        np.testing.assert_array_equal(res.values, vals)
