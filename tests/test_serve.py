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


def test_pool_cap_stop_readmits_with_twice_the_reservation():
    """A solve that outgrows its reservation (the library's AMRGPU_ENOMEM under the pool
    cap) gives the reservation back and is admitted again, first in line, with twice as
    much; the reserved total never passes the budget and the accounting returns to zero."""
    from amrclaw_b200 import AmrError
    reqs = serve.synthetic_requests(12, rate=2000.0, seed=9, scale="small")
    need = {r.rid: (2 if r.rid % 3 == 0 else 1) * r.est_bytes() for r in reqs}
    seen = {}
    live = {"bytes": 0, "max": 0}
    mu = threading.Lock()

    def fake(req, keep):
        with mu:
            seen.setdefault(req.rid, []).append(req.reservation())
            live["bytes"] += req.reservation(); live["max"] = max(live["max"], live["bytes"])
        try:
            time.sleep(0.01)
            if req.reservation() < need[req.rid]:
                raise AmrError("amrgpu_run failed: device pool limit reached", serve.ENOMEM)
            return float(req.n * req.n), 1.0, None, 1.0, float(need[req.rid])
        finally:
            with mu:
                live["bytes"] -= req.reservation()

    budget = 6 * max(r.est_bytes() for r in reqs)
    out = serve.serve(reqs, budget_bytes=budget, slots=4, runner=fake)
    s = out["summary"]
    assert s["completed"] == 12 and s["failed"] == 0
    assert s["pool_retries"] == sum(1 for r in reqs if r.rid % 3 == 0)
    for r in reqs:
        e = r.est_bytes()
        assert seen[r.rid] == ([e, 2 * e] if r.rid % 3 == 0 else [e])
    assert live["max"] <= budget and live["bytes"] == 0


def test_pool_cap_stop_is_final_at_the_whole_budget():
    from amrclaw_b200 import AmrError
    reqs = serve.synthetic_requests(2, rate=2000.0, seed=2, scale="small")

    def fake(req, keep):
        raise AmrError("amrgpu_run failed: device pool limit reached", serve.ENOMEM)

    out = serve.serve(reqs, budget_bytes=4 * max(r.est_bytes() for r in reqs), slots=2, runner=fake)
    s = out["summary"]
    assert s["failed"] == 2 and s["completed"] == 0
    assert all(r.error and "pool limit" in r.error for r in out["results"])


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


@pytest.mark.gpu
def test_pool_cap_stops_a_solve_with_enomem():
    """amrgpu_set_pool_limit: a cap below what the pools hold is refused (EINVAL); a cap at
    what they hold makes the first growth of a refining run stop with AMRGPU_ENOMEM."""
    from amrclaw_b200 import AmrError, Solver, problems
    rd = problems.euler_quadrants(64, levels=3, ratio=4, tfinal=0.02)
    # level 3 everywhere from t = 0.005: the first regrid after that outgrows the pools
    rd.regiondata.regions = [[3, 3, 0.005, 1e9, 0.0, 1.0, 0.0, 1.0]]
    with Solver(rd) as s:
        held = int(s.info()["pool_bytes"])
        assert held > 0
        with pytest.raises(AmrError) as e:
            s.set_pool_limit(held - 8)
        assert e.value.code == 2
        s.set_pool_limit(held)
        with pytest.raises(AmrError) as e:
            s.run(0)
        assert e.value.code == serve.ENOMEM and "pool limit" in str(e.value)
    with Solver(rd, pool_limit=1 << 34) as s:  # a roomy cap changes nothing
        s.run(0)
        assert s.info()["finished"] == 1.0


@pytest.mark.gpu
def test_cross_request_step_batching_identical_alone_and_in_the_mix():
    """Level steps of concurrent solves of the same plugin and precision go out in shared
    launches (step2_batch_kernel); every result is bit-identical to the solve run alone."""
    reqs = serve.synthetic_requests(8, rate=100000.0, seed=11, scale="small")
    for k, r in enumerate(reqs):
        r.kind = "euler" if k % 2 == 0 else "acoustics"
        r.params = {}
        r.precision = "fp64" if k % 2 == 0 else "fp32"
        r.n = 32 + 4 * (k // 2); r.levels = 2; r.ratio = 2; r.tfinal = 0.06
    alone = {r.rid: serve.run_one(r, keep_values=True) for r in reqs}
    out = serve.serve(reqs, budget_bytes=1 << 34, slots=8, keep_values=True, batch_us=3000)
    s = out["summary"]
    assert s["completed"] == len(reqs)
    st = s["step_batching"]
    assert st["level_steps_submitted"] > 0
    assert st["level_steps_in_shared_launches"] > 0 and st["mean_solves_per_launch"] > 1.0
    for res in out["results"]:
        cells, mass, vals, _, _ = alone[res.rid]
        assert res.cell_updates == cells
        np.testing.assert_array_equal(res.values, vals)


@pytest.mark.gpu
def test_step_batching_refuses_bad_windows_and_3d():
    import configs
    from amrclaw_b200 import AmrError, Solver, problems
    with Solver(problems.acoustics_pulse(32, levels=2, ratio=2, tfinal=0.02)) as s:
        with pytest.raises(AmrError) as e:
            s.set_step_batching(-1)
        assert e.value.code == 2
        s.set_step_batching(100)
        s.set_step_batching(0)
        s.run(0)
    with Solver(configs.euler_blast(n=8, levels=1, tfinal=0.01, max1d=8)) as s3:
        with pytest.raises(AmrError) as e:
            s3.set_step_batching(100)
        assert e.value.code == 2
