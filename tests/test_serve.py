"""Continuous-batching server: admission by HBM budget, overlap of requests, results
equal to each simulation run alone (bit-exact: the batched kernels compute every cell
with the same operations whatever else shares the launch)."""
from __future__ import annotations

import numpy as np
import pytest

from fire_b200 import _abi as A
from fire_b200.serve import FireXServer, Request, poisson_stream
from fire_b200.sim import FireXSim, make_options, planned_device_bytes


def _req(dims, steps, seed, arrival=0.0, P=12, R=10):
    X, Y, Z = dims
    r = max(2.0, X / 8)
    opts = dict(pressure_iterations=P, correction_iterations=R, seed=seed, velocity_noise=0.05, emission_jitter=0.1,
                spheres=[dict(center=(X / 2, Y / 10 + r, Z / 2), radius=r, fuel=1.0, temperature=1500.0)])
    return Request(dims=dims, steps=steps, options=opts, arrival=arrival, keep=("flow", "species", "pressure"))


def test_poisson_stream_is_seeded_and_bounded():
    fam = [(64, 96, 64), (96, 144, 96)]
    a = poisson_stream(40.0, 2.0, fam, (60, 600), seed=5)
    b = poisson_stream(40.0, 2.0, fam, (60, 600), seed=5)
    assert [(r.dims, r.steps, r.arrival) for r in a] == [(r.dims, r.steps, r.arrival) for r in b]
    assert 40 <= len(a) <= 120  # 80 expected
    assert all(0 < r.arrival <= 2.0 and 60 <= r.steps <= 600 and r.dims in fam for r in a)
    assert all(a[i].arrival < a[i + 1].arrival for i in range(len(a) - 1))


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [A.PRECISION_F32, A.PRECISION_MIXED])
def test_each_request_equals_its_run_alone(precision):
    reqs = [_req((32, 48, 32), 5, 1), _req((48, 64, 40), 3, 2, arrival=0.0), _req((16, 20, 24), 7, 3),
            _req((64, 96, 64), 4, 4)]
    srv = FireXServer(precision=precision)
    ids = [srv.submit(r) for r in reqs]
    # a late request joins while the others run
    srv.tick()
    ids.append(srv.submit(_req((32, 40, 24), 3, 9)))
    reqs.append(_req((32, 40, 24), 3, 9))
    while srv.tick():
        pass
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["ticks"] == 7
    assert st["p50_step_ms"] is not None and st["p99_step_ms"] >= st["p50_step_ms"]
    for rid, r in zip(ids, reqs):
        res = srv.poll(rid)
        assert res["status"] == "done"
        alone = FireXSim(r.dims, make_options(**{**r.options, "precision": precision}))
        alone.step(r.steps, r.dt)
        for f in r.keep:
            assert np.array_equal(res["fields"][f], alone.read(f)), (r.dims, f)
        alone.close()
    srv.close()


@pytest.mark.gpu
def test_admission_waits_for_memory_and_rejects_oversize():
    a, b = _req((64, 96, 64), 3, 1), _req((64, 96, 64), 2, 2)
    need = planned_device_bytes(a.dims, make_options(**{**a.options, "precision": A.PRECISION_MIXED}))
    srv = FireXServer(budget_bytes=int(need * 1.5))  # room for one at a time
    ia, ib = srv.submit(a), srv.submit(b)
    big = srv.submit(_req((512, 512, 512), 1, 3))
    assert srv.poll(big)["status"] == "rejected"
    srv.tick()
    assert srv.poll(ia)["status"] == "running" and srv.poll(ib)["status"] == "queued"
    while srv.tick():
        pass
    assert srv.poll(ia)["status"] == "done" and srv.poll(ib)["status"] == "done"
    assert srv.poll(ib)["queue_wait_s"] > 0.0
    assert srv.used == 0 and len(srv.batch) == 0
    srv.close()


def test_tick_budget_bounds_the_estimated_tick():
    from fire_b200.serve import FIXED_SWEEP_EQUIVALENTS, TickBudget
    tb = TickBudget(target_ms=10.0, initial_rate=1e6)
    opts = make_options(pressure_iterations=20, correction_iterations=10)
    w = TickBudget.work((10, 10, 10), opts)
    assert w == 1000 * (30 + FIXED_SWEEP_EQUIVALENTS)
    assert tb.fits(0.0, 1e12, members=0)  # an empty batch always takes the oldest request
    assert tb.fits(0.0, 5e6, members=1) and not tb.fits(6e6, 5e6, members=1)
    tb.observe(1e7, 5.0)  # measured 2e6 per ms: the estimate moves toward it
    assert 1e6 < tb.rate < 2e6
    for _ in range(50):
        tb.observe(1e7, 5.0)
    assert tb.rate == pytest.approx(2e6, rel=1e-6)
    assert tb.fits(1e7, 0.9e7, members=3) and not tb.fits(1e7, 1.1e7, members=3)


@pytest.mark.gpu
def test_tick_target_admits_by_work_and_results_stay_exact():
    """A tick target below one member's work admits one request per tick-batch: every tick
    steps a single member, requests wait in the queue and each result equals its run alone."""
    reqs = [_req((32, 48, 32), 3, 11), _req((16, 20, 24), 2, 12), _req((32, 40, 24), 2, 13)]
    srv = FireXServer(tick_target_ms=1e-6)
    ids = [srv.submit(r) for r in reqs]
    members = []
    while True:
        srv._admit()
        members.append(len(srv.slots))
        if not srv.tick():
            break
    assert max(members) == 1
    st = srv.stats()
    assert st["completed"] == 3 and st["ticks"] == 7
    assert st["p50_latency_s"] is not None and st["p99_latency_s"] >= st["p50_latency_s"]
    for rid, r in zip(ids, reqs):
        res = srv.poll(rid)
        alone = FireXSim(r.dims, make_options(**{**r.options, "precision": A.PRECISION_MIXED}))
        alone.step(r.steps, r.dt)
        for f in r.keep:
            assert np.array_equal(res["fields"][f], alone.read(f)), (r.dims, f)
        alone.close()
    srv.close()
