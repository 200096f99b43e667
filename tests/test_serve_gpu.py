"""Serving loop: results are the same alone and in a mix (continuous batching with joins and
leaves between chunks), memory admission holds requests back until the pool frees, and a
real-time Poisson run serves everything with latency percentiles."""
import pytest

from mcstreamer_b200 import jumc, lxcat
from mcstreamer_b200.serve import (BYTES_PER_SLOT, StopRule, SwarmRequest, SwarmServer, percentiles,
                                   poisson_requests, serial_latencies)

DENS = 2.5e25
DT = 1e-13
RULE = StopRule(rel=0.05, min_steps=20, block=5, min_blocks=4, max_steps=160)


@pytest.fixture(scope="module")
def tables(ctx):
    tabs = [jumc.CollisionTable(lxcat.synthetic_table(v), ctx) for v in (0, 1, 2, 3)]
    yield tabs
    for t in tabs:
        t.close()


def _reqs():
    return [SwarmRequest(0, 1, 900.0, 3000, 11, 0.0), SwarmRequest(1, 0, 400.0, 1500, 12, 0.0),
            SwarmRequest(2, 3, 30.0, 2500, 13, 0.0), SwarmRequest(3, 2, 700.0, 5000, 14, 0.0),
            SwarmRequest(4, 1, 150.0, 800, 15, 0.0)]


def _key(r):
    return (r.rid, r.steps, r.k_ion, r.k_ion_err3, r.settled, r.drift, r.mean_energy)


@pytest.mark.gpu
def test_result_same_alone_and_in_mix(ctx, tables):
    mixed = SwarmServer(ctx, tables, DT, DENS, budget_bytes=64e6, rule=RULE, max_instances=8, chunk=7)
    try:
        got = mixed.run(_reqs(), realtime=False)
    finally:
        mixed.close()
    assert [r.rid for r in got] == [0, 1, 2, 3, 4]
    assert any(r.k_ion > 0 for r in got)
    for req, r in zip(_reqs(), got):
        alone = SwarmServer(ctx, tables, DT, DENS, budget_bytes=16e6, rule=RULE, max_instances=2, chunk=16)
        try:
            (a,) = alone.run([req], realtime=False)
        finally:
            alone.close()
        assert _key(a) == _key(r)


@pytest.mark.gpu
def test_memory_admission_waits_for_room(ctx, tables):
    reqs = _reqs()
    # pool for about two of the largest requests at once
    budget = 2.2 * 2 * 5000 * BYTES_PER_SLOT
    srv = SwarmServer(ctx, tables, DT, DENS, budget_bytes=budget, rule=RULE, max_instances=8, chunk=8)
    peak = [0]
    try:
        def watch(_):
            peak[0] = max(peak[0], srv.pool_slots - srv.free_slots)
        got = srv.run(reqs, realtime=False, on_response=watch)
    finally:
        srv.close()
    assert len(got) == len(reqs)
    assert max(r.admitted for r in got) >= min(r.finished for r in got)   # someone waited for a leave
    assert peak[0] <= srv.pool_slots


@pytest.mark.gpu
def test_realtime_poisson_run(ctx, tables):
    reqs = poisson_requests(40.0, 0.5, seed=4, n_range=(512, 4096))
    srv = SwarmServer(ctx, tables, DT, DENS, budget_bytes=256e6, rule=RULE, max_instances=64, chunk=16)
    try:
        got = srv.run(reqs)
    finally:
        srv.close()
    assert len(got) == len(reqs)
    lat = [r.latency for r in got]
    assert min(lat) > 0
    p = percentiles(lat)
    assert p["p50"] <= p["p95"] <= p["p99"]
    ser = serial_latencies([r.arrival for r in got], [0.01] * len(got))
    assert (ser >= 0.01 - 1e-12).all()
