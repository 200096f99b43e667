"""Host logic of the serving loop (no GPU): the stopping rule decides at the same step
whatever the chunking, the serial-server latency model, and the seeded request stream."""
import numpy as np

from mcstreamer_b200.serve import StopRule, percentiles, poisson_requests, serial_latencies


def _decide_in_chunks(rule, nu, chunk):
    T = rule.first_check()
    for end in range(chunk, len(nu) + chunk, chunk):
        out = rule.evaluate(nu[:min(end, len(nu))], T)
        T = out[4]
        if out[0] > 0:
            return out[:4]
    return None


def test_stop_step_is_independent_of_chunking():
    rng = np.random.default_rng(1)
    rule = StopRule(rel=0.01, min_steps=50, block=10, min_blocks=5, max_steps=3000)
    for scale in (0.02, 0.05, 0.2):
        nu = 1e9 * (1.0 + scale * rng.standard_normal(4000))
        ref = _decide_in_chunks(rule, nu, 1)
        for chunk in (3, 7, 16, 64):
            assert _decide_in_chunks(rule, nu, chunk) == ref


def test_zero_rate_settles_and_cap_bounds():
    rule = StopRule(min_steps=20, block=5, min_blocks=4, max_steps=100)
    T, k, err, settled, _ = rule.evaluate(np.zeros(60))
    assert (T, k, err, settled) == (40, 0.0, 0.0, True)
    rng = np.random.default_rng(2)
    noisy = np.abs(rng.standard_normal(150))
    T, k, err, settled, _ = rule.evaluate(noisy)
    assert T == 100 and not settled and err > 0.01 * k


def test_block_means_error():
    rule = StopRule(min_steps=0, block=4, min_blocks=2)
    nu = np.repeat([1.0, 3.0, 1.0, 3.0], 4)
    k, err = rule.stats(nu)
    assert k == 2.0
    assert np.isclose(err, 3 * np.std([1, 3, 1, 3], ddof=1) / 2)


def test_serial_latencies_fifo():
    lat = serial_latencies([0.0, 0.5, 0.6, 10.0], [1.0, 1.0, 1.0, 1.0])
    np.testing.assert_allclose(lat, [1.0, 1.5, 2.4, 1.0])
    p = percentiles(lat)
    assert p["p50"] <= p["p95"] <= p["p99"] <= 2.4


def test_poisson_requests_seeded():
    a = poisson_requests(200.0, 2.0, seed=4)
    b = poisson_requests(200.0, 2.0, seed=4)
    assert [(r.arrival, r.n, r.en_td, r.gas, r.seed) for r in a] == [(r.arrival, r.n, r.en_td, r.gas, r.seed) for r in b]
    assert 300 < len(a) < 500
    assert all(1024 <= r.n <= 2_097_152 and 10.0 <= r.en_td <= 1000.0 and 0 <= r.gas < 4 for r in a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
