"""Host logic of the serving driver (no GPU): the Poisson schedule and the
latency / throughput summary."""
import numpy as np

from kc_cuda_b200 import serving


def test_poisson_schedule_is_seeded_and_has_the_rate():
    a = serving.poisson_arrivals(20000, rate=50.0, seed=5)
    b = serving.poisson_arrivals(20000, rate=50.0, seed=5)
    assert np.array_equal(a, b)
    assert a[0] == 0.0 and np.all(np.diff(a) >= 0)
    gaps = np.diff(a)
    assert abs(gaps.mean() - 1 / 50.0) < 0.05 / 50.0 * 4  # mean gap within a few standard errors
    # Exponential gaps: coefficient of variation near 1.
    assert 0.9 < gaps.std() / gaps.mean() < 1.1
    assert not np.array_equal(a, serving.poisson_arrivals(20000, rate=50.0, seed=6))


def test_percentiles_match_numpy():
    v = np.random.default_rng(1).exponential(3.0, size=1001)
    assert serving.percentile(v, 50) == np.percentile(v, 50)
    assert serving.percentile(v, 99) == np.percentile(v, 99)
    assert np.isnan(serving.percentile([], 50))


def test_summary_throughput_and_latencies():
    submitted = [(i, 10.0 + 0.5 * i) for i in range(4)]
    results = [{"ms_latency": 100.0 * (i + 1), "ms_wait": 1.0, "wave": i // 2, "wave_graphs": 2} for i in range(4)]
    s = serving.summarize(submitted, results)
    # Last result at 10 + 1.5 + 0.4 s; span from 10 s.
    assert abs(s["span_s"] - 1.9) < 1e-9
    assert abs(s["graphs_per_s"] - 4 / 1.9) < 1e-9
    assert s["p50_ms"] == 250.0
    assert s["waves"] == 2 and s["mean_wave_graphs"] == 2.0


def test_drive_submits_in_order_on_schedule():
    seen = []
    out = serving.drive([0.0, 0.01, 0.02], lambda i: seen.append(i) or 100 + i)
    assert seen == [0, 1, 2]
    assert [r for r, _ in out] == [100, 101, 102]
    ts = [t for _, t in out]
    assert ts[2] - ts[0] >= 0.02 - 1e-3
