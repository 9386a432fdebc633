"""Host driver for the serving loop (kt_server_*): Poisson arrivals, result
collection and latency summaries.

The serving workload is requests drawn from the batched mix (graph i of the
mix for request i), arriving as a Poisson process at a fixed rate with a fixed
seed; a request's latency is measured by the library from its submission to
its result (kt_request_result.ms_latency).
"""
from __future__ import annotations

import time
from typing import Callable, Dict, List, Sequence

import numpy as np


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times (seconds from the first request) of n requests of a
    Poisson process with `rate` requests/s: cumulative exponential gaps, the
    first request at 0."""
    if n <= 0:
        return np.zeros(0)
    if rate <= 0:
        raise ValueError("rate must be positive")
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, size=n)
    gaps[0] = 0.0
    return np.cumsum(gaps)


def drive(arrivals: Sequence[float], submit: Callable[[int], int]) -> List[tuple]:
    """Submits request i at arrivals[i] (host clock); returns (request id,
    submission time) pairs.  A late submission is sent at once, so the
    schedule is kept on average."""
    out = []
    t0 = time.perf_counter()
    for i, t in enumerate(arrivals):
        d = t0 + float(t) - time.perf_counter()
        if d > 0:
            time.sleep(d)
        ts = time.perf_counter()
        out.append((submit(i), ts))
    return out


def percentile(values: Sequence[float], q: float) -> float:
    """q-th percentile (0..100) by linear interpolation between order
    statistics (numpy's default)."""
    if len(values) == 0:
        return float("nan")
    return float(np.percentile(np.asarray(values, dtype=np.float64), q))


def summarize(submitted: Sequence[tuple], results: Sequence[dict]) -> Dict[str, float]:
    """Latency percentiles and throughput of a served run.  Throughput is
    completed requests over the span from the first submission to the last
    result (each result's time = its submission + its latency)."""
    lat = [r["ms_latency"] for r in results]
    waits = [r["ms_wait"] for r in results]
    t_first = min(ts for _, ts in submitted)
    t_last = max(ts + r["ms_latency"] / 1e3 for (_, ts), r in zip(submitted, results))
    span = max(t_last - t_first, 1e-9)
    waves = {r["wave"] for r in results}
    return {
        "requests": len(results),
        "p50_ms": percentile(lat, 50),
        "p99_ms": percentile(lat, 99),
        "mean_ms": float(np.mean(lat)) if lat else float("nan"),
        "max_ms": float(np.max(lat)) if lat else float("nan"),
        "wait_p50_ms": percentile(waits, 50),
        "span_s": span,
        "graphs_per_s": len(results) / span,
        "waves": len(waves),
        "mean_wave_graphs": float(np.mean([r["wave_graphs"] for r in results])) if results else 0.0,
        "per_lane": per_lane(results),
    }


def per_lane(results: Sequence[dict]) -> List[Dict[str, float]]:
    """Per lane: requests, latency p50/p99, wait p50, in-wave time p50
    (latency - wait) and waves."""
    out = []
    for lane in sorted({r.get("lane", 0) for r in results}):
        rs = [r for r in results if r.get("lane", 0) == lane]
        out.append({
            "lane": int(lane), "requests": len(rs),
            "p50_ms": percentile([r["ms_latency"] for r in rs], 50),
            "p99_ms": percentile([r["ms_latency"] for r in rs], 99),
            "wait_p50_ms": percentile([r["ms_wait"] for r in rs], 50),
            "in_wave_p50_ms": percentile([r["ms_latency"] - r["ms_wait"] for r in rs], 50),
            "waves": len({r["wave"] for r in rs}),
        })
    return out
