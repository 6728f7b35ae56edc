"""CPU tests of the serving host logic (arrival schedule, summaries)."""
import numpy as np


def test_poisson_arrivals_rate_and_mix():
    import serve
    arr = serve.poisson_arrivals(2000.0, 30.0, seed=3)
    assert abs(len(arr) / 30.0 - 2000.0) < 60  # Poisson count: sd ~ sqrt(60000)/30 ~ 8 per s
    t = np.array([a for a, _ in arr])
    assert np.all(np.diff(t) > 0) and t[-1] < 30.0
    sizes = [s for _, s in arr]
    for size, p in zip(serve.SERVED_SIZES, serve.SERVED_PROBS):
        assert abs(sizes.count(size) / len(sizes) - p) < 0.01
    pts = np.mean([a * b * c for a, b, c in sizes])
    assert abs(pts / 1e6 - 15.7) < 0.3  # mean 15.7M points per request


def test_summarize_percentiles():
    import serve
    reqs = [serve.Request(i, (4, 4, 4), arrival=0.0, start=0.0, done=(i + 1) * 1e-3) for i in range(100)]
    s = serve.summarize(reqs, 0.1)
    assert abs(s["p50_ms"] - 50.5) < 1e-9 and abs(s["p99_ms"] - 99.01) < 1e-9
    assert s["requests"] == 100
