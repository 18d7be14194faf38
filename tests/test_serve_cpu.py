"""Host-side pieces of the serving loop (no GPU): the request stream and its statistics."""
import numpy as np

from yarnball_b200 import serve


def test_poisson_requests_shape_and_determinism():
    a = serve.poisson_requests(50.0, 4.0, seed=3)
    b = serve.poisson_requests(50.0, 4.0, seed=3)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert 120 < len(a) < 280  # ~200 expected
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert np.all(gaps > 0) and abs(np.mean(gaps) - 1 / 50.0) < 0.01
    sizes = np.array([r.vertices for r in a])
    assert sizes.min() >= 64 and sizes.max() <= 1_000_000
    assert 8000 < np.median(sizes) < 32000  # lognormal median 16,384
    for r in a:
        lens, kb = r.spec
        assert lens.sum() == r.vertices and np.all(lens >= 3)
        assert 1e-9 <= kb <= 1e-7 and r.frames == 30


def test_percentiles():
    p = serve.percentiles(list(range(1, 101)))
    assert p["p50"] == 50.5 and abs(p["p99"] - 99.01) < 1e-9
    assert serve.percentiles([])["p50"] is None
