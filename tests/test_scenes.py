"""Synthetic workload generators: determinism and the geometric guarantees they promise."""
import numpy as np

from yarnball_b200 import scenes


def _min_nonadjacent_distance(pos, lens):
    from tests.np_ref import closest

    segs = []
    off = 0
    for y, m in enumerate(lens):
        for i in range(m - 1):
            segs.append((y, i, pos[off + i].astype(np.float64), pos[off + i + 1].astype(np.float64)))
        off += m
    best = np.inf
    for a in range(len(segs)):
        ya, ia, p0, p1 = segs[a]
        for b in range(a + 1, len(segs)):
            yb, ib, q0, q1 = segs[b]
            if ya == yb and abs(ia - ib) <= 2:
                continue
            u, v = closest(p1 - p0, q0 - p0, q1 - p0)
            best = min(best, np.linalg.norm(u * (p1 - p0) - ((q0 - p0) * (1 - v) + (q1 - p0) * v)))
    return best


def test_random_walks_deterministic_and_valid():
    lens = np.array([40, 25, 60], np.int32)
    a = scenes.random_walks(123, lens, cube=0.02)
    b = scenes.random_walks(123, lens, cube=0.02)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, scenes.random_walks(124, lens, cube=0.02))
    off = 0
    for m in lens:
        seg = np.linalg.norm(np.diff(a[off:off + m].astype(np.float64), axis=0), axis=1)
        assert np.allclose(seg, scenes.SEG_LEN, rtol=1e-5)
        off += m
    assert a.min() >= -1e-6 and a.max() <= 0.02 + 1e-6
    assert _min_nonadjacent_distance(a, lens) >= scenes.MIN_DIST * (1 - 1e-5)


def test_batch_scene_independent_of_threads():
    spec = scenes.batched_spec(seed=3, num_scenes=6, cap=100000, max_yarns=5, min_len=16, max_len=200)
    flat = np.concatenate(spec[1]).astype(np.int32)
    a = scenes.random_walks_batch(3, spec[0], flat, threads=1)
    b = scenes.random_walks_batch(3, spec[0], flat, threads=4)
    assert np.array_equal(a, b)


def test_batched_spec_respects_cap_and_ranges():
    yarns, lens, kbend = scenes.batched_spec()
    total = sum(int(l.sum()) for l in lens)
    assert total <= 8388608 and len(yarns) <= 512
    assert all(1 <= k <= 64 for k in yarns)
    allens = np.concatenate(lens)
    assert allens.min() >= 64 and allens.max() <= 4096
    assert min(kbend) >= 1e-9 and max(kbend) <= 1e-7


def test_readme_positions():
    p = scenes.readme_positions()
    assert p.shape == (64, 3)
    assert np.allclose(p[5], [2e-5 * 5 * (5 - 16) + 0.002, -0.01, 0], atol=1e-9)
    assert np.array_equal(p[32:, 0], -p[:32, 0])
