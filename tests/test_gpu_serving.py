"""Continuous batching: requests that join and leave a device-resident batch between frames
give, each, exactly the result they give when simulated alone (bit for bit: a scene's state
travels with it, contacts are re-detected every substep, and the Newton kernel shape is the
same)."""
import numpy as np
import pytest

from yarnball_b200 import serve

pytestmark = pytest.mark.gpu

SHAPE = (128, 0)


def _requests():
    specs = [
        ((np.array([300, 200, 120], np.int32), 3e-8), 0, 4),
        ((np.array([500, 64], np.int32), 1e-9), 0, 6),
        ((np.array([150, 150, 150, 150], np.int32), 5e-8), 2, 3),
        ((np.array([800], np.int32), 1e-7), 3, 5),
        ((np.array([90, 400, 77], np.int32), 2e-9), 3, 2),
    ]
    reqs = []
    for i, (spec, tick, frames) in enumerate(specs):
        r = serve.Request(i, float(tick), spec, frames=frames, seed=100 + i)
        reqs.append(r)
    return reqs


def test_each_request_same_alone_and_in_the_mix():
    reqs = _requests()
    server = serve.Server(shape=SHAPE)
    pending = sorted(reqs, key=lambda r: r.arrival)
    t = 0
    while pending or server.busy():
        while pending and pending[0].arrival <= t:
            server.submit(pending.pop(0))
        server.step(float(t))
        t += 1
        assert t < 100
    assert server.gathers >= 3  # scenes joined and left between frames
    assert max(server.frame_sizes) > max(r.vertices for r in reqs)  # frames really were shared
    for r in reqs:
        assert r.result is not None
        pos, vel, q = serve.run_alone(r, SHAPE)
        assert np.array_equal(r.result[0], pos), r.id
        assert np.array_equal(r.result[1], vel), r.id
        assert np.array_equal(r.result[2], q), r.id
    server.close()


def test_gather_recycles_allocation():
    from yarnball_b200.sim import Sim

    reqs = _requests()[:3]
    sims = [serve.build_request_sim(r, SHAPE) for r in reqs]
    a = Sim.gather([(s, 0) for s in sims], capacity=10000)
    b = Sim.gather([(a, 1), (a, 0)], capacity=10000)
    c = Sim.gather([(b, 1)], recycle=a)
    assert c is a and c.numScenes == 1 and c.numVerts == reqs[0].vertices
    for s in sims:
        s.close()
    b.close()
    c.close()
