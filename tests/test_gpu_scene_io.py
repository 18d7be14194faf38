"""Scene construction on the GPU: glueEndpoints' nearest-vertex search (k_glue.cu) against the
restatement in oracle/curves.py, and buildFromJSON (io/jsonBuilder.cpp:8-172) end to end on
a synthetic .poly scene: reader + resampling, parameters, configure, glue, pins, upload, and a
frame of simulation."""
import json

import numpy as np
import pytest

import yarnball_b200 as yb
from oracle import curves as oc
from yarnball_b200.sim import Sim

pytestmark = pytest.mark.gpu


def _yarns(rng, k, m, box, step=2e-3):
    pts, lens = [], []
    for _ in range(k):
        p = rng.uniform(0, box, 3)
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        c = [p]
        for _ in range(m - 1):
            d = d + 0.3 * rng.standard_normal(3)
            d /= np.linalg.norm(d)
            c.append(c[-1] + step * d)
        pts.append(np.array(c))
        lens.append(m)
    return np.concatenate(pts).astype(np.float32), lens


def _fill(sim, pos, lens, offset=0):
    v = sim.verts[offset:offset + len(pos)]
    v["pos"] = pos
    ends = np.cumsum(lens) - 1
    v["flags"] = 2
    v["flags"][ends] = 0


@pytest.mark.parametrize("radius", [4e-3, 1e-2])
def test_glue_endpoints_matches_restatement(radius):
    rng = np.random.default_rng(3)
    pos, lens = _yarns(rng, 40, 24, 0.03)
    sim = Sim(len(pos))
    _fill(sim, pos, lens)
    want_pos, want_cid = oc.glue_endpoints(sim.verts["pos"], sim.verts["flags"], sim.verts["connectionIndex"], radius)
    sim.glueEndpoints(radius)
    assert (want_cid >= 0).sum() > 10
    np.testing.assert_array_equal(sim.verts["connectionIndex"], want_cid)
    np.testing.assert_array_equal(sim.verts["pos"], want_pos)
    sim.close()


def test_glue_endpoints_stays_inside_each_scene():
    rng = np.random.default_rng(4)
    pa, la = _yarns(rng, 12, 20, 0.02)
    pb, lb = _yarns(rng, 9, 30, 0.02)  # same region of space, another scene
    sim = Sim(scenes=[len(pa), len(pb)])
    _fill(sim, pa, la, 0)
    _fill(sim, pb, lb, len(pa))
    ranges = [(0, len(pa)), (len(pa), len(pa) + len(pb))]
    want_pos, want_cid = oc.glue_endpoints(sim.verts["pos"], sim.verts["flags"], sim.verts["connectionIndex"],
                                           8e-3, ranges)
    sim.glueEndpoints(8e-3)
    np.testing.assert_array_equal(sim.verts["connectionIndex"], want_cid)
    np.testing.assert_array_equal(sim.verts["pos"], want_pos)
    c = sim.verts["connectionIndex"]
    for i in np.where(c >= 0)[0]:
        assert (i < len(pa)) == (c[i] < len(pa))
    sim.close()


def _poly_scene(tmp_path):
    rng = np.random.default_rng(5)
    chains = []
    for k in range(6):  # cm units: the JSON builder scales by 0.01
        t = np.linspace(0, 1, 30)
        base = np.array([k * 0.8, 0.0, 0.0])
        c = base + np.stack([0.3 * np.sin(6 * t), 8 * t, 0.3 * np.cos(5 * t + k)], 1)
        chains.append(c + 0.01 * rng.standard_normal(c.shape))
    ang = np.linspace(0, 2 * np.pi, 40, endpoint=False)
    loop = np.stack([2.0 + 1.5 * np.cos(ang), 4.0 + 1.5 * np.sin(ang), np.full_like(ang, 1.0)], 1)
    pts, segs = [], []
    for c in chains:
        b = len(pts)
        pts += list(c)
        segs += [(b + i, b + i + 1) for i in range(len(c) - 1)]
    b = len(pts)
    pts += list(loop)
    segs += [(b + i, b + (i + 1) % len(loop)) for i in range(len(loop))]
    lines = ["POINTS"] + ["%d: %.7g %.7g %.7g" % ((i + 1,) + tuple(p)) for i, p in enumerate(pts)]
    lines += ["POLYS"] + ["%d: %d %d" % (k + 1, a + 1, c + 1) for k, (a, c) in enumerate(segs)] + ["END", ""]
    text = "\n".join(lines)
    path = tmp_path / "scene.poly"
    path.write_text(text)
    return path, text


def test_build_from_json_end_to_end(tmp_path):
    poly, text = _poly_scene(tmp_path)
    doc = """{
        // a scene in the reference's format
        "curveFile": %s,
        "resampleLength": 2e-3,
        "curveRadius": 0.0010,
        "glueEndpoints": 0.004,
        "fixBorders": [0, 0, 0, 0.005, 0, 0],
        "fixVertex": [[0.02, 0.04, 0.01], [0.0, 0.0, 0.0, 0.003], 5],
        "simulation": {
            "density": 1e-3,
            "frictionCoeff": 0.25,
            "kStretch": 1e-1,
            "kBend": 2e-7,
            "kCollision": 2e-4,
            "kFriction": 5,
            "damping": 1e-7,
            "gravity": [0, -9.8, 0],
            "drag": 0.1,
            "maxTimeStep": 5e-4,
            "numIterations": 6,
            "detectionPeriod": 2,
            "detectionScaler": 1.1,
            "stepLimit": true,
            "velStepLimit": true,
        },
    }""" % json.dumps(str(poly))
    cfg = tmp_path / "scene.json"
    cfg.write_text(doc)
    sim = yb.buildFromJSON(str(cfg))

    # geometry: reader + resampling + glue, as restated
    T = np.diag([0.01, 0.01, 0.01, 1.0]).astype(np.float32)
    curves, closed = oc.curves_poly(text, 2e-3, T.T.reshape(16), False, True)
    pos, flags, cid = oc.from_curves(curves, closed)
    assert closed == [False] * 6 + [True]
    pos, cid = oc.glue_endpoints(pos, flags, cid, 0.004)
    np.testing.assert_array_equal(sim.verts["connectionIndex"], cid)
    np.testing.assert_array_equal(sim.verts["pos"], pos)

    # parameters
    m = sim.meta
    assert m.radius == np.float32(np.float32(0.05) * np.float32(1e-3))
    assert m.barrierThickness == np.float32(np.float32(2 * (1 - np.float32(0.05))) * np.float32(1e-3))
    assert (m.numItr, m.detectionPeriod, m.useStepSizeLimit, m.useVelocityRadius) == (6, 2, 1, 1)
    assert m.frictionCoeff == np.float32(0.25) and m.kFriction == np.float32(5) and m.drag == np.float32(0.1)
    assert sim.maxH == np.float32(5e-4)

    # pins: bottom border band, the vertex closest to (0.02, 0.04, 0.01), a sphere, index 5
    inv = sim.verts["invMass"]
    p = sim.verts["pos"]
    lo_y = np.float32(np.float32(p[:, 1].min() - np.float32(0.01) * np.float32(m.radius)) + np.float32(0.005))
    band = p[:, 1] < lo_y
    assert band.sum() > 0 and np.all(inv[band] == 0)
    d2 = ((p - np.float32([0.02, 0.04, 0.01])) ** 2).sum(1)
    assert inv[int(np.argmin(d2))] == 0
    assert np.all(inv[(p ** 2).sum(1) < 0.003 ** 2] == 0)
    assert inv[5] == 0
    assert (inv > 0).sum() > len(inv) // 2

    sim.advance(1 / 30.0)
    sim.download()
    assert np.all(np.isfinite(sim.verts["pos"]))
    assert np.abs(sim.verts["pos"] - pos).max() > 0
    sim.close()
