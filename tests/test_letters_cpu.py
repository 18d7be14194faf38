"""The reference's own example scenes (KittenEngine/configs/letter*.json with the .poly curve
models they name), read in place when the reference project is present: the engine's readers
(read, transform, Catmull-Rom resampling, closed curves broken up) against the restatement in
oracle/curves.py, bit for bit, and the committed letter-I fixture against a fresh build from the
reference's files."""
import os
import sys

import numpy as np
import pytest

import yarnball_b200 as yb
from oracle import curves as oc

ROOT = os.environ.get("YB_REFERENCE_ROOT", "/root/reference")
CONFIGS = os.path.join(ROOT, "KittenEngine", "configs")
HERE = os.path.dirname(os.path.abspath(__file__))

pytestmark = pytest.mark.skipif(not os.path.isdir(CONFIGS), reason="reference example scenes not present")


def _golden():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_letters

    return make_letters


@pytest.mark.parametrize("letter", ["letterI", "letterS"])
def test_reference_letter_scene_readers_match_restatement(letter):
    ml = _golden()
    cfg, pos, flags, cid, _, _ = ml.letter_scene(ROOT, letter)
    T = np.diag([0.01, 0.01, 0.01, 1.0]).astype(np.float32)
    sim = yb.readFromPoly(os.path.join(ROOT, "KittenEngine", cfg["curveFile"]), float(cfg["resampleLength"]), T,
                          bool(cfg.get("breakUpClosedCurves", False)), True)
    assert sim.numVerts == len(pos) > 10000
    np.testing.assert_array_equal(sim.verts["pos"], pos)
    np.testing.assert_array_equal(sim.verts["flags"], flags)
    np.testing.assert_array_equal(sim.verts["connectionIndex"], cid)
    sim.close()


def test_letter_fixture_is_the_reference_scene():
    ml = _golden()
    cfg, pos, flags, cid, jsha, psha = ml.letter_scene(ROOT, "letterI")
    d = np.load(os.path.join(HERE, "golden", "letter_I.npz"))
    np.testing.assert_array_equal(d["pos"], pos)
    np.testing.assert_array_equal(d["flags"], flags)
    np.testing.assert_array_equal(d["cid"], cid)
    assert str(d["json_sha256"]) == jsha and str(d["poly_sha256"]) == psha
