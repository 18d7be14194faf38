"""The reference's example scene letterI (KittenEngine/configs/letterI.json) through
buildFromJSON with the reference's own scene and solver settings (maxTimeStep 4e-4, 4
iterations, detection every 4 substeps, detection scaler 1.1, pins by fixVertex), one frame
against the FP64 oracle.

The geometry comes from the committed fixture tests/golden/letter_I.npz (the reference's model
read and resampled, checked against the reference's files by tests/test_letters_cpu.py); it is
written back as a .poly in metres (identity transform) for the JSON builder, whose resampling
of the already uniform curve moves no vertex by more than a small fraction of a segment.

Tolerances: one substep within 1e-5 x segment length of the FP64 oracle; one frame (84
substeps) relative error <= 1e-3 (max position error / max displacement).  The frame bound is
looser than the 1e-4 of the benchmark scenes: this scene's contacts are 2000x stiffer
(kCollision 2e-4 against 1e-7) and its single 26 m yarn is knitted into itself, so FP32
rounding in the barrier terms is amplified more over the frame (measured 3.7e-4)."""
import json
import os

import numpy as np
import pytest

import oracle
import yarnball_b200 as yb

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _scene(tmp_path):
    d = np.load(os.path.join(HERE, "golden", "letter_I.npz"))
    cfg = json.loads(str(d["config"]))
    pos, lens = d["pos"], d["yarn_lengths"]
    lines, segs, b = ["POINTS"], [], 0
    for i, p in enumerate(pos):
        lines.append("%d: %.9g %.9g %.9g" % (i + 1, p[0], p[1], p[2]))
    for n in lens:
        segs += [(b + i, b + i + 1) for i in range(n - 1)]
        b += n
    lines += ["POLYS"] + ["%d: %d %d" % (k + 1, a + 1, c + 1) for k, (a, c) in enumerate(segs)] + ["END", ""]
    poly = tmp_path / "letter_I_m.poly"
    poly.write_text("\n".join(lines))
    cfg["curveFile"] = str(poly)
    cfg["transform"] = [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0]]
    path = tmp_path / "letterI.json"
    path.write_text(json.dumps(cfg))
    return str(path), cfg, pos


def test_letter_I_with_the_reference_settings_vs_fp64_oracle(tmp_path):
    path, cfg, pos0 = _scene(tmp_path)
    sim = yb.buildFromJSON(path)
    m = sim.meta
    sc = cfg["simulation"]
    assert (m.numItr, m.detectionPeriod) == (sc["numIterations"], sc["detectionPeriod"])
    assert sim.maxH == np.float32(sc["maxTimeStep"])
    assert abs(sim.numVerts - len(pos0)) < 0.01 * len(pos0)
    # fixVertex: the vertex nearest to each listed point is pinned
    p = sim.verts["pos"]
    for q in cfg["fixVertex"]:
        assert sim.verts["invMass"][int(np.argmin(((p - np.float32(q)) ** 2).sum(1)))] == 0
    maxH = float(np.float32(sc["maxTimeStep"]))
    x0 = sim.read_state_f64()[0]
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    sim.step()                      # one substep of maxH
    orc.advance(maxH, maxH)
    assert np.abs(sim.read_state_f64()[0] - orc.state()["pos"]).max() <= 1e-5 * 2e-3
    sim.advance(1 / 30.0)
    orc.advance(1 / 30.0, maxH)
    pos = sim.read_state_f64()[0]
    ref = orc.state()["pos"]
    disp = np.abs(ref - x0).max()
    assert disp > 1e-4
    assert np.abs(pos - ref).max() / disp <= 1e-3, np.abs(pos - ref).max() / disp
    assert sim.stepCount() == 1 + int(np.ceil(np.float32(1 / 30.0) / np.float32(sc["maxTimeStep"])))
    sim.close()
    orc.close()
