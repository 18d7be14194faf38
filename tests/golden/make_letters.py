"""Writes tests/golden/letter_I.npz from the reference's own example scene (run where the
reference project is present; the GPU machines only read the fixture).

Source: KittenEngine/configs/letterI.json and the curve model it names
(configs/models/letter_I.poly).  The fixture holds the scene as the reference's buildFromJSON
builds it before configure - the .poly read with the JSON's transform (default scale 0.01),
Catmull-Rom resampling to resampleLength and closed curves broken up - computed by this
repository's restatement of the reference's readers (oracle/curves.py, which the CPU tests
check against the engine's readers on the reference's files), plus the JSON's scene and solver
settings.  Provenance: the SHA-256 of the JSON and of the .poly.

    python tests/golden/make_letters.py [reference project root]
"""
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import curves as oc  # noqa: E402


def lenient_json(text):
    """The reference's JSON files carry // comments and trailing commas (jsoncpp accepts both)."""
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r",(\s*[}\]])", r"\1", text)
    return json.loads(text)


def letter_scene(root, name):
    ke = os.path.join(root, "KittenEngine")
    jpath = os.path.join(ke, "configs", name + ".json")
    jtext = open(jpath).read()
    cfg = lenient_json(jtext)
    poly = os.path.join(ke, cfg["curveFile"])
    ptext = open(poly).read()
    T = np.diag([0.01, 0.01, 0.01, 1.0]).astype(np.float32)
    curves, closed = oc.curves_poly(ptext, float(cfg["resampleLength"]), T.T.reshape(16),
                                    bool(cfg.get("breakUpClosedCurves", False)), True)
    pos, flags, cid = oc.from_curves(curves, closed)
    return cfg, pos, flags, cid, hashlib.sha256(jtext.encode()).hexdigest(), hashlib.sha256(ptext.encode()).hexdigest()


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    cfg, pos, flags, cid, jsha, psha = letter_scene(root, "letterI")
    lens = np.diff(np.concatenate([[0], np.nonzero((flags & 2) == 0)[0] + 1]))
    np.savez_compressed(os.path.join(HERE, "letter_I.npz"), pos=pos.astype(np.float32), flags=flags.astype(np.uint32),
                        cid=cid.astype(np.int32), yarn_lengths=lens.astype(np.int32), config=json.dumps(cfg),
                        json_sha256=jsha, poly_sha256=psha)
    print("letter_I.npz: %d vertices, %d yarns" % (len(pos), len(lens)))


if __name__ == "__main__":
    main()
