"""Curve readers and the Catmull-Rom resampler (io/reader.cpp, io/resample.h) on CPU: the
library's C++ against the restatement in oracle/curves.py, bit for bit, on synthetic files;
hand-worked properties of the resampler; the reference's error messages."""
import ctypes
import math
import struct

import numpy as np
import pytest

from oracle import curves as oc
from yarnball_b200 import _abi
from yarnball_b200 import sim as ybsim

SCALE = np.diag([0.01, 0.01, 0.01, 1.0])  # the JSON builder's default transform


def _helix(m, turns=2.0, radius=1.0, pitch=0.5, noise=0.0, seed=0):
    rng = np.random.default_rng(seed)
    t = np.linspace(0, 2 * math.pi * turns, m)
    p = np.stack([radius * np.cos(t), radius * np.sin(t), pitch * t / (2 * math.pi)], 1)
    return (p + noise * rng.standard_normal(p.shape)).astype(np.float32)


@pytest.mark.parametrize("m,tar,noise", [(12, 0.3, 0.0), (40, 0.11, 0.02), (200, 0.05, 0.01), (7, 0.9, 0.0)])
def test_resample_matches_restatement(m, tar, noise):
    pts = _helix(m, noise=noise, seed=m)
    got = ybsim.resampleCMR(pts, 1, m - 2, tar)
    want = oc.resample_cmr(pts, 1, m - 2, tar)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got, want)


def test_resample_straight_line_known_answer():
    # control points 1 apart on the x axis: the spline is the line x = t, so the resampled
    # points are the parameters themselves; they span [cmr[1], cmr[-2]] at about the target.
    pts = np.zeros((11, 3), np.float32)
    pts[:, 0] = np.arange(11)
    r = ybsim.resampleCMR(pts, 1, 9, 0.5)
    assert r[0, 0] == 1.0 and r[-1, 0] == 9.0
    assert np.all(r[:, 1:] == 0)
    seg = np.diff(r[:, 0])
    assert np.all(seg > 0)
    assert abs(seg.mean() - 0.5) < 1e-3 and np.abs(seg - 0.5).max() < 0.05
    assert len(r) == 17


def test_resample_short_curve_is_unchanged():
    pts = _helix(3)
    np.testing.assert_array_equal(ybsim.resampleCMR(pts, 1, 1, 0.1), pts)


def _bcc_bytes(curves, kind=b"C0", closed=()):
    out = [struct.pack("<3sB2sbbQQ40s", b"BCC", 0x44, kind, 3, 1, len(curves), sum(map(len, curves)), b"\0" * 40)]
    for i, c in enumerate(curves):
        m = len(c)
        out.append(struct.pack("<i", -m if i in closed else m))
        out.append(np.asarray(c, np.float32).tobytes())
    return b"".join(out)


def _check_sim(sim, curves, closed):
    pos, flags, cid = oc.from_curves(curves, closed)
    assert sim.numVerts == len(pos)
    np.testing.assert_array_equal(sim.verts["pos"], pos)
    np.testing.assert_array_equal(sim.verts["flags"], flags)
    np.testing.assert_array_equal(sim.verts["connectionIndex"], cid)


@pytest.mark.parametrize("kind,resample,break_up", [(b"C0", True, False), (b"PL", True, False),
                                                   (b"C0", False, True), (b"C0", True, True)])
def test_read_bcc(tmp_path, kind, resample, break_up):
    curves = [_helix(30, seed=1) * 40, _helix(2, seed=2) * 40, _helix(9, turns=0.5, seed=3) * 40,
              _helix(55, turns=3, noise=0.05, seed=4) * 40]
    data = _bcc_bytes(curves, kind, closed={3})
    p = tmp_path / "c.bcc"
    p.write_bytes(data)
    sim = ybsim.readFromBCC(str(p), 2e-3, SCALE, break_up, resample)
    want_c, want_closed = oc.curves_bcc(data, 2e-3, SCALE.T.reshape(16), break_up, resample)
    assert len(want_c) == 3  # the 2-point curve is dropped
    _check_sim(sim, want_c, want_closed)
    sim.close()


def test_read_obj(tmp_path):
    a = _helix(25, seed=5) * 30
    b = _helix(18, turns=1, seed=6) * 30
    lines = ["# test", "o curves"] + ["v %.9g %.9g %.9g" % tuple(p) for p in np.concatenate([a, b])]
    la = " ".join(str(i + 1) for i in range(25))
    lb = " ".join(str(25 + i + 1) for i in range(18)) + " 26"  # closed loop: first index repeated
    lines += ["l " + la, "l " + lb, "l 1 2", ""]
    text = "\n".join(lines)
    p = tmp_path / "c.obj"
    p.write_text(text)
    for break_up in (False, True):
        sim = ybsim.readFromOBJ(str(p), 1.5e-3, SCALE, break_up, True)
        want_c, want_closed = oc.curves_obj(text, 1.5e-3, SCALE.T.reshape(16), break_up, True)
        assert want_closed == [False, not break_up]
        _check_sim(sim, want_c, want_closed)
        sim.close()


def _poly_text(chains, loops, shuffle_seed=None):
    pts, segs = [], []
    for c in chains:
        base = len(pts)
        pts += list(c)
        segs += [(base + i, base + i + 1) for i in range(len(c) - 1)]
    for c in loops:
        base = len(pts)
        pts += list(c)
        segs += [(base + i, base + (i + 1) % len(c)) for i in range(len(c))]
    if shuffle_seed is not None:
        np.random.default_rng(shuffle_seed).shuffle(segs)
    lines = ["POINTS"] + ["%d: %.9g %.9g %.9g" % ((i + 1,) + tuple(p)) for i, p in enumerate(pts)]
    lines += ["POLYS"] + ["%d: %d %d" % (k + 1, a + 1, b + 1) for k, (a, b) in enumerate(segs)]
    return "\n".join(lines + ["END", ""])


@pytest.mark.parametrize("break_up,resample", [(False, True), (True, True), (False, False)])
def test_read_poly(tmp_path, break_up, resample):
    chain = _helix(40, seed=7) * 20
    short = _helix(3, seed=8) * 20  # dropped: fewer than 4 points
    loop = _helix(33, turns=1, pitch=0.0, seed=9)[:-1] * 20
    text = _poly_text([chain, short], [loop], shuffle_seed=1)
    p = tmp_path / "c.poly"
    p.write_text(text)
    sim = ybsim.readFromPoly(str(p), 1e-3, SCALE, break_up, resample)
    want_c, want_closed = oc.curves_poly(text, 1e-3, SCALE.T.reshape(16), break_up, resample)
    assert want_closed == [False, not break_up]
    _check_sim(sim, want_c, want_closed)
    sim.close()


def _status_and_message(fn, path):
    lib = _abi.load()
    out = ctypes.c_void_p()
    st = getattr(lib, fn)(path, ctypes.c_float(1e-3), None, 0, 1, ctypes.byref(out))
    return st, lib.yb_last_io_error().decode(), out.value


def test_reader_errors(tmp_path):
    st, msg, h = _status_and_message("yb_read_bcc", b"/nonexistent-dir/x.bcc")
    assert st == 14 and msg == "Could not open file" and not h
    bad = tmp_path / "bad.bcc"
    bad.write_bytes(b"XYZ" + b"\0" * 61)
    assert _status_and_message("yb_read_bcc", str(bad).encode())[:2] == (15, "Unsupported BCC file")
    two_d = tmp_path / "2d.bcc"
    hdr = bytearray(_bcc_bytes([_helix(5)]))
    hdr[6] = 2
    two_d.write_bytes(bytes(hdr))
    assert _status_and_message("yb_read_bcc", str(two_d).encode())[:2] == (15, "Only curves in 3D are supported")
    graph = tmp_path / "g.poly"
    graph.write_text("POINTS\n1: 0 0 0\n2: 1 0 0\n3: 0 1 0\n4: 0 0 1\nPOLYS\n1: 1 2\n2: 1 3\n3: 1 4\nEND\n")
    assert _status_and_message("yb_read_poly", str(graph).encode())[:2] == (15, "Graphs not allowed.")
    ids = tmp_path / "ids.poly"
    ids.write_text("POINTS\n1: 0 0 0\n3: 1 0 0\nEND\n")
    assert _status_and_message("yb_read_poly", str(ids).encode())[:2] == (15, "Error parsing .poly. Point id mismatch.")
    st, msg, _ = _status_and_message("yb_read_obj", b"/nonexistent-dir/x.obj")
    assert st == 14 and msg == "Could not open file."


def test_json_errors(tmp_path):
    lib = _abi.load()
    out = ctypes.c_void_p()
    assert lib.yb_build_from_json(b"/nonexistent-dir/s.json", ctypes.byref(out)) == 14
    assert lib.yb_last_io_error().decode() == "Error opening file"
    bad = tmp_path / "bad.json"
    bad.write_text('{"curveFile": "x.poly", "resampleLength": }')
    assert lib.yb_build_from_json(str(bad).encode(), ctypes.byref(out)) == 15
    assert lib.yb_last_io_error().decode().startswith("Error parsing the JSON file")
    missing = tmp_path / "m.json"
    missing.write_text('{ // a comment\n "curveFile": "/nonexistent-dir/c.poly", "resampleLength": 2e-3, }')
    assert lib.yb_build_from_json(str(missing).encode(), ctypes.byref(out)) == 14


def test_glue_restatement_known_answer():
    # yarn A: x axis 0..5 mm; yarn B starts 0.5 mm above A's vertex 3 and runs up the y axis.
    a = np.stack([np.arange(6) * 1e-3, np.zeros(6), np.zeros(6)], 1)
    b = np.stack([np.full(5, 3e-3), 5e-4 + np.arange(5) * 1e-3, np.zeros(5)], 1)
    pos = np.concatenate([a, b]).astype(np.float32)
    flags = np.full(11, 2, np.uint32)
    flags[[5, 10]] = 0
    cid = np.full(11, -1, np.int32)
    p2, c2 = oc.glue_endpoints(pos, flags, cid, 1e-3)
    # endpoints: 0 (A start), 5 (A end), 6 (B start), 10 (B end); only B's start is near A
    assert c2[6] == 3 and c2[3] == 6 and (c2 >= 0).sum() == 2
    np.testing.assert_array_equal(p2[6], np.float32([3e-3, 2.5e-4, 0]))
    np.testing.assert_array_equal(p2[3], p2[6])
    # a smaller radius joins nothing
    assert (oc.glue_endpoints(pos, flags, cid, 4e-4)[1] >= 0).sum() == 0
