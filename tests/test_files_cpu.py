"""The exporter restatement (oracle/files.py) against hand-worked known answers for the
reference's formats (io/fileExport.cpp:6-100), and the library's file entry points on CPU."""
import ctypes
import struct

import numpy as np

from oracle import files as ofiles
from yarnball_b200 import _abi


def _verts(flags, pos=None):
    v = np.zeros(len(flags), dtype=_abi.VERTEX_DTYPE)
    v["flags"] = flags
    v["pos"] = pos if pos is not None else np.arange(3 * len(flags), dtype=np.float32).reshape(-1, 3) / 8
    return v


def test_curve_runs_follow_has_next():
    # two yarns of 3 and 2 vertices, then a lone vertex, then a run left open at the end
    flags = [3, 3, 1, 2, 1, 0, 2, 3]
    assert ofiles.curve_runs(flags) == [(0, 2), (3, 4)]


def test_bcc_known_answer():
    v = _verts([2, 3, 1, 2, 1])
    data = ofiles.bcc_bytes(v)
    assert len(data) == 64 + (4 + 3 * 12) + (4 + 2 * 12)
    assert data[:8] == b"BCC\x44C0\x03\x01"
    assert struct.unpack_from("<QQ", data, 8) == (2, 5)
    assert data[24:64] == b"\0" * 40
    assert struct.unpack_from("<i", data, 64) == (3,)
    assert struct.unpack_from("<3f", data, 68) == (0.0, 0.125, 0.25)
    assert ofiles.bcc_bytes(v, True)[4:6] == b"PL"
    r = ofiles.read_bcc(data)
    assert r["end"] == len(data)
    np.testing.assert_array_equal(np.concatenate(r["curves"]), v["pos"])


def test_obj_known_answer():
    v = _verts([2, 1, 0], pos=np.array([[0.5, 0, 0], [0, 1e-3, 0], [0, 0, -2]], np.float32))
    text = ofiles.obj_text(v)
    lines = text.split("\n")
    assert lines[:5] == ["# YarnBall Sim", "", "o YarnBall", "", "# Vertices (in meters)"]
    assert lines[5] == "v 0.5000000000000000 0.0000000000000000 0.0000000000000000"
    # 1e-3 as a float32 promoted to double, printed with 16 decimals
    assert lines[6] == "v 0.0000000000000000 0.0010000000474975 0.0000000000000000"
    assert lines[9] == "# Curves"
    assert lines[10] == "l 1 2"


def test_obj_and_bcc_agree_on_curves():
    rng = np.random.default_rng(0)
    flags = rng.integers(0, 4, size=200).astype(np.uint32)
    flags[-1] = 0
    v = _verts(flags, rng.standard_normal((200, 3)).astype(np.float32))
    runs = ofiles.curve_runs(flags)
    obj_curves = [l for l in ofiles.obj_text(v).split("\n") if l.startswith("l ")]
    assert len(obj_curves) == len(runs)
    for line, (s, e) in zip(obj_curves, runs):
        idx = [int(t) - 1 for t in line.split()[1:]]
        assert idx == list(range(s, e + 1))


def test_run_open_at_the_end():
    # A run still open at the last vertex is written by the OBJ exporter (unterminated) and
    # dropped by the BCC exporter, as in the reference.
    v = _verts([2, 1, 2, 2])
    assert ofiles.obj_text(v).endswith("l 1 2\nl 3 4 5")
    assert struct.unpack_from("<Q", ofiles.bcc_bytes(v), 8) == (1,)


def test_file_entry_points_validate_arguments_on_cpu():
    lib = _abi.load()
    assert lib.yb_export_bcc(None, b"x.bcc", 0) != 0
    assert lib.yb_export_obj(None, b"x.obj") != 0
    assert lib.yb_save_state(None, b"x.ybck") != 0
    out = ctypes.c_void_p()
    assert lib.yb_load_state(b"/nonexistent-dir/x.ybck", ctypes.byref(out)) != 0
    assert not out.value


def test_mesher_stream_known_answers():
    from oracle import mesher
    assert mesher.splitmix64(0) == 0xE220A8397B1DCDAF  # SplitMix64's published first output for seed 0
    a, b = mesher.Xoroshiro128p(0x12345678), mesher.Xoroshiro128p(0x12345678)
    xs = [a.uniform() for _ in range(1000)]
    assert xs == [b.uniform() for _ in range(1000)]
    assert all(0.0 <= x <= 1.0 for x in xs) and 0.45 < sum(xs) / len(xs) < 0.55
    r = mesher.Xoroshiro128p(1)
    s0, s1 = r.s0, r.s1
    assert r.next() == (s0 + s1) & mesher.M64
