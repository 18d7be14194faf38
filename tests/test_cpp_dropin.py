"""The C++ drop-in header (include/yarnball/YarnBall.h) compiles against the README example
unchanged, links to the engine library, and (on a GPU) gives the same result as the Python
mirror of the same calls."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path, name="readme_example"):
    exe = str(tmp_path / name)
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
           "-L", os.path.join(ROOT, "yarnball_b200", "_lib"), "-lyarnball_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "yarnball_b200", "_lib"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))
    assert os.path.exists(_build(tmp_path, "bounds_example"))


@pytest.mark.gpu
def test_dropin_bounds_is_a_box(tmp_path):
    """bounds() returns a box with the reference's aabb methods (absorb, pad, contains,
    intersects, center, volume) that holds every vertex after a frame."""
    exe = _build(tmp_path, "bounds_example")
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    assert out[0] == "64" and out[1] == "1" and out[2] == "1"
    assert float(out[3]) > 0 and np.isfinite(float(out[4]))


@pytest.mark.gpu
def test_dropin_readme_matches_python(tmp_path):
    from yarnball_b200 import scenes

    exe = _build(tmp_path)
    out = subprocess.run([exe, "3"], check=True, capture_output=True, text=True).stdout.split("\n")
    p31 = np.array([float(x) for x in out[0].split()], np.float32)
    p63 = np.array([float(x) for x in out[1].split()], np.float32)
    assert out[2].strip() == "steps %d" % (3 * 34)
    sim = scenes.build_readme()
    for _ in range(3):
        sim.advance(1 / 30.0)
    sim.download()
    assert np.array_equal(sim.verts["pos"][31], p31)
    assert np.array_equal(sim.verts["pos"][63], p63)


def test_dropin_readers(tmp_path):
    """YarnBall::readFromPoly through the drop-in header (no GPU needed) matches the Python
    reader, and a malformed file throws with the reference's message."""
    from tests.test_curves_cpu import _helix, _poly_text
    from yarnball_b200 import sim as ybsim

    exe = str(tmp_path / "reader_example")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "reader_example.cpp"),
           "-L", os.path.join(ROOT, "yarnball_b200", "_lib"), "-lyarnball_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "yarnball_b200", "_lib"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    poly = tmp_path / "c.poly"
    poly.write_text(_poly_text([_helix(40, seed=1) * 20], [_helix(25, turns=1, pitch=0.0, seed=2)[:-1] * 20]))
    out = subprocess.run([exe, "poly", str(poly)], check=True, capture_output=True, text=True).stdout.split()
    sim = ybsim.readFromPoly(str(poly), 2e-3, np.diag([0.01, 0.01, 0.01, 1.0]))
    assert int(out[0]) == sim.numVerts and int(out[1]) == 2
    assert np.array_equal(np.float32([float(x) for x in out[2:5]]), sim.verts["pos"][0])
    sim.close()
    bad = tmp_path / "bad.poly"
    bad.write_text("POINTS\n1: 0 0 0\n2: 1 0 0\n3: 0 1 0\n4: 0 0 1\nPOLYS\n1: 1 2\n2: 1 3\n3: 1 4\nEND\n")
    r = subprocess.run([exe, "poly", str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and r.stdout.strip() == "error: Graphs not allowed."
