"""The C++ drop-in header (include/yarnball/YarnBall.h) compiles against the README example
unchanged, links to the engine library, and (on a GPU) gives the same result as the Python
mirror of the same calls."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = str(tmp_path / "readme_example")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "readme_example.cpp"),
           "-L", os.path.join(ROOT, "yarnball_b200", "_lib"), "-lyarnball_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "yarnball_b200", "_lib"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


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
