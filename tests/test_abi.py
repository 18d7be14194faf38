"""The C ABI library loads without a GPU and exports every function declared in include/*.h;
the oracle library exports its checker API."""
import ctypes
import os
import re

import pytest

import oracle
from yarnball_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(path):
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(yb_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_abi.LIB_PATH)
    names = []
    for h in ("yarnball_b200.h", "yarnball_b200_scenes.h"):
        names += declared_functions(os.path.join(ROOT, "include", h))
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header():
    names = declared_functions(os.path.join(ROOT, "include", "yarnball_b200.h"))
    names += declared_functions(os.path.join(ROOT, "include", "yarnball_b200_scenes.h"))
    assert sorted(set(names) - set(_abi.SIGNATURES)) == []


def test_struct_layouts():
    assert ctypes.sizeof(_abi.YbVertex) == 32
    assert ctypes.sizeof(_abi.YbMeta) == ctypes.sizeof(oracle.OrcMeta) == 29 * 4


def test_status_strings_and_cpu_errors():
    lib = _abi.load()
    assert lib.yb_status_string(0) == b"ok"
    assert b"MAX_COLLISIONS" in lib.yb_status_string(8)
    h = ctypes.c_void_p()
    assert lib.yb_create(2, ctypes.byref(h)) == 2  # too few vertices (YarnBall.cu:12)
    assert lib.yb_create(3, ctypes.byref(h)) == 0
    # advancing before configure is refused, not crashed
    assert lib.yb_advance(h, ctypes.c_float(0.01), None) == 3
    assert lib.yb_set_kbend(h, -1, ctypes.c_float(1e-8)) == 3
    lib.yb_destroy(h)


def test_oracle_exports():
    lib = oracle.load()
    for name in oracle._SIG:
        assert hasattr(lib, name)


def test_scene_rng_is_xoshiro256ss_seeded_by_splitmix64():
    # xoshiro256** seeded with four SplitMix64 outputs of seed 0: first outputs computed
    # from the published algorithm in pure Python
    M = (1 << 64) - 1

    def splitmix(x):
        x = (x + 0x9E3779B97F4A7C15) & M
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return x, z ^ (z >> 31)

    def rotl(v, k):
        return ((v << k) | (v >> (64 - k))) & M

    x, s = 0, []
    for _ in range(4):
        x, z = splitmix(x)
        s.append(z)
    outs = []
    for _ in range(5):
        r = (rotl((s[1] * 5) & M, 7) * 9) & M
        t = (s[1] << 17) & M
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45)
        outs.append(r)
    lib = _abi.load()
    assert [lib.yb_rng_u64(0, i) for i in range(5)] == outs


def test_batch_scenes_must_share_a_schedule():
    """The scenes of a batch advance on one schedule (shared substep loop, detection cadence,
    BVH rebuild clock and Newton launches), so configure refuses a batch whose scenes' meta
    disagree on numItr, detectionPeriod or bvhRebuildPeriod (the reference keeps them per Sim,
    YarnBall.h:63-114, step.cpp:46-49).  The check runs before any device work."""
    import numpy as np

    from yarnball_b200 import sim as ybsim

    for field, value in [("numItr", 4), ("detectionPeriod", 2), ("bvhRebuildPeriod", 0.05)]:
        s = ybsim.Sim(scenes=[8, 8])
        for k in range(2):
            s.verts["pos"][8 * k:8 * k + 8] = np.stack([np.arange(8) * 2e-3, np.full(8, 0.01 * k), np.zeros(8)], 1)
        setattr(s.scene_meta(1), field, value)
        with pytest.raises(RuntimeError):
            s.configure()
        assert s._lib.yb_configure(s._h, ctypes.c_float(1e-3)) == 1  # YB_ERR_INVALID_ARGUMENT
        s.close()


def test_walk_mode_and_small_path_switches():
    """Broadphase walk modes 0 (per query), 1 (per warp of 32 queries) and 2 (per query with
    cooperative record loads, the default) are accepted, other values refused; the
    small-simulation switch takes 0 or 1.  No device work is needed to set them."""
    lib = _abi.load()
    h = ctypes.c_void_p()
    assert lib.yb_create(64, ctypes.byref(h)) == 0
    mode = ctypes.c_int32()
    assert lib.yb_get_traversal(h, ctypes.byref(mode)) == 0 and mode.value == 2
    for m in (0, 1, 2):
        assert lib.yb_set_traversal(h, m) == 0
        assert lib.yb_get_traversal(h, ctypes.byref(mode)) == 0 and mode.value == m
    for m in (-1, 3):
        assert lib.yb_set_traversal(h, m) == 1  # YB_ERR_INVALID_ARGUMENT
    assert lib.yb_set_small_path(h, 0) == 0 and lib.yb_set_small_path(h, 1) == 0
    assert lib.yb_set_small_path(h, 2) == 1
    lib.yb_destroy(h)
