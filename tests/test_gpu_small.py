"""The one-block path for small simulations (<= 256 vertices: every substep of an advance in
one launch) against the multi-block path (BVH detection, per-substep kernels) with the same
load-balanced Newton kernel: identical positions, velocities and rotors, bit for bit, frame
after frame, including contacts, detection every few substeps and the FP64 build."""
import numpy as np
import pytest

from yarnball_b200 import scenes

pytestmark = pytest.mark.gpu


def _tangle(precision="fp32", meta=None):
    """6 yarns x 40 vertices in a 1 cm cube: 240 vertices with many contacts."""
    return scenes.build_pile(seed=4, yarns=6, verts=40, cube=0.01, precision=precision, meta=meta)


CASES = {
    "readme": lambda: scenes.build_readme(),
    "tangle": lambda: _tangle(),
    "tangle_fp64": lambda: _tangle("fp64"),
    "tangle_detect3_itr5": lambda: _tangle(meta={"detectionPeriod": 3, "numItr": 5}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_small_path_equals_multi_block_path(name):
    a, b = CASES[name](), CASES[name]()
    b.set_small_path(False)
    for s in (a, b):
        s.set_tuning(128, 0, True, False)
    launches = []
    for f in range(6):
        l0 = a.launch_count()
        a.advance(1 / 30.0)
        launches.append(a.launch_count() - l0)
        b.advance(1 / 30.0)
        for x, y in zip(a.read_state_f64(), b.read_state_f64()):
            assert np.array_equal(x, y), (name, f)
    assert a.stepCount() == b.stepCount() == 6 * 34
    assert max(launches) <= 2  # the one-block kernel (+ the final state readback, none)
    if name.startswith("tangle"):
        na, _, _ = a.debug_contacts()
        assert na.sum() > 0
    assert a.penetrations() == b.penetrations()
    assert a.min_pair_distance() == b.min_pair_distance()
    a.close()
    b.close()
