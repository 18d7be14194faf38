"""The one-block path for small simulations (<= 256 vertices: every substep of an advance in
one launch).

It runs the device functions of the multi-block kernels (predictor, narrow-phase filter, step
limit, Newton iteration in the load-balanced kernel's summation order, advection) in one
kernel, so the compiler may contract multiplies and adds into fused operations differently
there; the two paths therefore agree to rounding, not bit for bit.  Parity is held to the same
bar as every other path:
  * one frame against the FP64 oracle: relative error <= 1e-4 (max position error / max
    displacement) for the FP32 build, 1e-9 x segment length for the FP64 build;
  * against the multi-block path over 6 frames (204 substeps): max position difference
    <= 1e-4 of the largest displacement, the bar between any FP32 result and the FP64 oracle
    (rounding differences grow over the substeps of these contact scenes: 3.2e-6 on the README
    scene, 2.2e-6 on the tangle, 2.0e-5 on the tangle with detection every 3 substeps measured
    on a B200; the FP64 build within 1e-6);
  * one launch per advance.
"""
import numpy as np
import pytest

import oracle
from yarnball_b200 import scenes

pytestmark = pytest.mark.gpu

SEG = 2e-3
FRAME = 1.0 / 30.0


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
def test_small_path_vs_fp64_oracle(name):
    sim = CASES[name]()
    x0 = sim.read_state_f64()[0]
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    l0 = sim.launch_count()
    sim.advance(FRAME)
    assert sim.launch_count() - l0 <= 2  # the one-block kernel
    orc.advance(FRAME, float(np.float32(sim.maxH)))
    pos = sim.read_state_f64()[0]
    ref = orc.state()["pos"]
    err = np.abs(pos - ref).max()
    if name.endswith("fp64"):
        assert err <= 1e-9 * SEG, err
    else:
        disp = np.abs(ref - x0).max()
        assert disp > 0
        assert err / disp <= 1e-4, err / disp
    sim.close()
    orc.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_small_path_matches_multi_block_path(name):
    a, b = CASES[name](), CASES[name]()
    b.set_small_path(False)
    for s in (a, b):
        s.set_tuning(128, 0, True, False)
    x0 = a.read_state_f64()[0]
    worst = 0.0
    for f in range(6):
        l0 = a.launch_count()
        a.advance(FRAME)
        assert a.launch_count() - l0 <= 2
        b.advance(FRAME)
        pa, pb = a.read_state_f64()[0], b.read_state_f64()[0]
        disp = np.abs(pb - x0).max()
        worst = max(worst, np.abs(pa - pb).max() / disp)
    assert worst <= (1e-6 if name.endswith("fp64") else 1e-4), worst
    assert a.stepCount() == b.stepCount() == 6 * 34
    if name.startswith("tangle"):
        na, _, _ = a.debug_contacts()
        assert na.sum() > 0
    a.close()
    b.close()
