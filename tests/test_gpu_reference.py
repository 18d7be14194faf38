"""The oracle pinned to the reference's own code.

oracle/refbuild compiles the reference's kernels (KittenEngine/YarnBall/sim/iteration.cu,
collision.cu, cosserat.cu, YarnBall.cu) and math headers (Common.h, Rotor.h, SymMat.h)
unchanged for sm_100a; oracle/reference.py runs them.  These tests compare them with the oracle
(oracle/yb_oracle.cpp) on the same inputs, so that the engine's parity tests against the oracle
are parity with the reference.

Tolerances (stated here, used below):
  * math helpers (closest points, rotor product / rotation / fromTo / normalisation, hess3 update
    and 3x3 solve), the predictor (initItr), the contact lists as sorted sets, the step limits
    and the advection: bit-exact between the oracle's FP32 restatement and the reference's
    kernels built with every multiply and add rounded separately;
  * one substep of the reference's kernels (either build) against the FP64 oracle: positions
    within 1e-4 x segment length; orientations within 1e-3 rad.  The reference updates iterates
    in place (cosseratItr across thread blocks, quaternionLambdaItr across warps, each reading
    neighbours that the same launch may already have updated), so its result depends on thread
    scheduling, changes from run to run, and differs from the strict Jacobi iteration of the
    oracle and the engine by the iteration's residual: on the contact-heavy pile measured
    0.9e-5, 1.35e-5, 1.35e-5 and 2.4e-5 x segment length and 3.4e-5 to 1.2e-4 rad in five runs
    on B200s; 1e-6 x segment length and less on the other scenes;
  * the README scene over 150 frames (5100 substeps), each substep of the reference started
    from its own state and compared with the FP64 oracle's substep from that state: the same
    per-substep bounds.
"""
import numpy as np
import pytest

import oracle
from oracle import reference as R
from yarnball_b200 import scenes

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="reference kernels not built (oracle/_ref)")]

SEG = 2e-3
H = 1.0 / 1020.0


def _same_bits(a, b):
    a = np.ascontiguousarray(a, np.float32).ravel()
    b = np.ascontiguousarray(b, np.float32).ravel()
    return bool(np.all((a.view(np.int32) == b.view(np.int32)) | (np.isnan(a) & np.isnan(b))))


def quat_angle(q1, q2):
    q1 = q1 / np.linalg.norm(q1, axis=1, keepdims=True)
    q2 = q2 / np.linalg.norm(q2, axis=1, keepdims=True)
    s = np.sign(np.sum(q1 * q2, axis=1, keepdims=True))
    s[s == 0] = 1
    return 2 * np.arctan2(np.linalg.norm(q1 - s * q2, axis=1), np.linalg.norm(q1 + s * q2, axis=1))


def _segments(rng, n):
    """Segment pairs relative to a0 = 0 (as every kernel calls the helper), including the
    degenerate cases: parallel, collinear overlapping, zero-length, shared endpoints."""
    x = (rng.standard_normal((n, 12)) * 1e-3).astype(np.float32)
    x[:, :3] = 0
    k = n // 8
    x[:k, 9:12] = x[:k, 6:9] + x[:k, 3:6] * np.float32(0.7)                       # parallel
    x[k:2 * k, 6:9] = x[k:2 * k, 3:6] * np.float32(0.3)                             # collinear overlap
    x[k:2 * k, 9:12] = x[k:2 * k, 3:6] * np.float32(1.6)
    x[2 * k:3 * k, 3:6] = 0                                                         # zero-length a
    x[3 * k:4 * k, 9:12] = x[3 * k:4 * k, 6:9]                                      # zero-length b
    x[4 * k:5 * k, 6:9] = x[4 * k:5 * k, 3:6]                                       # shared endpoint
    return x


def test_math_helpers_bit_exact():
    rng = np.random.default_rng(1)
    n = 20000
    q = rng.standard_normal((n, 4)).astype(np.float32)
    v3a = rng.standard_normal((n, 3)).astype(np.float32)

    def unit(a):
        return (a / np.linalg.norm(a, axis=1, keepdims=True)).astype(np.float32)

    f0, f1 = unit(rng.standard_normal((n, 3))), unit(rng.standard_normal((n, 3)))
    f1[:100] = -f0[:100]  # opposite directions: fromTo's orthogonal-basis branch
    f1[100:200] = f0[100:200]
    h = (rng.standard_normal((n, 6)) * np.float32(0.1) + np.array([5, 5, 5, 0, 0, 0])).astype(np.float32)
    cases = [(0, [_segments(rng, n)]), (1, [q, rng.standard_normal((n, 4))]), (2, [q, v3a]), (3, [f0, f1]),
             (4, [q]), (5, [h, unit(v3a), rng.random((n, 1)), rng.standard_normal((n, 3))])]
    for op, ins in cases:
        r = R.math(op, *ins)
        o = R.oracle_math(op, *ins)
        if isinstance(r, tuple):
            assert _same_bits(r[0], o[0]) and _same_bits(r[1], o[1]), op
        else:
            assert _same_bits(r, o), op


def _engine_state(build, frames):
    sim = build()
    for _ in range(frames):
        sim.advance(1 / 30.0)
    sim.download()
    st = (sim.verts.copy(), sim.vels.astype(np.float32).copy(), sim.qs.copy(), sim.qRests.copy(),
          sim.debug_last_vel().astype(np.float32), sim.scene_meta(0).as_struct())
    sim.close()
    return st


def _pair(state, variant="nofma", mode=oracle.FP32):
    v, vel, q, qr, lv, meta = state
    ref = R.RefSim(v, vel, q, qr, meta, variant=variant)
    ref.write_state(last_vel=lv)
    orc = oracle.OracleSim(v, vel, q, qr, [meta], mode=mode, last_vel=lv.astype(np.float64))
    return ref, orc


SCENES = {
    "dense_pile": lambda: scenes.build_pile(seed=9, yarns=96, verts=64, cube=0.03),
    "readme": lambda: scenes.build_readme(),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_predictor_detection_step_limit_bit_exact(name):
    """initItr, detectCollisions (+ the list filter) and recomputeStepLimit of the reference,
    from a moving state, against the oracle's FP32 restatement: identical bits and sets."""
    state = _engine_state(SCENES[name], 2)
    ref, orc = _pair(state)
    ref.phase(R.PHASE_SET_H, H)
    ref.phase(R.PHASE_INIT)
    orc.phases(1, H)
    st = orc.state()
    assert _same_bits(ref.read("dx"), st["dx"])
    assert _same_bits(ref.read("lastVel"), st["lastVel"])
    ref.phase(R.PHASE_DETECT)
    ref.phase(R.PHASE_STEP_LIMIT)
    orc.phases(2)
    assert not ref.info()["truncated"]
    nc_r, lists_r = ref.lists()
    nc_o, lists_o, sl_o = orc.contacts()
    assert np.array_equal(nc_r, nc_o)
    for i in np.nonzero(nc_r)[0]:
        assert np.array_equal(lists_r[i], lists_o[i]), i
    segs = (state[0]["flags"] & 2) != 0
    assert _same_bits(ref.read("stepLimit")[segs], sl_o[segs])
    if name == "dense_pile":
        assert nc_r.sum() > 1000


def test_advection_bit_exact():
    """endItr (velocity from the iterate, advection) of the reference against the oracle's FP32
    restatement, on the predictor's iterate (identical inputs)."""
    state = _engine_state(SCENES["dense_pile"], 2)
    ref, orc = _pair(state)
    ref.phase(R.PHASE_SET_H, H)
    ref.phase(R.PHASE_INIT)
    orc.phases(1, H)
    ref.phase(R.PHASE_END)
    orc.phases(32)
    st = orc.state()
    assert _same_bits(ref.read("verts")["pos"], st["pos"])
    im = state[0]["invMass"] != 0
    assert _same_bits(ref.read("y")[im], st["vel"][im])


@pytest.mark.parametrize("name", sorted(SCENES))
def test_one_substep_vs_fp64_oracle(name):
    """A whole substep of the reference's kernels (as the reference builds them, and with
    separately rounded operations) against the FP64 oracle from the same state."""
    state = _engine_state(SCENES[name], 2)
    for variant in ("fma", "nofma"):
        ref, orc = _pair(state, variant=variant, mode=oracle.FP64)
        ref.advance(H)
        orc.advance(H, 1e-3)
        st = orc.state()
        pos = ref.read("verts")["pos"].astype(np.float64)
        assert np.abs(pos - st["pos"]).max() <= 1e-4 * SEG, (variant, np.abs(pos - st["pos"]).max())
        segs = (state[0]["flags"] & 2) != 0
        assert quat_angle(ref.read("q")[segs].astype(np.float64), st["q"][segs]).max() <= 1e-3
        ref.close()
        orc.close()


def test_readme_150_frames_every_substep_vs_fp64_oracle():
    """Config 1 as specified: the README scene advanced 150 frames of 1/30 s (5100 substeps)
    by the reference's kernels; every substep is checked against the FP64 oracle's substep
    from the reference's own state at its start."""
    sim = scenes.build_readme()
    sim.download()
    v, vel, q, qr = sim.verts.copy(), sim.vels.astype(np.float32).copy(), sim.qs.copy(), sim.qRests.copy()
    meta = sim.scene_meta(0).as_struct()
    sim.close()
    ref = R.RefSim(v, vel, q, qr, meta, variant="fma")
    h = float(np.float32(1 / 30.0) / np.float32(34))
    worst_p = worst_q = 0.0
    segs = (v["flags"] & 2) != 0
    for f in range(150):
        for s in range(34):
            vr, velr, lvr, qq, m = ref.read("verts"), ref.read("y"), ref.read("lastVel"), ref.read("q"), ref.meta()
            orc = oracle.OracleSim(vr, velr, qq, qr, [m], mode=oracle.FP64, last_vel=lvr.astype(np.float64),
                                   step_counter=34 * f + s)
            assert ref.advance(h) == 0
            orc.advance(h, 1e-3)
            st = orc.state()
            worst_p = max(worst_p, float(np.abs(ref.read("verts")["pos"].astype(np.float64) - st["pos"]).max()))
            worst_q = max(worst_q, float(quat_angle(ref.read("q")[segs].astype(np.float64), st["q"][segs]).max()))
            orc.close()
    assert ref.info()["stepCount"] == 5100
    assert worst_p <= 1e-5 * SEG, worst_p
    assert worst_q <= 1e-5, worst_q
    ref.close()
