"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle.

Tolerances (stated here, used below):
  * positions after one substep: max |x_gpu - x_fp64| <= 1e-5 x segment length
  * orientations after one substep: max angle(q_gpu, q_fp64) <= 1e-5 rad
  * after one frame (34 substeps): relative error <= 1e-4, measured as
    max_i |x_gpu - x_fp64| / max_i |x_fp64 - x_start|  (error relative to the motion)
  * contact lists and step limits after detection: bit-exact against the FP32 oracle that
    follows the engine's precision policy (same positions and predictor output)
  * FP64 build against the FP64 oracle: 1e-9 x segment length
"""
import numpy as np
import pytest

import oracle
import yarnball_b200 as yb
from yarnball_b200 import scenes

pytestmark = pytest.mark.gpu

SEG = 2e-3
H = 1.0 / 1020.0


def quat_angle(q1, q2):
    q1 = q1 / np.linalg.norm(q1, axis=1, keepdims=True)
    q2 = q2 / np.linalg.norm(q2, axis=1, keepdims=True)
    s = np.sign(np.sum(q1 * q2, axis=1, keepdims=True))
    s[s == 0] = 1
    a = np.linalg.norm(q1 - s * q2, axis=1)
    b = np.linalg.norm(q1 + s * q2, axis=1)
    return 2 * np.arctan2(a, b)


def seg_rows(sim):
    return (sim.verts["flags"] & 2) != 0


def test_sort_matches_stable_argsort():
    rng = np.random.default_rng(3)
    for n, bits in [(1, 30), (7, 30), (2048, 30), (2049, 39), (100003, 39), (300000, 64)]:
        keys = rng.integers(0, 2**min(bits, 63), size=n, dtype=np.uint64)
        keys[: n // 3] = keys[0]  # many duplicates: stability matters
        vals = np.arange(n, dtype=np.int32)
        ko, vo = yb.sort_pairs(keys, vals, bits)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(ko, keys[order]), (n, bits)
        assert np.array_equal(vo, vals[order]), (n, bits)


def test_readme_one_substep_vs_fp64():
    sim = scenes.build_readme()
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    sim.advance(1e-3)  # exactly one substep
    orc.advance(1e-3, 1e-3)
    pos, vel, q = sim.read_state_f64()
    ref = orc.state()
    perr = np.abs(pos - ref["pos"]).max()
    assert perr <= 1e-5 * SEG, perr
    qerr = quat_angle(q[seg_rows(sim)], ref["q"][seg_rows(sim)]).max()
    assert qerr <= 1e-5, qerr


def test_readme_one_frame_rel_err():
    sim = scenes.build_readme()
    x0 = sim.verts["pos"].astype(np.float64).copy()
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    for _ in range(3):
        sim.advance(1 / 30.0)
        orc.advance(1 / 30.0, 1e-3)
    pos, _, q = sim.read_state_f64()
    ref = orc.state()
    rel = np.abs(pos - ref["pos"]).max() / np.abs(ref["pos"] - x0).max()
    assert rel <= 1e-4, rel


def test_readme_fp64_build_vs_fp64_oracle():
    sim = scenes.build_readme(precision="fp64")
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    sim.advance(1 / 30.0)
    orc.advance(1 / 30.0, 1e-3)
    pos, _, q = sim.read_state_f64()
    ref = orc.state()
    assert np.abs(pos - ref["pos"]).max() <= 1e-9 * SEG
    assert quat_angle(q[seg_rows(sim)], ref["q"][seg_rows(sim)]).max() <= 1e-9


def _compare_detection(sim, orc):
    """Predictor + detection on both sides from identical state; lists and limits bit-exact."""
    sim.debug_phases(1 | 2, H)
    orc.phases(1 | 2, H)
    nc_g, lists_g, sl_g = sim.debug_contacts()
    nc_o, lists_o, sl_o = orc.contacts()
    # the predictor output feeds the filter: it must agree bit for bit first
    dx_g = sim.debug_dx()
    dx_o = orc.state()["dx"]
    assert np.array_equal(dx_g.astype(np.float32), dx_o.astype(np.float32))
    assert np.array_equal(nc_g, nc_o)
    for i in np.nonzero(nc_g)[0]:
        assert np.array_equal(lists_g[i], lists_o[i]), i
    segs = seg_rows(sim)
    assert np.array_equal(sl_g[segs], sl_o[segs].astype(np.float32))
    return int(nc_g.sum())


def test_pile_small_pair_set_bit_exact():
    sim = scenes.build_pile(seed=11, yarns=96, verts=64)
    orc = oracle.from_sim(sim, mode=oracle.FP32_MIXED)
    total = _compare_detection(sim, orc)
    assert total > 0


def test_pile_full_pair_set_bit_exact():
    sim = scenes.build_pile(seed=1)
    orc = oracle.from_sim(sim, mode=oracle.FP32_MIXED)
    total = _compare_detection(sim, orc)
    assert total > 100000


def test_pile_small_substep_vs_fp64():
    sim = scenes.build_pile(seed=5, yarns=64, verts=64)
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    sim.advance(1e-3)
    orc.advance(1e-3, 1e-3)
    pos, _, q = sim.read_state_f64()
    ref = orc.state()
    perr = np.abs(pos - ref["pos"]).max()
    assert perr <= 1e-5 * SEG, perr
    qerr = quat_angle(q[seg_rows(sim)], ref["q"][seg_rows(sim)]).max()
    assert qerr <= 1e-5, qerr


def test_dense_pile_substep_vs_fp64():
    """Contact-heavy: 96 yarns x 64 vertices in a 3 cm cube (segments with more contacts than
    the staged ones exercise both contact paths of the Newton kernel)."""
    sim = scenes.build_pile(seed=9, yarns=96, verts=64, cube=0.03)
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    sim.advance(1e-3)
    orc.advance(1e-3, 1e-3)
    nc, _, _ = sim.debug_contacts()
    assert nc.max() > 8 and nc.mean() > 2
    pos, _, q = sim.read_state_f64()
    ref = orc.state()
    perr = np.abs(pos - ref["pos"]).max()
    assert perr <= 1e-5 * SEG, perr
    qerr = quat_angle(q[seg_rows(sim)], ref["q"][seg_rows(sim)]).max()
    assert qerr <= 1e-5, qerr


SHAPES = [(256, 1, False), (128, 1, False), (256, 2, False), (256, 4, False), (512, 4, False), (256, 8, False),
          (512, 8, False), (128, 1, True), (256, 1, True), (256, 4, True), (128, 0, False), (128, 0, True)]


@pytest.mark.parametrize("shape", SHAPES)
def test_every_newton_kernel_shape_vs_fp64(shape):
    """Each autotuner candidate (threads, lanes per vertex, pipelined; lanes 0 = balanced)
    meets the one-substep tolerance on the contact-heavy dense pile."""
    sim = scenes.build_pile(seed=9, yarns=96, verts=64, cube=0.03)
    sim.set_tuning(shape[0], shape[1], True, shape[2])
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    sim.advance(1e-3)
    orc.advance(1e-3, 1e-3)
    pos, _, q = sim.read_state_f64()
    ref = orc.state()
    assert np.abs(pos - ref["pos"]).max() <= 1e-5 * SEG
    assert quat_angle(q[seg_rows(sim)], ref["q"][seg_rows(sim)]).max() <= 1e-5


def test_batched_equals_alone():
    spec = scenes.batched_spec(seed=5, num_scenes=5, cap=200000, max_yarns=12, min_len=32, max_len=400)
    assert len(spec[0]) == 5
    batch, spec = scenes.build_batched(seed=5, spec=spec)
    batch.advance(1 / 30.0)
    pos_b, _, q_b = batch.read_state_f64()
    for s in range(len(spec[0])):
        alone = scenes.build_scene_alone(spec, s, seed=5)
        alone.advance(1 / 30.0)
        pos_a, _, q_a = alone.read_state_f64()
        o0, o1 = batch.sceneOffsets[s], batch.sceneOffsets[s + 1]
        assert np.array_equal(pos_b[o0:o1], pos_a), s
        assert np.array_equal(q_b[o0:o1], q_a), s
        alone.close()


def test_device_pin_driver_follows_prescribed_rotation():
    """The device-side kinematic driver places driven pins exactly on the prescribed rotation
    (the reference's twist scenario, KittenEngine/main.cpp:54-87, rotateY about +y) and agrees
    with the host-side download/move/upload driver after one frame.  The comparison stops
    after one frame: from the second frame on the host driver's upload() clears every
    vertex's Kahan compensation term (about 1e-7 m at y = 1 m) while the device driver clears
    only the driven pins', and the twisted bundle buckles, which amplifies that difference."""
    a = scenes.build_twist(grid=3, verts=512)
    b = scenes.build_twist(grid=3, verts=512)
    x0 = a.read_state_f64()[0]
    groups, center = scenes.device_twist(a, omega=2 * np.pi)
    drv = scenes.TwistDriver(b, omega=2 * np.pi)
    a.advance(1 / 30.0)
    drv.frame(1 / 30.0)
    pa = a.read_state_f64()[0]
    pb = b.read_state_f64()[0]
    disp = np.abs(pb - x0).max()
    assert disp > 0
    assert np.abs(pa - pb).max() <= 1e-4 * disp
    frames = 3
    for _ in range(frames - 1):
        a.advance(1 / 30.0)
    pa = a.read_state_f64()[0]
    top = groups == 1
    # driven pins at the start of the last frame plus h v over its substeps = rotation at t = frames/30
    ang = 2 * np.pi * frames / 30.0
    c, s = np.cos(ang), np.sin(ang)
    d = x0[top] - center
    expect = np.stack([c * d[:, 0] + s * d[:, 2], d[:, 1], -s * d[:, 0] + c * d[:, 2]], 1) + center
    assert np.abs(pa[top] - expect).max() < 2e-6
    a.close()
    b.close()


def test_upload_rejects_bad_connection_index_and_keeps_the_state():
    """upload() validates connection indices on host threads while the copies run; a bad
    index is rejected before the device state changes, and the simulation stays usable."""
    sim = scenes.build_readme()
    sim.advance(1 / 30.0)
    sim.download()
    before = sim.read_state_f64()[0]
    good = sim.verts["connectionIndex"].copy()
    sim.verts["connectionIndex"][5] = sim.numVerts + 7
    with pytest.raises(RuntimeError):
        sim.upload()
    np.testing.assert_array_equal(sim.read_state_f64()[0], before)
    sim.verts["connectionIndex"][:] = good
    sim.upload()
    sim.advance(1 / 30.0)
    assert np.all(np.isfinite(sim.read_state_f64()[0]))
    sim.close()


def _oracle_residuals(orc, h, iters):
    """The FP64 oracle's largest iterate change per Newton iteration of one substep with
    detection (predictor, detection and step limits, then one iteration at a time)."""
    orc.phases(1 | 2, h)
    prev = orc.state()["dx"][:, :3].copy()
    out = []
    for _ in range(iters):
        orc.phases(16)
        cur = orc.state()["dx"][:, :3].copy()
        out.append(np.linalg.norm(cur - prev, axis=1).max())
        prev = cur
    return np.array(out)


def test_step_residuals_is_a_plain_step():
    """yb_step_residuals advances exactly as yb_step does (bit-exact state, same step count)
    and reports one finite, decreasing-overall residual per Newton iteration."""
    a = scenes.build_pile(seed=5, yarns=64, verts=64)
    b = scenes.build_pile(seed=5, yarns=64, verts=64)
    for _ in range(3):
        r = a.step_residuals()
        b.step()
        assert len(r) == a.meta.numItr
        assert np.all(np.isfinite(r)) and r[-1] < r[0]
    assert a.stepCount() == b.stepCount() == 3
    for x, y in zip(a.read_state_f64(), b.read_state_f64()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_step_residuals_fp64_vs_fp64_oracle():
    """The FP64 build's per-iteration residuals equal the FP64 oracle's to 1e-8 of the first."""
    sim = scenes.build_pile(seed=5, yarns=64, verts=64, precision="fp64")
    orc = oracle.from_sim(sim, mode=oracle.FP64)
    r = sim.step_residuals()
    ref = _oracle_residuals(orc, 1e-3, len(r))
    assert np.abs(r - ref).max() <= 1e-8 * ref[0], (r, ref)
    sim.close()


def test_min_pair_distance_is_the_listed_minimum():
    """The running minimum of the contacts' centre-line distances equals an FP64 evaluation
    over the listed contacts (within 1e-7 m: FP32 relative coordinates), and starts at +inf."""
    from tests.np_ref import closest

    sim = scenes.build_pile(seed=9, yarns=96, verts=64, cube=0.03)
    assert sim.min_pair_distance() == np.inf
    sim.debug_phases(1 | 2, H)
    pos = sim.read_state_f64()[0]
    nc, lists, _ = sim.debug_contacts()
    best = np.inf
    for i in np.nonzero(nc)[0]:
        a0 = pos[i]
        a1 = pos[i + 1] - a0
        for j in lists[i]:
            b0, b1 = pos[j] - a0, pos[j + 1] - a0
            u, v = closest(a1, b0, b1)
            best = min(best, float(np.linalg.norm(u * a1 - (b0 * (1 - v) + b1 * v))))
    got = sim.min_pair_distance()
    assert np.isfinite(best) and abs(got - best) <= 1e-7, (got, best)
    sim.advance(1 / 30.0)
    assert 0.0 < sim.min_pair_distance() <= got
    sim.close()


def test_stored_contact_lists_are_sorted():
    """The list pass sorts every contact list in place (by its thread up to 16 entries, by
    its warp beyond): on the full pile, with lists of more than 16 entries, every stored list
    is strictly increasing and the pair set is that of the FP32 oracle."""
    sim = scenes.build_pile(seed=1)
    orc = oracle.from_sim(sim, mode=oracle.FP32_MIXED)
    _compare_detection(sim, orc)
    nc, lists, _ = sim.debug_contacts(raw=True)
    assert nc.max() > 16
    for i in np.nonzero(nc)[0]:
        assert np.all(np.diff(lists[i]) > 0), i
    sim.close()
