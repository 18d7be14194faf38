"""GPU parity on the paths the benchmark times and on the reference's non-default schedules.

The batched workload detects contacts every substep but rebuilds the BVH only every 0.1 s of
simulated time (KittenEngine/YarnBall/sim/collision.cu:101-108), so about 99 % of its
detections run on a refitted tree; these tests compare that path, and the schedule switches of
MetaData (detectionPeriod, numItr, useStepSizeLimit, useVelocityRadius: step.cpp:46-50,
collision.cu:160-171), with the CPU oracle.

Tolerances (stated here, used below):
  * contact lists, step limits and the predictor output after detection on a refitted tree:
    bit-exact against the FP32 oracle that follows the engine's precision policy, from the same
    state (positions, velocities, previous velocities);
  * FP64 build against the FP64 oracle after one frame (34 substeps): 1e-9 x segment length;
  * FP32 build against the FP64 oracle after one frame: relative error <= 1e-4,
    max_i |x_gpu - x_fp64| / max_i |x_fp64 - x_start|;
  * FP64 diagnostics against the oracle's FP64 evaluation of the same state and lists: 1e-9
    relative (only the summation order differs).
"""
import numpy as np
import pytest

import oracle
from yarnball_b200 import scenes
from yarnball_b200.sim import Sim

pytestmark = pytest.mark.gpu

SEG = 2e-3
H = 1.0 / 1020.0
FRAME = 1.0 / 30.0


def _oracle_from(sim, mode):
    """Oracle holding the engine's current state: positions, velocities and rotors as the
    host sees them after download(), plus the previous-substep velocities the predictor uses,
    and the engine's step counter (it decides which substeps detect)."""
    sim.download()
    return oracle.from_sim(sim, mode=mode, last_vel=sim.debug_last_vel(), step_counter=sim.stepCount())


def _compare_lists(sim, orc):
    nc_g, lists_g, sl_g = sim.debug_contacts()
    nc_o, lists_o, sl_o = orc.contacts()
    assert np.array_equal(nc_g, nc_o)
    for i in np.nonzero(nc_g)[0]:
        assert np.array_equal(lists_g[i], lists_o[i]), i
    segs = (sim.verts["flags"] & 2) != 0
    assert np.array_equal(sl_g[segs], sl_o[segs].astype(np.float32))
    return nc_g


def _refit_detection_bit_exact(sim, frames):
    for _ in range(frames):
        sim.advance(FRAME)
    # every detection since the first substep ran on a refit of the tree built then
    assert sim.stepCount() < 102
    orc = _oracle_from(sim, oracle.FP32_MIXED)
    sim.debug_phases(1 | 4, H)  # predictor, then detection on the refitted tree
    orc.phases(1 | 2, H)        # predictor, then the oracle's own (grid) detection
    assert np.array_equal(sim.debug_dx().astype(np.float32), orc.state()["dx"].astype(np.float32))
    nc = _compare_lists(sim, orc)
    assert nc.sum() > 0
    return nc


def test_refit_detection_pile_bit_exact():
    """A pile that has moved for two frames: the pair set found on the refitted tree equals
    the oracle's, bit for bit, with nonzero velocities in the predictor and velocity radii."""
    sim = scenes.build_pile(seed=9, yarns=96, verts=64, cube=0.03)
    nc = _refit_detection_bit_exact(sim, 2)
    assert nc.mean() > 2
    sim.close()


def test_refit_detection_batch_bit_exact():
    """The same on a sample of the batched workload (24 scenes of uneven size)."""
    spec = scenes.batched_spec(seed=7, num_scenes=24, cap=1500000)
    assert len(spec[0]) >= 20
    sim, _ = scenes.build_batched(seed=7, spec=spec)
    _refit_detection_bit_exact(sim, 2)
    sim.close()


def _dense_pile(precision, meta=None, yarns=96, verts=64, seed=9):
    return scenes.build_pile(seed=seed, yarns=yarns, verts=verts, cube=0.03, precision=precision, meta=meta)


VARIANTS = {
    "detectionPeriod2": dict(detectionPeriod=2),
    "detectionPeriod4": dict(detectionPeriod=4),
    "numItr4": dict(numItr=4),
    "noStepSizeLimit": dict(useStepSizeLimit=0),
    "noVelocityRadius": dict(useVelocityRadius=0),
    # the settings of the reference's example scenes (KittenEngine/configs/letterS.json)
    "letterS": dict(numItr=4, detectionPeriod=4, detectionScaler=1.1),
}


def _rel_err(pos, ref, x0):
    return np.abs(pos - ref).max() / np.abs(ref - x0).max()


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_schedule_variant_vs_fp64_oracle(name):
    """Each schedule switch, one frame on the contact-heavy dense pile: the FP64 build follows
    the FP64 oracle to 1e-9 x segment length, the FP32 build to 1e-4 relative."""
    meta = VARIANTS[name]
    maxH = 4e-4 if name == "letterS" else 1e-3
    for prec in ("fp64", "fp32"):
        sim = _dense_pile(prec, meta)
        sim.maxH = maxH
        x0 = sim.read_state_f64()[0]
        orc = oracle.from_sim(sim, mode=oracle.FP64)
        sim.advance(FRAME)
        orc.advance(FRAME, maxH)
        pos = sim.read_state_f64()[0]
        ref = orc.state()["pos"]
        if prec == "fp64":
            assert np.abs(pos - ref).max() <= 1e-9 * SEG, (name, np.abs(pos - ref).max())
        else:
            assert _rel_err(pos, ref, x0) <= 1e-4, (name, _rel_err(pos, ref, x0))
        sim.close()
        orc.close()


def _dense_batch(precision, num_scenes=24, seed=21):
    """A batch of small, dense pile scenes (2.2 cm cubes) of uneven size: contact-heavy."""
    rng = np.random.default_rng(seed)
    yarns = rng.integers(6, 24, size=num_scenes)
    verts = rng.integers(40, 96, size=num_scenes)
    counts = [int(y * v) for y, v in zip(yarns, verts)]
    sim = Sim(scenes=counts, precision=precision)
    off = 0
    for s in range(num_scenes):
        lens = np.full(int(yarns[s]), int(verts[s]), np.int32)
        pos = scenes.random_walks(seed * 1000 + s, lens, cube=0.022)
        scenes.fill_yarns(sim, pos, lens, offset=off)
        off += counts[s]
    sim.set_meta_all(**scenes.PILE_META)
    sim.configure()
    for s in range(num_scenes):
        sim.setKBend(float(10 ** rng.uniform(-9, -7)), scene=s)
    sim.setKStretch(2e-2)
    sim.maxH = 1e-3
    sim.upload()
    return sim


def test_contact_heavy_batch_full_frame_vs_fp64_oracle():
    """A full frame of a contact-heavy batch (24 scenes, mean contact list > 3 entries): the
    FP64 build against the FP64 oracle to 1e-9 x segment length, and the FP32 build (the
    production precision) against the FP64 oracle to 1e-4 relative."""
    for prec in ("fp64", "fp32"):
        sim = _dense_batch(prec)
        x0 = sim.read_state_f64()[0]
        orc = oracle.from_sim(sim, mode=oracle.FP64)
        sim.advance(FRAME)
        orc.advance(FRAME, 1e-3)
        nc, _, _ = sim.debug_contacts()
        segs = (sim.verts["flags"] & 2) != 0
        assert nc[segs].mean() > 3, nc[segs].mean()
        pos = sim.read_state_f64()[0]
        ref = orc.state()["pos"]
        if prec == "fp64":
            assert np.abs(pos - ref).max() <= 1e-9 * SEG, np.abs(pos - ref).max()
        else:
            assert _rel_err(pos, ref, x0) <= 1e-4, _rel_err(pos, ref, x0)
        sim.close()
        orc.close()


def _pinned_scene(yarns):
    """Straight pinned yarns given as (start, end, vertex count) triples (nothing moves)."""
    counts = [v for _, _, v in yarns]
    sim = Sim(int(sum(counts)))
    off = 0
    for a, b, v in yarns:
        t = np.linspace(0.0, 1.0, v)[:, None]
        p = (np.asarray(a, np.float64) * (1 - t) + np.asarray(b, np.float64) * t).astype(np.float32)
        scenes.fill_yarns(sim, p, [v], offset=off, pin_first=True, pin_last=True)
        sim.verts["invMass"][off:off + v] = 0.0
        off += v
    for k, val in scenes.PILE_META.items():
        setattr(sim.meta, k, val)
    sim.configure()
    sim.setKBend(1e-8)
    sim.setKStretch(2e-2)
    sim.upload()
    return sim


def test_contact_overflow_is_reported_clamped_and_recoverable():
    """More than MAX_COLLISIONS_PER_SEGMENT (128) contacts on one segment: advance reports
    the reference's error (collision.cu:81-90, YarnBall.cu:283-286), the list holds 128 valid,
    distinct partners, and once the input is fixed the simulation runs on without error."""
    spine = ((0.0, 0.0, 0.0), (0.15, 0.0, 0.0), 2)  # one 15 cm segment
    crossers = [((1e-3 + 6e-4 * k, 3e-4, -1e-3), (1e-3 + 6e-4 * k, 3e-4, 1e-3), 3) for k in range(200)]
    sim = _pinned_scene([spine] + crossers)
    sim.printErrors = False
    with pytest.raises(RuntimeError):
        sim.advance(1e-3)
    assert sim.lastErrorCode == Sim.ERROR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED
    nc, lists, _ = sim.debug_contacts()
    assert nc[0] == 128
    part = lists[0]
    assert len(np.unique(part)) == 128
    segs = np.nonzero((sim.verts["flags"] & 2) != 0)[0]
    assert np.all(np.isin(part, segs)) and np.all(part >= 2)
    # the lists of the crossing segments stay within the cap
    assert nc[1:].max() <= 128
    # fix the input: lift the crossing yarns 5 cm away from the spine
    sim.download()
    sim.verts["pos"][2:, 1] += 0.05
    sim.upload()
    sim.advance(1e-3)
    nc2, _, _ = sim.debug_contacts()
    assert nc2[0] == 0 and nc2.max() < 128
    sim.close()


def test_interpenetration_warning_on_hard_core_contact():
    """Two crossing segments whose centre-lines are 30 um apart (2 radius = 50 um): advance
    raises WARNING_SEGMENT_INTERPENETRATION (YarnBall.h:121) and counts the contact."""
    a = ((-4e-3, 0.0, 0.0), (4e-3, 0.0, 0.0), 5)
    b = ((0.0, 3e-5, -2e-3), (0.0, 3e-5, 2e-3), 3)
    sim = _pinned_scene([a, b])
    assert sim.lastWarningCode == Sim.ERROR_NONE
    sim.advance(1e-3)
    assert sim.lastWarningCode == Sim.WARNING_SEGMENT_INTERPENETRATION
    assert sim.penetrations() >= 1
    assert abs(sim.min_pair_distance() - 3e-5) < 1e-7
    sim.close()
    # the same pair 80 um apart touches the barrier but not the hard cores: no warning
    b = ((0.0, 8e-5, -2e-3), (0.0, 8e-5, 2e-3), 3)
    sim = _pinned_scene([a, b])
    sim.advance(1e-3)
    assert sim.lastWarningCode == Sim.ERROR_NONE and sim.penetrations() == 0
    sim.close()


def test_diagnostics_vs_oracle_fp64_evaluation():
    """yb_diagnostics (FP64 energies, max speed, min gap, pair count) on a moving contact-heavy
    pile equals the oracle's FP64 evaluation of the same state and contact lists."""
    sim = _dense_pile("fp32")
    for _ in range(2):
        sim.advance(FRAME)
    orc = _oracle_from(sim, oracle.FP32_MIXED)
    sim.debug_phases(1 | 4, H)
    orc.phases(1 | 2, H)
    _compare_lists(sim, orc)
    g = sim.diagnostics()
    o = orc.diagnostics()
    for key in ("kinetic", "gravity", "stretch", "bend", "barrier", "max_speed", "min_gap", "pairs"):
        assert np.isfinite(g[key]), key
        assert abs(g[key] - o[key]) <= 1e-9 * max(abs(o[key]), 1e-30), (key, g[key], o[key])
    assert g["kinetic"] > 0 and g["barrier"] > 0 and g["pairs"] > 0
    sim.close()


@pytest.mark.parametrize("which", ["pile", "batch"])
def test_packet_and_per_query_traversal_give_the_same_lists(which):
    """The three broadphase walks (per warp of 32 queries, the default; per query; per query
    with the warp's node records loaded cooperatively) keep the same pairs, on a rebuilt and on
    a refitted tree; all equal the oracle's."""
    if which == "pile":
        build = lambda: scenes.build_pile(seed=1)  # noqa: E731  (the full 262,144-vertex pile)
    else:
        spec = scenes.batched_spec(seed=7, num_scenes=24, cap=1500000)
        build = lambda: scenes.build_batched(seed=7, spec=spec)[0]  # noqa: E731
    out = {}
    for packet in (1, 0, 2):
        sim = build()
        sim.set_traversal(packet)
        sim.advance(FRAME)
        orc = _oracle_from(sim, oracle.FP32_MIXED)
        sim.debug_phases(1 | 4, H)  # refitted tree
        orc.phases(1 | 2, H)
        _compare_lists(sim, orc)
        sim.debug_phases(2)         # rebuilt tree on the same state
        out[packet] = sim.debug_contacts()
        _compare_lists(sim, orc)
        sim.close()
        orc.close()
    assert np.array_equal(out[1][0], out[0][0]) and np.array_equal(out[1][0], out[2][0])


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_packed_lists_equal_the_sorted_rows(precision):
    """The list pass packs every vertex's sorted contact row into consecutive slots in vertex
    order (what the Newton kernels read): the offsets are the running sum of the list lengths,
    each vertex's slots hold exactly its sorted row, after a detection on a refitted tree and
    after a list pass without detection."""
    spec = scenes.batched_spec(seed=7, num_scenes=24, cap=1500000)
    sim = scenes.build_batched(seed=7, spec=spec, precision=precision)[0]
    sim.advance(FRAME)
    for mask in (1 | 4, 8):
        sim.debug_phases(mask, H)
        nc, rows, _ = sim.debug_contacts(raw=True)
        off, cols = sim.debug_packed_contacts()
        assert off[0] == 0 and np.all(np.diff(off.astype(np.int64)) == nc)
        assert int(off[-1]) == int(nc.sum()) > 0
        with_c = np.nonzero(nc)[0]
        assert np.array_equal(cols, np.concatenate([rows[k] for k in with_c]))
        # each row ascending (the list pass sorted it): every step inside a row increases
        inside = np.ones(len(cols), bool)
        inside[off[with_c].astype(np.int64)] = False
        assert np.all(np.diff(cols.astype(np.int64))[inside[1:]] > 0)
    sim.close()
