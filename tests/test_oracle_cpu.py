"""CPU checks of the oracle: known answers derived independently, and agreement with the
second restatement in tests/np_ref.py.  PARITY UNPINNED: the reference itself cannot run
here and ships no golden vectors, so these checks pin the oracle to mathematics and to an
independent implementation instead."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from tests import np_ref
from yarnball_b200 import scenes


def _meta_dict(m):
    return {f: (list(getattr(m, f)) if isinstance(getattr(m, f), ctypes.Array) else getattr(m, f))
            for f, _ in m._fields_}


def _np_state(v, q, qr):
    n = len(v)
    return dict(pos=v["pos"].astype(np.float64), vel=np.zeros((n, 3)), lastVel=np.zeros((n, 3)),
                q=q.astype(np.float64), qRest=qr.astype(np.float64), invMass=v["invMass"].astype(np.float64),
                lRest=v["lRest"].astype(np.float64), kStretch=v["kStretch"].astype(np.float64),
                cid=v["connectionIndex"].astype(np.int64), flags=v["flags"].astype(np.int64))


# ---- closest points ----------------------------------------------------------------------
def _brute(a1, b0, b1, n=401):
    t = np.linspace(0, 1, n)
    P = t[:, None] * a1[None, :]
    Q = b0[None, :] * (1 - t[:, None]) + b1[None, :] * t[:, None]
    d = np.linalg.norm(P[:, None, :] - Q[None, :, :], axis=2)
    i, j = np.unravel_index(np.argmin(d), d.shape)
    # refine around the grid minimum with a local fine grid
    tu = np.clip(np.linspace(t[i] - 2.0 / n, t[i] + 2.0 / n, 201), 0, 1)
    tv = np.clip(np.linspace(t[j] - 2.0 / n, t[j] + 2.0 / n, 201), 0, 1)
    P = tu[:, None] * a1[None, :]
    Q = b0[None, :] * (1 - tv[:, None]) + b1[None, :] * tv[:, None]
    return np.linalg.norm(P[:, None, :] - Q[None, :, :], axis=2).min()


def _alg_dist(a1, b0, b1):
    u, v = np_ref.closest(a1, b0, b1)
    return np.linalg.norm(u * a1 - (b0 * (1 - v) + b1 * v))


@pytest.mark.parametrize("case", range(40))
def test_closest_points_random_vs_brute_force(case):
    rng = np.random.default_rng(case)
    a1, b0, b1 = rng.normal(size=3), rng.normal(size=3), rng.normal(size=3)
    assert _alg_dist(a1, b0, b1) <= _brute(a1, b0, b1) + 1e-9


def test_closest_points_special_cases():
    x = np.array([1.0, 0.0, 0.0])
    # crossing at distance 0.3 in the middle
    u, v = np_ref.closest(x, np.array([0.5, -1.0, 0.3]), np.array([0.5, 1.0, 0.3]))
    assert abs(u - 0.5) < 1e-12 and abs(v - 0.5) < 1e-12
    # exactly parallel, overlapping: the 0/0 parameter falls back to 0.5 and stays exact
    d = _alg_dist(x, np.array([0.25, 0.2, 0.0]), np.array([1.25, 0.2, 0.0]))
    assert abs(d - 0.2) < 1e-12
    # collinear overlapping segments touch
    assert _alg_dist(x, np.array([0.5, 0.0, 0.0]), np.array([2.0, 0.0, 0.0])) < 1e-12
    # endpoint to endpoint
    d = _alg_dist(x, np.array([2.0, 1.0, 0.0]), np.array([3.0, 2.0, 0.0]))
    assert abs(d - np.sqrt(2.0)) < 1e-12
    # a zero-length segment gives NaN parameters, as the reference formula does; the
    # reference's configure rejects zero-length segments before any of this runs
    u, v = np_ref.closest(x, np.array([0.5, 1.0, 0.0]), np.array([0.5, 1.0, 0.0]))
    assert np.isnan(v)


# ---- barrier --------------------------------------------------------------------------
@pytest.mark.parametrize("d", [1e-3, 3e-3, 0.01, 0.1, 0.5, 0.9, 0.999])
def test_barrier_derivatives_match_finite_differences(d):
    kCol, invb = 1.3e-4, 1.0 / 9.5e-4

    def E(x):
        return -kCol / invb * (x - 1) ** 2 * np.log(x)

    eps = 1e-7 * d
    dE = (E(d + eps) - E(d - eps)) / (2 * eps)
    e2 = 1e-4 * d
    d2E = (E(d + e2) - 2 * E(d) + E(d - e2)) / e2**2
    dH, ff = np_ref.barrier(d, kCol, invb)
    # ff is the force magnitude along the normal per unit distance: -dE/dd * invb
    assert ff == pytest.approx(-dE * invb, rel=1e-6)
    assert dH == pytest.approx(d2E * invb * invb, rel=1e-3)
    assert dH > 0 and ff >= 0  # convex, repulsive


# ---- solve and orientation update ----------------------------------------------------------
def test_quaternion_update_properties():
    rng = np.random.default_rng(0)
    e1 = np.array([1.0, 0.0, 0.0])
    for _ in range(20):
        v = rng.normal(size=3)
        b = rng.normal(size=4)
        lam = np.linalg.norm(v) + np.linalg.norm(b)
        r = np_ref.qmul(np_ref.qmul(np.concatenate([v, [0.0]]), b), np.array([1.0, 0, 0, 0])) + lam * b
        q = r / np.linalg.norm(r)
        assert abs(np.linalg.norm(q) - 1) < 1e-12
        # with a vanishing bending term the update aligns the material axis with -v (the tangent)
        b_small = 1e-9 * b
        lam = np.linalg.norm(v) + np.linalg.norm(b_small)
        r = np_ref.qmul(np_ref.qmul(np.concatenate([v, [0.0]]), b_small), np.array([1.0, 0, 0, 0])) + lam * b_small
        q = r / np.linalg.norm(r)
        t = np_ref.qrot(q, e1)
        assert np.allclose(t, -v / np.linalg.norm(v), atol=1e-6)


# ---- oracle vs the numpy restatement ---------------------------------------------------------
def _compare_one_substep(pos, lens, kbend, meta_fields, tol):
    v, q, qr, m = oracle.prepare_scene(pos, lens, kbend, meta_fields)
    h = float(np.float32(1 / 30.0) / np.float32(34))
    orc = oracle.OracleSim(v, np.zeros((len(v), 3), np.float32), q, qr, [m], mode=oracle.FP64)
    orc.advance(h, h)
    ref = orc.state()
    nc_o, lists_o, sl_o = orc.contacts()
    md = _meta_dict(m)
    md["lastH"] = md["h"]
    md["h"] = float(np.float32(h))
    new, cols, sl = np_ref.substep(_np_state(v, q, qr), md)
    for i in range(len(v)):
        assert list(lists_o[i]) == cols[i]
    assert np.abs(ref["pos"] - new["pos"]).max() <= tol
    assert np.abs(ref["q"] - new["q"]).max() <= 1e-9
    return int(nc_o.sum())


def test_oracle_matches_numpy_readme():
    pos = scenes.readme_positions()
    _compare_one_substep(pos, [32, 32], 1e-8, {"kCollision": 1e-7}, tol=1e-12)


def test_oracle_matches_numpy_contacts():
    lens = np.full(6, 14, np.int32)
    pos = scenes.random_walks(3, lens, cube=0.0125)
    ncont = _compare_one_substep(pos, lens, 1e-8, scenes.PILE_META, tol=1e-11)
    assert ncont > 0


# ---- host setup ------------------------------------------------------------------------
def test_configure_matches_reference_semantics():
    pos = scenes.readme_positions()
    v, q, qr = oracle.default_vertices(64)
    v["pos"] = pos
    v["invMass"][[0, 32, 63]] = 0
    v["flags"][31] = 0
    st, v2, q2, qr2, im, mx, mn = oracle.configure(v, q, qr)
    assert st == 0
    # flags: hasPrev follows the previous hasNext; fixOrientation where no segment starts
    assert v2["flags"][31] == 1 | 8 and v2["flags"][32] == 2 | 4 and v2["flags"][0] == 2 | 4
    assert v2["flags"][30] == 1 | 2  # last segment of yarn 0 has no next orientation
    # rest lengths and lumped masses
    seg = np.linalg.norm(pos[1:] - pos[:-1], axis=1)
    assert np.allclose(v2["lRest"][:31], seg[:31], rtol=1e-6)
    m = 0.5 * 1e-3 * (v2["lRest"][4] + v2["lRest"][5])
    assert v2["invMass"][5] == pytest.approx(1 / m, rel=1e-5)
    assert v2["invMass"][0] == 0 and im[0] == 0
    # frames: q_i e1 is the unit tangent; rest rotors have magnitude 5 before setKBend
    for i in range(31):
        t = np_ref.qrot(q2[i].astype(np.float64), np.array([1.0, 0, 0]))
        assert np.allclose(t, (pos[i + 1] - pos[i]) / seg[i], atol=1e-6)
    assert np.allclose(np.linalg.norm(qr2[:31], axis=1), 5.0, rtol=1e-6)
    # dangling vertex and zero-length segment errors
    v3 = v.copy(); v3["flags"][:] = 0
    assert oracle.configure(v3, q, qr)[0] == 4
    v4 = v.copy(); v4["pos"][5] = v4["pos"][4]
    assert oracle.configure(v4, q, qr)[0] == 5


def test_engine_host_configure_is_bit_exact_with_oracle():
    """The engine's configure (host part) against the oracle's restatement.  On a machine
    without a GPU the engine reports the CUDA error after the host part has run."""
    import yarnball_b200 as yb

    s = yb.Sim(64)
    s.verts["pos"][:] = scenes.readme_positions()
    s.verts["invMass"][[0, 32, 63]] = 0
    s.verts["flags"][31] = 0
    v0, q0, qr0 = s.verts.copy(), s.qs.copy(), s.qRests.copy()
    try:
        s.configure()
    except yb.YarnBallError as e:
        assert e.status == 9  # CUDA unavailable: host part done
    st, v, q, qr, im, mx, mn = oracle.configure(v0, q0, qr0)
    assert st == 0
    assert np.array_equal(v.view(np.uint8), s.verts.copy().view(np.uint8))
    assert np.array_equal(q, s.qs) and np.array_equal(qr, s.qRests)
    assert np.array_equal(im, s.initialInvMasses)


def test_reference_kernel_build():
    """The recipe in oracle/refbuild compiles the reference's own kernels from its sources
    (when they are present here) into oracle/_ref, and the host harness loads and exports its
    entry points without a GPU."""
    from oracle import reference as R
    from oracle.refbuild import build as rb

    if os.path.isdir(os.path.join(rb.reference_root(), "KittenEngine", "YarnBall")):
        assert rb.build()
    if not R.available():
        pytest.skip("reference sources absent and no prebuilt oracle/_ref")
    lib = ctypes.CDLL(R.LIB_PATH)
    for name in R._SIG:
        assert hasattr(lib, name), name
    for p in R.FATBINS.values():
        assert os.path.getsize(p) > 10000


def test_oracle_scene_generator_matches_engine_generator():
    """The host-only build of the scene generator that the CPU reference arm uses gives the
    engine library's geometry, bit for bit."""
    spec = scenes.batched_spec(7, 3, 10**6)
    flat = np.concatenate(spec[1]).astype(np.int32)
    assert np.array_equal(oracle.random_walks_batch(7, spec[0], flat), scenes.random_walks_batch(7, spec[0], flat))
