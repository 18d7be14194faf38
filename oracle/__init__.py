"""CPU oracle bindings (test infrastructure only).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker; never
by the product.  The oracle is a C++/OpenMP restatement of the reference's substep
(oracle/yb_oracle.cpp).  It is pinned to the reference's own kernels, compiled unchanged from
the reference's sources for the GPU by oracle/refbuild and run through oracle/reference.py.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libyb_oracle.so")

FP64, FP32, FP32_MIXED = 0, 1, 2

_d = ctypes.POINTER(ctypes.c_double)
_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int32)
_v = ctypes.c_void_p

_SIG = {
    "orc_configure": (ctypes.c_int, [ctypes.c_int, ctypes.c_float, _v, _f, _f, _f, _f, _f]),
    "orc_set_kstretch": (None, [ctypes.c_int, _v, ctypes.c_float]),
    "orc_set_kbend": (None, [ctypes.c_int, _v, _f, ctypes.c_float]),
    "orc_upload_meta": (ctypes.c_int, [_v]),
    "orc_create": (_v, [ctypes.c_int, ctypes.c_int]),
    "orc_destroy": (None, [_v]),
    "orc_set_state": (None, [_v, _v, _f, _f, _f, _i, ctypes.c_int, _v]),
    "orc_set_meta": (None, [_v, ctypes.c_int, _v]),
    "orc_set_last_vel": (None, [_v, _d]),
    "orc_set_schedule": (None, [_v, ctypes.c_uint64]),
    "orc_advance": (ctypes.c_int, [_v, ctypes.c_float, ctypes.c_float]),
    "orc_phases": (ctypes.c_int, [_v, ctypes.c_int, ctypes.c_float]),
    "orc_get_state": (None, [_v, _d, _d, _d, _d, _d]),
    "orc_get_contacts": (None, [_v, _i, _i, _d]),
    "orc_diagnostics": (None, [_v, _d]),
    "orc_penetrations": (ctypes.c_int64, [_v]),
    "orc_set_threads": (None, [ctypes.c_int]),
    "orc_max_threads": (ctypes.c_int, []),
    "orc_math": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _f, _f, _f, _f, _f, _f]),
}

_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    # the reference's own kernels (oracle/_ref), when the reference's sources are present
    from .refbuild import build as refbuild

    refbuild.build()


def load():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIG.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def _p(a, t):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(t))


def meta_bytes(meta_struct):
    """The engine's YbMeta and the oracle's orc_meta share one layout."""
    return ctypes.string_at(ctypes.addressof(meta_struct), ctypes.sizeof(meta_struct))


def configure(verts, qs, qRests, density=1e-3):
    """Host setup (YarnBall.cu:91-157) on copies; returns (status, verts, qs, qRests, invMass0, maxSeg, minSeg)."""
    lib = load()
    v = np.ascontiguousarray(verts.copy())
    q = np.ascontiguousarray(np.array(qs, np.float32, copy=True))
    qr = np.ascontiguousarray(np.array(qRests, np.float32, copy=True))
    im = np.zeros(len(v), np.float32)
    mx, mn = ctypes.c_float(), ctypes.c_float()
    st = lib.orc_configure(len(v), density, v.ctypes.data, _p(q, ctypes.c_float), _p(qr, ctypes.c_float),
                           _p(im, ctypes.c_float), ctypes.byref(mx), ctypes.byref(mn))
    return st, v, q, qr, im, mx.value, mn.value


def set_kstretch(verts, k):
    load().orc_set_kstretch(len(verts), verts.ctypes.data, k)


def set_kbend(verts, qRests, k):
    load().orc_set_kbend(len(verts), verts.ctypes.data, _p(qRests, ctypes.c_float), k)


_SCENES = None


def random_walks_batch(seed, yarns_per_scene, yarn_lengths, seg_len=2e-3, cube=0.1, sigma=0.3, min_dist=None):
    """The seeded batched random-walk geometry (yb_scene_random_walks_batch) from the host-only
    build of the scene generator (no CUDA library loaded); same output as the engine's."""
    global _SCENES
    if _SCENES is None:
        path = os.path.join(HERE, "_build", "libyb_scenes.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.yb_scene_random_walks_batch.restype = ctypes.c_int
        lib.yb_scene_random_walks_batch.argtypes = [ctypes.c_uint64, ctypes.c_int32, _i, _i, ctypes.c_float,
                                                    ctypes.c_float, ctypes.c_float, ctypes.c_float, _f, ctypes.c_int32]
        _SCENES = lib
    if min_dist is None:  # 2 radius + 0.1 barrierThickness at yarn radius 0.5 mm
        min_dist = float(2 * np.float32(0.05 * 0.5e-3) + 0.1 * np.float32(1.9 * 0.5e-3))
    yps = np.ascontiguousarray(yarns_per_scene, dtype=np.int32)
    lens = np.ascontiguousarray(yarn_lengths, dtype=np.int32)
    out = np.zeros((int(lens.sum()), 3), np.float32)
    st = _SCENES.yb_scene_random_walks_batch(int(seed), len(yps), _p(yps, ctypes.c_int32), _p(lens, ctypes.c_int32),
                                             seg_len, cube, sigma, min_dist, _p(out, ctypes.c_float), 0)
    if st != 0:
        raise RuntimeError("batched random walk generation failed (%d)" % st)
    return out


def set_threads(t):
    load().orc_set_threads(int(t))


def max_threads():
    return int(load().orc_max_threads())


class OracleSim:
    """State + substep of the restated algorithm (FP64, FP32 or FP32 with the engine's policy)."""

    def __init__(self, verts, vels, qs, qRests, metas, mode=FP64, scene_of=None, last_vel=None, step_counter=0):
        self.lib = load()
        n = len(verts)
        self.n = n
        self.h = self.lib.orc_create(n, mode)
        v = np.ascontiguousarray(verts)
        vel = np.ascontiguousarray(vels, dtype=np.float32)
        q = np.ascontiguousarray(qs, dtype=np.float32)
        qr = np.ascontiguousarray(qRests, dtype=np.float32)
        mb = b"".join(meta_bytes(m) for m in metas)
        mbuf = ctypes.create_string_buffer(mb, len(mb))
        so = None
        if scene_of is not None:
            so = np.ascontiguousarray(scene_of, dtype=np.int32)
        self.lib.orc_set_state(self.h, v.ctypes.data, _p(vel, ctypes.c_float), _p(q, ctypes.c_float),
                               _p(qr, ctypes.c_float), _p(so, ctypes.c_int32) if so is not None else None,
                               len(metas), ctypes.cast(mbuf, ctypes.c_void_p))
        if last_vel is not None:
            lv = np.ascontiguousarray(last_vel, dtype=np.float64)
            self.lib.orc_set_last_vel(self.h, _p(lv, ctypes.c_double))
        if step_counter:
            self.lib.orc_set_schedule(self.h, int(step_counter))

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def advance(self, dt, maxH=1e-3):
        return self.lib.orc_advance(self.h, float(dt), float(maxH))

    def phases(self, mask, h=0.0):
        return self.lib.orc_phases(self.h, int(mask), float(h))

    def state(self):
        n = self.n
        pos = np.zeros((n, 3)); vel = np.zeros((n, 3)); q = np.zeros((n, 4)); dx = np.zeros((n, 4)); lv = np.zeros((n, 3))
        self.lib.orc_get_state(self.h, _p(pos, ctypes.c_double), _p(vel, ctypes.c_double), _p(q, ctypes.c_double),
                               _p(dx, ctypes.c_double), _p(lv, ctypes.c_double))
        return dict(pos=pos, vel=vel, q=q, dx=dx[:, :3].copy(), lastVel=lv)

    def contacts(self):
        n = self.n
        nc = np.zeros(n, np.int32)
        cols = np.zeros(n * 128, np.int32)
        sl = np.zeros(n, np.float64)
        self.lib.orc_get_contacts(self.h, _p(nc, ctypes.c_int32), _p(cols, ctypes.c_int32), _p(sl, ctypes.c_double))
        lists = [cols[i + n * np.arange(nc[i])].copy() for i in range(n)]
        return nc, lists, sl

    def diagnostics(self):
        out = np.zeros(8)
        self.lib.orc_diagnostics(self.h, _p(out, ctypes.c_double))
        keys = ["kinetic", "gravity", "stretch", "bend", "barrier", "max_speed", "min_gap", "pairs"]
        return dict(zip(keys, out.tolist()))

    def penetrations(self):
        return int(self.lib.orc_penetrations(self.h))


class OrcMeta(ctypes.Structure):
    """orc_meta (same layout as the reference MetaData host fields)."""

    _fields_ = [
        ("gravity", ctypes.c_float * 3), ("numItr", ctypes.c_int32), ("worldFloorNormal", ctypes.c_float * 3),
        ("worldFloorPos", ctypes.c_float), ("h", ctypes.c_float), ("lastH", ctypes.c_float), ("time", ctypes.c_float),
        ("numVerts", ctypes.c_int32), ("damping", ctypes.c_float), ("drag", ctypes.c_float),
        ("frictionCoeff", ctypes.c_float), ("kCollision", ctypes.c_float), ("kFriction", ctypes.c_float),
        ("detectionRadius", ctypes.c_float), ("scaledDetectionRadius", ctypes.c_float), ("radius", ctypes.c_float),
        ("accelerationRatio", ctypes.c_float), ("barrierThickness", ctypes.c_float),
        ("detectionScaler", ctypes.c_float), ("bvhRebuildPeriod", ctypes.c_float), ("detectionPeriod", ctypes.c_int32),
        ("maxSegLen", ctypes.c_float), ("minSegLen", ctypes.c_float), ("useStepSizeLimit", ctypes.c_int32),
        ("useVelocityRadius", ctypes.c_int32),
    ]


VERTEX_DTYPE = np.dtype([("pos", "<f4", (3,)), ("invMass", "<f4"), ("lRest", "<f4"), ("kStretch", "<f4"),
                         ("connectionIndex", "<i4"), ("flags", "<u4")])


def default_meta(n, maxH=1e-3):
    """Sim::Sim defaults, YarnBall.cu:14-35."""
    m = OrcMeta()
    m.gravity[:] = [0.0, -9.8, 0.0]
    m.numVerts = n
    m.h = maxH
    m.drag = 0.2
    m.damping = 1e-6
    m.radius = 1e-4
    m.barrierThickness = 8e-4
    m.accelerationRatio = 1.0
    m.kCollision = 1e-5
    m.detectionScaler = 1.2
    m.frictionCoeff = 0.1
    m.kFriction = 5.0
    m.detectionPeriod = 1
    m.useStepSizeLimit = 1
    m.useVelocityRadius = 1
    m.bvhRebuildPeriod = 0.1
    m.numItr = 8
    return m


def default_vertices(n):
    """Per-vertex defaults of Sim::Sim (YarnBall.cu:42-50)."""
    v = np.zeros(n, VERTEX_DTYPE)
    v["invMass"] = 1.0
    v["lRest"] = 1.0
    v["kStretch"] = 100.0
    v["connectionIndex"] = -1
    v["flags"] = 2
    v["flags"][-1] = 0
    q = np.zeros((n, 4), np.float32)
    q[:, 3] = 1.0
    qr = np.zeros((n, 4), np.float32)
    qr[:, 3] = 5.0
    return v, q, qr


def prepare_scene(pos, lens, kbend, meta_fields, kstretch=2e-2, density=1e-3, pin_first=True, pin_last=False):
    """One scene of yarn polylines set up as the reference host code does (defaults,
    configure, setKBend, setKStretch, uploadMeta); returns (verts, qs, qRests, meta)."""
    n = len(pos)
    v, q, qr = default_vertices(n)
    v["pos"] = pos
    ends = np.cumsum(lens) - 1
    v["flags"][ends] = 0
    if pin_first:
        v["invMass"][ends - np.asarray(lens) + 1] = 0.0
    if pin_last:
        v["invMass"][ends] = 0.0
    m = default_meta(n)
    for k, val in meta_fields.items():
        setattr(m, k, val)
    st, v, q, qr, _, mx, mn = configure(v, q, qr, density)
    if st != 0:
        raise RuntimeError("oracle configure failed (%d)" % st)
    m.maxSegLen, m.minSegLen = mx, mn
    set_kbend(v, qr, kbend)
    set_kstretch(v, kstretch)
    if load().orc_upload_meta(ctypes.addressof(m)) != 0:
        raise RuntimeError("invalid scene parameters")
    return v, q, qr, m


def build_scenes(pos_list, yarn_lengths_list, kbend_list, meta_fields, kstretch=2e-2, density=1e-3, mode=FP32,
                 pin_first=True):
    """Scenes assembled entirely on the oracle side (its own configure restatement): each
    scene is a list of yarn polylines; returns an OracleSim holding all of them."""
    verts, qs, qrs, metas, scene_of = [], [], [], [], []
    for s, (pos, lens, kb) in enumerate(zip(pos_list, yarn_lengths_list, kbend_list)):
        n = len(pos)
        v, q, qr, m = prepare_scene(pos, lens, kb, meta_fields, kstretch, density, pin_first)
        verts.append(v); qs.append(q); qrs.append(qr); metas.append(m)
        scene_of.append(np.full(n, s, np.int32))
    vall = np.concatenate(verts)
    return OracleSim(vall, np.zeros((len(vall), 3), np.float32), np.concatenate(qs), np.concatenate(qrs), metas,
                     mode=mode, scene_of=np.concatenate(scene_of) if len(metas) > 1 else None)


def from_sim(sim, mode=FP64, **kw):
    """Oracle state from a yarnball_b200 Sim's host arrays and parameters (after configure)."""
    metas = [sim.scene_meta(s).as_struct() for s in range(sim.numScenes)]
    scene_of = None
    if sim.numScenes > 1:
        scene_of = np.repeat(np.arange(sim.numScenes, dtype=np.int32), np.diff(sim.sceneOffsets))
    return OracleSim(sim.verts.copy(), sim.vels.copy(), sim.qs.copy(), sim.qRests.copy(), metas, mode=mode,
                     scene_of=scene_of, **kw)
