"""Python mirror of YarnBall::Sim (KittenEngine/YarnBall/YarnBall.h:116-206).

Same names, argument meaning and error behaviour as the C++ class: the host arrays
`verts`, `qs`, `qRests`, `vels` are numpy views of the library-owned host memory, `meta`
reads and writes the MetaData fields, and failures raise RuntimeError (YarnBallError)
where the reference throws std::runtime_error.  All computation happens in the CUDA engine
behind the C ABI.
"""
import ctypes
import os

import numpy as np

from . import _abi
from ._abi import YbMeta, check, ptr


class VertexFlags:
    """YarnBall::VertexFlags, YarnBall.h:34-40."""

    hasPrev = 1
    hasNext = 2
    hasNextOrientation = 4
    fixOrientation = 8
    colliding = 16


MAX_COLLISIONS_PER_SEGMENT = 128


class _MetaView:
    """Attribute access to one scene's MetaData; every write goes through yb_set_meta."""

    def __init__(self, sim, scene):
        object.__setattr__(self, "_sim", sim)
        object.__setattr__(self, "_scene", scene)

    def _get(self):
        m = YbMeta()
        check(self._sim._lib.yb_get_meta(self._sim._h, self._scene, ctypes.byref(m)), "meta")
        return m

    def __getattr__(self, name):
        v = getattr(self._get(), name)
        if isinstance(v, ctypes.Array):
            return np.array(v[:], dtype=np.float32)
        return v

    def __setattr__(self, name, value):
        m = self._get()
        cur = getattr(m, name)
        if isinstance(cur, ctypes.Array):
            for i, x in enumerate(value):
                cur[i] = x
        else:
            setattr(m, name, value)
        check(self._sim._lib.yb_set_meta(self._sim._h, self._scene, ctypes.byref(m)), "meta")

    def as_struct(self):
        return self._get()


class Sim:
    ERROR_NONE = 0
    ERROR_MAX_COLLISIONS_PER_SEGMENT_EXCEEDED = 1
    WARNING_SEGMENT_INTERPENETRATION = 2

    def __init__(self, numVerts=None, *, scenes=None, precision="fp32", _handle=None):
        """Sim(numVerts) as YarnBall.cu:11-51, or a batch of independent scenes
        (scenes = list of vertex counts).  precision: "fp32" or "fp64"."""
        self._lib = _abi.load()
        if _handle is not None:
            self._h = _handle
        else:
            self._h = ctypes.c_void_p()
            prec = {"fp32": 0, "fp64": 1}[precision]
            if scenes is None:
                if numVerts is None:
                    raise ValueError("numVerts or scenes required")
                scenes = [int(numVerts)]
            counts = np.ascontiguousarray(np.asarray(scenes, dtype=np.int32))
            check(self._lib.yb_create_batch(len(counts), ptr(counts, ctypes.c_int32), prec, ctypes.byref(self._h)),
                  "Sim")
        self._bind_views()
        self.meta = _MetaView(self, 0)
        self.printErrors = True

    def _bind_views(self):
        """(Re)creates the numpy views of the host arrays for the current layout."""
        nv, ns, pr = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.yb_info(self._h, ctypes.byref(nv), ctypes.byref(ns), ctypes.byref(pr)))
        self.numScenes = ns.value
        offs = [0]
        for s in range(ns.value):
            f, c = ctypes.c_int32(), ctypes.c_int32()
            check(self._lib.yb_scene_range(self._h, s, ctypes.byref(f), ctypes.byref(c)))
            offs.append(f.value + c.value)
        self.sceneOffsets = np.array(offs, np.int64)
        self.numVerts = nv.value
        self.precision = "fp64" if pr.value == 1 else "fp32"
        vp = ctypes.c_void_p()
        qp, qrp, vlp = _abi.c_float_p(), _abi.c_float_p(), _abi.c_float_p()
        check(self._lib.yb_host_arrays(self._h, ctypes.byref(vp), ctypes.byref(qp), ctypes.byref(qrp),
                                       ctypes.byref(vlp)), "host arrays")
        n = self.numVerts
        raw = (ctypes.c_char * (32 * n)).from_address(vp.value)
        self.verts = np.frombuffer(raw, dtype=_abi.VERTEX_DTYPE, count=n)
        self.qs = np.ctypeslib.as_array(qp, shape=(n, 4))
        self.qRests = np.ctypeslib.as_array(qrp, shape=(n, 4))
        self.vels = np.ctypeslib.as_array(vlp, shape=(n, 3))

    # ---- lifecycle -------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.yb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- parameters ------------------------------------------------------------------
    def scene_meta(self, scene):
        return _MetaView(self, scene)

    def set_meta_all(self, **fields):
        """Sets the same MetaData fields on every scene of a batch."""
        for s in range(self.numScenes):
            mv = self.scene_meta(s)
            for k, v in fields.items():
                setattr(mv, k, v)

    @property
    def maxH(self):
        v = ctypes.c_float()
        check(self._lib.yb_get_max_h(self._h, ctypes.byref(v)))
        return v.value

    @maxH.setter
    def maxH(self, value):
        check(self._lib.yb_set_max_h(self._h, float(value)), "maxH")

    # ---- YarnBall::Sim API -----------------------------------------------------------
    def configure(self, density=1e-3):
        check(self._lib.yb_configure(self._h, float(density)), "configure")

    def setKBend(self, k=3e-9, scene=-1):
        check(self._lib.yb_set_kbend(self._h, int(scene), float(k)), "setKBend")

    def setKStretch(self, k=1e-2, scene=-1):
        check(self._lib.yb_set_kstretch(self._h, int(scene), float(k)), "setKStretch")

    def upload(self):
        check(self._lib.yb_upload(self._h), "upload")

    def download(self):
        check(self._lib.yb_download(self._h), "download")

    def zeroVelocities(self):
        check(self._lib.yb_zero_velocities(self._h), "zeroVelocities")

    def advance(self, dt):
        out = ctypes.c_float()
        st = self._lib.yb_advance(self._h, float(dt), ctypes.byref(out))
        if st != 0 and self.printErrors:
            import sys

            sys.stderr.write("ERROR: %s\n" % self._lib.yb_status_string(st).decode())
        check(st, "advance")
        return out.value

    def step(self, dt=None):
        check(self._lib.yb_step(self._h, float(dt or 0.0)), "step")

    def stepCount(self):
        v = ctypes.c_uint64()
        check(self._lib.yb_step_count(self._h, ctypes.byref(v)))
        return v.value

    def bounds(self, scene=-1):
        b = np.zeros(6, dtype=np.float32)
        check(self._lib.yb_bounds(self._h, int(scene), ptr(b, ctypes.c_float)), "bounds")
        return b[:3].copy(), b[3:].copy()

    def collisionStats(self):
        tot, segs, mx = ctypes.c_uint64(), ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.yb_collision_stats(self._h, ctypes.byref(tot), ctypes.byref(segs), ctypes.byref(mx)))
        return int(tot.value), int(segs.value), int(mx.value)

    def printCollisionStats(self):
        tot, segs, _ = self.collisionStats()
        print("Total collisions: %d" % tot)
        print("Segments with collisions: %d/%d" % (segs, self.numVerts))

    @property
    def lastErrorCode(self):
        e, w = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.yb_last_error(self._h, ctypes.byref(e), ctypes.byref(w)))
        return e.value

    @property
    def lastWarningCode(self):
        e, w = ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.yb_last_error(self._h, ctypes.byref(e), ctypes.byref(w)))
        return w.value

    @property
    def initialInvMasses(self):
        p = _abi.c_float_p()
        c = ctypes.c_int32()
        check(self._lib.yb_initial_inv_masses(self._h, ctypes.byref(p), ctypes.byref(c)))
        if c.value == 0:
            return np.zeros(0, np.float32)
        return np.ctypeslib.as_array(p, shape=(c.value,)).copy()

    # ---- additions -------------------------------------------------------------------
    def set_tuning(self, iterThreads=128, lanesPerVertex=0, useGraphs=True, pipelined=False):
        check(self._lib.yb_set_tuning(self._h, int(iterThreads), int(lanesPerVertex), 1 if pipelined else 0,
                                      1 if useGraphs else 0), "tuning")

    def get_tuning(self):
        t, l, p, g = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(self._lib.yb_get_tuning(self._h, ctypes.byref(t), ctypes.byref(l), ctypes.byref(p), ctypes.byref(g)))
        return t.value, l.value, bool(p.value), bool(g.value)

    def autotune(self):
        """Times every Newton-kernel shape on the current state and keeps the fastest:
        returns (threads, lanes per vertex, pipelined, ms per launch)."""
        t, l, p, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_float()
        check(self._lib.yb_autotune(self._h, ctypes.byref(t), ctypes.byref(l), ctypes.byref(p), ctypes.byref(ms)),
              "autotune")
        return t.value, l.value, bool(p.value), ms.value

    def set_pin_motion(self, groups, motions):
        """Device-side kinematic driver: groups (uint8 per vertex, 0 = free) select one of the
        motions (dicts with center, axis, omega, velocity, tStart, tEnd); None switches it off."""
        if groups is None:
            check(self._lib.yb_set_pin_motion(self._h, None, 0, None), "set_pin_motion")
            return
        g = np.ascontiguousarray(groups, dtype=np.uint8)
        arr = (_abi.YbPinMotion * len(motions))()
        for i, m in enumerate(motions):
            arr[i].center[:] = list(m.get("center", (0, 0, 0)))
            arr[i].axis[:] = list(m.get("axis", (0, 1, 0)))
            arr[i].omega = m.get("omega", 0.0)
            arr[i].velocity[:] = list(m.get("velocity", (0, 0, 0)))
            arr[i].tStart = m.get("tStart", 0.0)
            arr[i].tEnd = m.get("tEnd", 1e30)
        check(self._lib.yb_set_pin_motion(self._h, ptr(g, ctypes.c_uint8), len(motions), arr), "set_pin_motion")

    # ---- files ------------------------------------------------------------------------
    def exportToBCC(self, path, exportAsPolyline=False):
        """Sim::exportToBCC (io/fileExport.cpp:6-63): downloads, then writes every curve."""
        check(self._lib.yb_export_bcc(self._h, os.fsencode(path), int(bool(exportAsPolyline))), "exportToBCC")

    def exportToOBJ(self, path):
        """Sim::exportToOBJ (io/fileExport.cpp:65-100)."""
        check(self._lib.yb_export_obj(self._h, os.fsencode(path)), "exportToOBJ")

    def exportFiberMesh(self, path):
        """Sim::exportFiberMesh (io/fiberMesher.cpp:9-157): fibres and fuzz as OBJ polylines."""
        check(self._lib.yb_export_fiber_mesh(self._h, os.fsencode(path)), "exportFiberMesh")

    def save_state(self, path):
        """Full-state checkpoint; Sim.load_state(path) continues bit-identically."""
        check(self._lib.yb_save_state(self._h, os.fsencode(path)), "save_state")

    @staticmethod
    def load_state(path):
        lib = _abi.load()
        out = ctypes.c_void_p()
        check(lib.yb_load_state(os.fsencode(path), ctypes.byref(out)), "load_state")
        return Sim(_handle=out)

    def glueEndpoints(self, searchRadius):
        """Sim::glueEndpoints (io/jsonBuilder.cpp:174-212) on the host arrays; the nearest-vertex
        search runs on the GPU, joins are applied in ascending endpoint order."""
        check(self._lib.yb_glue_endpoints(self._h, float(searchRadius)), "glueEndpoints")

    def download_scene(self, scene):
        check(self._lib.yb_download_scene(self._h, int(scene)), "download_scene")

    def device_bytes(self):
        v = ctypes.c_uint64()
        check(self._lib.yb_device_bytes(self._h, ctypes.byref(v)))
        return int(v.value)

    @staticmethod
    def gather(sources, recycle=None, capacity=0):
        """A batch made of copies of scenes (sim, scene) taken device to device; reuses the
        device allocation of `recycle` (a batch) when it is large enough, else allocates room
        for max(total, capacity) vertices."""
        lib = _abi.load()
        n = len(sources)
        sims = (ctypes.c_void_p * n)(*[s._h.value for s, _ in sources])
        idx = np.ascontiguousarray([int(k) for _, k in sources], dtype=np.int32)
        out = ctypes.c_void_p()
        rec = recycle._h if recycle is not None else None
        check(lib.yb_batch_gather(n, sims, ptr(idx, ctypes.c_int32), rec, int(capacity), ctypes.byref(out)), "gather")
        if recycle is not None and out.value == recycle._h.value:
            recycle._bind_views()
            return recycle
        return Sim(_handle=out)

    def set_stream(self, stream_handle):
        """Launch on a caller's cudaStream_t (int handle, e.g. torch's stream.cuda_stream); 0 = own."""
        check(self._lib.yb_set_stream(self._h, ctypes.c_void_p(int(stream_handle) or None)), "set_stream")

    PROFILE_CLASSES = ["init", "bvh_rebuild", "bvh_refit", "traverse", "step_limit", "iter", "end"]

    def profile_advance(self, dt):
        """advance(dt) with per-kernel-class device times (ms) and launch counts."""
        ms = np.zeros(7, np.float64)
        ln = np.zeros(7, np.uint64)
        check(self._lib.yb_profile_advance(self._h, float(dt), ptr(ms, ctypes.c_double), ptr(ln, ctypes.c_uint64)),
              "profile_advance")
        return dict(zip(self.PROFILE_CLASSES, ms.tolist())), dict(zip(self.PROFILE_CLASSES, ln.tolist()))

    def launch_count(self):
        v = ctypes.c_uint64()
        check(self._lib.yb_launch_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def penetrations(self):
        v = ctypes.c_int64()
        check(self._lib.yb_penetration_count(self._h, ctypes.byref(v)))
        return int(v.value)

    def min_pair_distance(self):
        """Smallest centre-line distance (m) of any listed contact at substep start since creation."""
        v = ctypes.c_double()
        check(self._lib.yb_min_pair_distance(self._h, ctypes.byref(v)), "min_pair_distance")
        return v.value

    def diagnostics(self):
        """FP64 energies and contact statistics of the device state (see yarnball_b200.h)."""
        out = np.zeros(8, np.float64)
        check(self._lib.yb_diagnostics(self._h, ptr(out, ctypes.c_double)), "diagnostics")
        keys = ["kinetic", "gravity", "stretch", "bend", "barrier", "max_speed", "min_gap", "pairs"]
        return dict(zip(keys, out.tolist()))

    def step_residuals(self):
        """One substep of maxH (as step()) returning the largest iterate change of each Newton
        iteration (FP64, metres)."""
        out = np.zeros(256, np.float64)
        cnt = ctypes.c_int32()
        check(self._lib.yb_step_residuals(self._h, ptr(out, ctypes.c_double), len(out), ctypes.byref(cnt)),
              "step_residuals")
        return out[:min(cnt.value, len(out))].copy()

    def read_state_f64(self):
        n = self.numVerts
        pos = np.zeros((n, 3)); vel = np.zeros((n, 3)); q = np.zeros((n, 4))
        check(self._lib.yb_read_state_f64(self._h, ptr(pos, ctypes.c_double), ptr(vel, ctypes.c_double),
                                          ptr(q, ctypes.c_double)), "read_state")
        return pos, vel, q

    def debug_contacts(self, raw=False):
        """(numCols, lists, stepLimit); each list sorted here, or as stored with raw=True."""
        n = self.numVerts
        nc = np.zeros(n, np.int32)
        cols = np.zeros(n * MAX_COLLISIONS_PER_SEGMENT, np.int32)
        sl = np.zeros(n, np.float32)
        check(self._lib.yb_debug_contacts(self._h, ptr(nc, ctypes.c_int32), ptr(cols, ctypes.c_int32),
                                          ptr(sl, ctypes.c_float)), "contacts")
        rows = cols.reshape(n, MAX_COLLISIONS_PER_SEGMENT)
        lists = [(rows[i, :nc[i]].copy() if raw else np.sort(rows[i, :nc[i]])) if nc[i] else np.zeros(0, np.int32)
                 for i in range(n)]
        return nc, lists, sl

    def debug_dx(self):
        dx = np.zeros((self.numVerts, 4))
        check(self._lib.yb_debug_dx(self._h, ptr(dx, ctypes.c_double)), "dx")
        return dx[:, :3].copy()

    def set_small_path(self, enable=True):
        """Advance simulations of at most 256 vertices with the one-block kernel (one launch
        per advance)."""
        check(self._lib.yb_set_small_path(self._h, 1 if enable else 0), "small path")

    def set_traversal(self, mode=2):
        """Broadphase walk: 2 (default) one per query with the warp's node records loaded
        cooperatively, True / 1 one per warp of 32 queries (packet), False / 0 one per query."""
        m = (1 if mode else 0) if isinstance(mode, bool) else int(mode)
        check(self._lib.yb_set_traversal(self._h, m), "traversal")

    def debug_packed_contacts(self):
        """(offsets, cols): the vertex-ordered packed lists of the last list pass."""
        off = np.zeros(self.numVerts + 1, np.uint32)
        check(self._lib.yb_debug_packed_contacts(self._h, ptr(off, ctypes.c_uint32), None, 0), "packed")
        cols = np.zeros(max(int(off[-1]), 1), np.int32)
        check(self._lib.yb_debug_packed_contacts(self._h, ptr(off, ctypes.c_uint32), ptr(cols, ctypes.c_int32),
                                                 int(off[-1])), "packed")
        return off, cols[:int(off[-1])]

    def debug_last_vel(self):
        lv = np.zeros((self.numVerts, 3))
        check(self._lib.yb_debug_last_vel(self._h, ptr(lv, ctypes.c_double)), "lastVel")
        return lv

    def debug_phases(self, mask, h=0.0):
        check(self._lib.yb_debug_phases(self._h, int(mask), float(h)), "phases")


def sort_pairs(keys, vals, bits):
    """Device radix sort of (uint64 key, int32 value) pairs by the low `bits` bits."""
    lib = _abi.load()
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    v = np.ascontiguousarray(vals, dtype=np.int32)
    ko = np.zeros_like(k)
    vo = np.zeros_like(v)
    check(lib.yb_debug_sort_pairs(ptr(k, ctypes.c_uint64), ptr(v, ctypes.c_int32), len(k), int(bits),
                                  ptr(ko, ctypes.c_uint64), ptr(vo, ctypes.c_int32)), "sort")
    return ko, vo


# ---- scene construction from files (io/reader.cpp, io/jsonBuilder.cpp) --------------------

def _io_check(status, where):
    if status != 0:
        msg = load_io_error()
        raise _abi.YarnBallError(status, where + (": " + msg if msg else ""))


def load_io_error():
    m = _abi.load().yb_last_io_error()
    return m.decode() if m else ""


def _transform(transform):
    """A 4x4 matrix in the usual row/column convention (applied as M @ [x, y, z, 1]) to the
    column-major float layout of glm::mat4; None = identity."""
    if transform is None:
        return None
    m = np.asarray(transform, np.float32).reshape(4, 4)
    return np.ascontiguousarray(m.T.reshape(16))


def _read(fn, path, targetSegLen, transform, breakUpClosedCurves, allowResample, where):
    lib = _abi.load()
    t = _transform(transform)
    out = ctypes.c_void_p()
    _io_check(getattr(lib, fn)(os.fsencode(path), float(targetSegLen), None if t is None else ptr(t, ctypes.c_float),
                               int(bool(breakUpClosedCurves)), int(bool(allowResample)), ctypes.byref(out)), where)
    return Sim(_handle=out)


def readFromBCC(path, targetSegLen, transform=None, breakUpClosedCurves=False, allowResample=True):
    """YarnBall::readFromBCC (io/reader.cpp:49-97): an unconfigured Sim with one yarn per curve."""
    return _read("yb_read_bcc", path, targetSegLen, transform, breakUpClosedCurves, allowResample, "readFromBCC")


def readFromOBJ(path, targetSegLen, transform=None, breakUpClosedCurves=False, allowResample=True):
    """YarnBall::readFromOBJ (io/reader.cpp:99-156)."""
    return _read("yb_read_obj", path, targetSegLen, transform, breakUpClosedCurves, allowResample, "readFromOBJ")


def readFromPoly(path, targetSegLen, transform=None, breakUpClosedCurves=False, allowResample=True):
    """YarnBall::readFromPoly (io/reader.cpp:158-293)."""
    return _read("yb_read_poly", path, targetSegLen, transform, breakUpClosedCurves, allowResample, "readFromPoly")


def buildFromJSON(path):
    """YarnBall::buildFromJSON (io/jsonBuilder.cpp:8-172): a configured, uploaded Sim."""
    out = ctypes.c_void_p()
    _io_check(_abi.load().yb_build_from_json(os.fsencode(path), ctypes.byref(out)), "buildFromJSON")
    return Sim(_handle=out)


def resampleCMR(points, start, end, targetSegLen):
    """Resample::resampleCMR (io/resample.h:143-187) on float xyz points."""
    lib = _abi.load()
    p = np.ascontiguousarray(np.asarray(points, np.float32).reshape(-1, 3))
    cnt = ctypes.c_int32()
    check(lib.yb_resample_cmr(ptr(p, ctypes.c_float), len(p), float(start), float(end), float(targetSegLen), None, 0,
                              ctypes.byref(cnt)), "resampleCMR")
    out = np.zeros((max(cnt.value, 1), 3), np.float32)
    check(lib.yb_resample_cmr(ptr(p, ctypes.c_float), len(p), float(start), float(end), float(targetSegLen),
                              ptr(out, ctypes.c_float), len(out), ctypes.byref(cnt)), "resampleCMR")
    return out[:cnt.value]
