"""The reference's own simulator kernels, run on the GPU (test infrastructure only).

oracle/refbuild/build.py compiles the reference's kernels (KittenEngine/YarnBall/sim/*.cu,
YarnBall.cu) unchanged into oracle/_ref/*.fatbin; oracle/_ref/libyb_ref.so loads a fatbin and
runs the reference's substep schedule around them.  Used by the tests as a second checker that
pins the oracle's restatement to the reference's code; never by the product.

Two builds of the kernels: "nofma" rounds every multiply and add separately (the arithmetic the
oracle's FP32 restatement performs, for bit-for-bit comparisons) and "fma" is the reference's
own build setting (nvcc's default contraction into fused multiply-adds).
"""
import ctypes
import os

import numpy as np

from . import VERTEX_DTYPE, OrcMeta

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "libyb_ref.so")
FATBINS = {"nofma": os.path.join(REF_DIR, "ref_nofma.fatbin"), "fma": os.path.join(REF_DIR, "ref.fatbin")}

_v = ctypes.c_void_p
_f = ctypes.POINTER(ctypes.c_float)
_SIG = {
    "ref_last_error": (ctypes.c_char_p, []),
    "ref_init": (ctypes.c_int, [ctypes.c_char_p]),
    "ref_create": (_v, [ctypes.c_int, ctypes.c_int, _v, _f, _f, _f, _v, ctypes.c_float]),
    "ref_destroy": (None, [_v]),
    "ref_advance": (ctypes.c_int, [_v, ctypes.c_float]),
    "ref_phase": (ctypes.c_int, [_v, ctypes.c_int, ctypes.c_float]),
    "ref_read": (ctypes.c_int, [_v, ctypes.c_int, _v]),
    "ref_write_state": (ctypes.c_int, [_v, _v, _f, _f, _f]),
    "ref_get_meta": (ctypes.c_int, [_v, _v]),
    "ref_set_meta": (ctypes.c_int, [_v, _v]),
    "ref_info": (None, [_v, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int),
                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint64)]),
    "ref_time_advance": (ctypes.c_int, [_v, ctypes.c_float, ctypes.c_int, _f]),
    "ref_math": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _f, _f, _f, _f, _f, _f]),
}

_LIB = None
_IDS = {}


def available():
    return os.path.exists(LIB_PATH) and all(os.path.exists(p) for p in FATBINS.values())


def load(variant="nofma"):
    """Loads the harness and the given kernel build; returns (library, kernel-build id)."""
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIG.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    if variant not in _IDS:
        i = _LIB.ref_init(FATBINS[variant].encode())
        if i < 0:
            raise RuntimeError("reference kernels: %s" % _LIB.ref_last_error().decode())
        _IDS[variant] = i
    return _LIB, _IDS[variant]


def _fp(a):
    return a.ctypes.data_as(_f)


PHASE_SET_H, PHASE_INIT, PHASE_DETECT, PHASE_STEP_LIMIT, PHASE_ITERATE, PHASE_END = range(6)
READ = dict(dx=0, y=1, lastVel=2, lastPos=3, numCols=4, cols=5, stepLimit=6, q=7, verts=8)


class RefSim:
    """A simulation on the reference's kernels, started from configured host arrays."""

    def __init__(self, verts, vels, qs, qRests, meta, maxH=1e-3, variant="nofma"):
        self.lib, lid = load(variant)
        self.n = len(verts)
        self._keep = [np.ascontiguousarray(verts), np.ascontiguousarray(vels, np.float32),
                      np.ascontiguousarray(qs, np.float32), np.ascontiguousarray(qRests, np.float32)]
        m = OrcMeta.from_buffer_copy(bytes(meta))
        self.h = self.lib.ref_create(lid, self.n, self._keep[0].ctypes.data, _fp(self._keep[1]), _fp(self._keep[2]),
                                     _fp(self._keep[3]), ctypes.addressof(m), float(maxH))
        if not self.h:
            raise RuntimeError("reference simulation: %s" % self.lib.ref_last_error().decode())

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, r, what):
        if r < 0:
            raise RuntimeError("reference %s: %s" % (what, self.lib.ref_last_error().decode()))
        return r

    def advance(self, dt):
        return self._ck(self.lib.ref_advance(self.h, float(dt)), "advance")

    def phase(self, p, value=0.0):
        return self._ck(self.lib.ref_phase(self.h, int(p), float(value)), "phase %d" % p)

    def read(self, what):
        n = self.n
        shape = {0: (n, 3), 1: (n, 3), 2: (n, 3), 3: (n, 3), 4: (n,), 5: (128, n), 6: (n,), 7: (n, 4)}
        w = READ[what]
        if w == 8:
            out = np.zeros(n, VERTEX_DTYPE)
        else:
            out = np.zeros(shape[w], np.int32 if w in (4, 5) else np.float32)
        self._ck(self.lib.ref_read(self.h, w, out.ctypes.data), "read")
        return out

    def lists(self):
        """Contact lists sorted ascending (the reference's order comes from atomics)."""
        nc = self.read("numCols")
        cols = self.read("cols")
        return nc, [np.sort(cols[: min(nc[i], 128), i]) for i in range(self.n)]

    def write_state(self, verts=None, vels=None, last_vel=None, qs=None):
        keep = []

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a

        v = arr(verts, VERTEX_DTYPE)
        vl, lv, q = arr(vels, np.float32), arr(last_vel, np.float32), arr(qs, np.float32)
        self._ck(self.lib.ref_write_state(self.h, v.ctypes.data if v is not None else None,
                                          _fp(vl) if vl is not None else None, _fp(lv) if lv is not None else None,
                                          _fp(q) if q is not None else None), "write_state")

    def meta(self):
        m = OrcMeta()
        self.lib.ref_get_meta(self.h, ctypes.addressof(m))
        return m

    def set_meta(self, m):
        self._ck(self.lib.ref_set_meta(self.h, ctypes.addressof(m)), "set_meta")

    def info(self):
        sc, pc = ctypes.c_uint64(), ctypes.c_uint64()
        e, w, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.ref_info(self.h, ctypes.byref(sc), ctypes.byref(e), ctypes.byref(w), ctypes.byref(t), ctypes.byref(pc))
        return dict(stepCount=sc.value, lastError=e.value, lastWarning=w.value, truncated=bool(t.value),
                    pairCandidates=pc.value)

    def time_advance(self, dt, frames):
        ms = ctypes.c_float()
        r = self._ck(self.lib.ref_time_advance(self.h, float(dt), int(frames), ctypes.byref(ms)), "time_advance")
        return r, ms.value


_MATH_IO = {0: ([12], [2]), 1: ([4, 4], [4]), 2: ([4, 3], [3]), 3: ([3, 3], [4]), 4: ([4], [4]),
            5: ([6, 3, 1, 3], [6, 3])}


def math(op, *inputs, variant="nofma", lib=None):
    """The reference's math helper `op` over arrays (one row per input); see ref_math.  With
    lib = the oracle's library, the oracle's restatement of the same helper instead."""
    ins, outs = _MATH_IO[op]
    n = len(inputs[0])
    arrs = [np.ascontiguousarray(np.asarray(x, np.float32).reshape(n, w)) for x, w in zip(inputs, ins)]
    arrs += [None] * (4 - len(arrs))
    res = [np.zeros((n, w), np.float32) for w in outs] + [None]
    ptrs = [(_fp(a) if a is not None else None) for a in arrs]
    out2 = _fp(res[1]) if res[1] is not None else None
    if lib is None:
        L, lid = load(variant)
        if L.ref_math(lid, op, n, *ptrs, _fp(res[0]), out2) < 0:
            raise RuntimeError("reference math: %s" % L.ref_last_error().decode())
    elif lib.orc_math(op, n, *ptrs, _fp(res[0]), out2) < 0:
        raise RuntimeError("oracle math op %d" % op)
    return res[0] if len(outs) == 1 else (res[0], res[1])


def oracle_math(op, *inputs):
    """The oracle's restatement of the reference's math helper `op` (CPU)."""
    from . import load as oload

    return math(op, *inputs, lib=oload())
