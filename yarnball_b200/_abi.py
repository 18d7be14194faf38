"""ctypes declarations of the C ABI in include/yarnball_b200.h and yarnball_b200_scenes.h.

The shared library is the product: every call here goes straight to the CUDA engine.  There
is no Python or CPU fallback; importing this module fails loudly when the library is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libyarnball_b200.so")

c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_uint64_p = ctypes.POINTER(ctypes.c_uint64)
c_int64_p = ctypes.POINTER(ctypes.c_int64)


class YbVertex(ctypes.Structure):
    """YarnBall::Vertex (YarnBall.h:52-61), 32 bytes."""

    _fields_ = [
        ("pos", ctypes.c_float * 3),
        ("invMass", ctypes.c_float),
        ("lRest", ctypes.c_float),
        ("kStretch", ctypes.c_float),
        ("connectionIndex", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
    ]


VERTEX_DTYPE = np.dtype(
    [
        ("pos", "<f4", (3,)),
        ("invMass", "<f4"),
        ("lRest", "<f4"),
        ("kStretch", "<f4"),
        ("connectionIndex", "<i4"),
        ("flags", "<u4"),
    ]
)
assert VERTEX_DTYPE.itemsize == 32


class YbMeta(ctypes.Structure):
    """YarnBall::MetaData without device pointers (YarnBall.h:63-114)."""

    _fields_ = [
        ("gravity", ctypes.c_float * 3),
        ("numItr", ctypes.c_int32),
        ("worldFloorNormal", ctypes.c_float * 3),
        ("worldFloorPos", ctypes.c_float),
        ("h", ctypes.c_float),
        ("lastH", ctypes.c_float),
        ("time", ctypes.c_float),
        ("numVerts", ctypes.c_int32),
        ("damping", ctypes.c_float),
        ("drag", ctypes.c_float),
        ("frictionCoeff", ctypes.c_float),
        ("kCollision", ctypes.c_float),
        ("kFriction", ctypes.c_float),
        ("detectionRadius", ctypes.c_float),
        ("scaledDetectionRadius", ctypes.c_float),
        ("radius", ctypes.c_float),
        ("accelerationRatio", ctypes.c_float),
        ("barrierThickness", ctypes.c_float),
        ("detectionScaler", ctypes.c_float),
        ("bvhRebuildPeriod", ctypes.c_float),
        ("detectionPeriod", ctypes.c_int32),
        ("maxSegLen", ctypes.c_float),
        ("minSegLen", ctypes.c_float),
        ("useStepSizeLimit", ctypes.c_int32),
        ("useVelocityRadius", ctypes.c_int32),
    ]


class YbPinMotion(ctypes.Structure):
    _fields_ = [("center", ctypes.c_float * 3), ("axis", ctypes.c_float * 3), ("omega", ctypes.c_float),
                ("velocity", ctypes.c_float * 3), ("tStart", ctypes.c_float), ("tEnd", ctypes.c_float)]


# name -> (restype, argtypes)
_P = ctypes.c_void_p
SIGNATURES = {
    "yb_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(_P)]),
    "yb_create_batch": (ctypes.c_int, [ctypes.c_int32, c_int32_p, ctypes.c_int32, ctypes.POINTER(_P)]),
    "yb_destroy": (None, [_P]),
    "yb_host_arrays": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(c_float_p), ctypes.POINTER(c_float_p),
                                      ctypes.POINTER(c_float_p)]),
    "yb_get_meta": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(YbMeta)]),
    "yb_set_meta": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(YbMeta)]),
    "yb_get_max_h": (ctypes.c_int, [_P, c_float_p]),
    "yb_set_max_h": (ctypes.c_int, [_P, ctypes.c_float]),
    "yb_configure": (ctypes.c_int, [_P, ctypes.c_float]),
    "yb_set_kstretch": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_float]),
    "yb_set_kbend": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_float]),
    "yb_upload": (ctypes.c_int, [_P]),
    "yb_download": (ctypes.c_int, [_P]),
    "yb_zero_velocities": (ctypes.c_int, [_P]),
    "yb_advance": (ctypes.c_int, [_P, ctypes.c_float, c_float_p]),
    "yb_step": (ctypes.c_int, [_P, ctypes.c_float]),
    "yb_step_count": (ctypes.c_int, [_P, c_uint64_p]),
    "yb_bounds": (ctypes.c_int, [_P, ctypes.c_int32, c_float_p]),
    "yb_collision_stats": (ctypes.c_int, [_P, c_uint64_p, c_int32_p, c_int32_p]),
    "yb_last_error": (ctypes.c_int, [_P, c_int32_p, c_int32_p]),
    "yb_initial_inv_masses": (ctypes.c_int, [_P, ctypes.POINTER(c_float_p), c_int32_p]),
    "yb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "yb_set_tuning": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "yb_get_tuning": (ctypes.c_int, [_P, c_int32_p, c_int32_p, c_int32_p, c_int32_p]),
    "yb_autotune": (ctypes.c_int, [_P, c_int32_p, c_int32_p, c_int32_p, c_float_p]),
    "yb_launch_count": (ctypes.c_int, [_P, c_uint64_p]),
    "yb_batch_gather": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(_P), c_int32_p, _P, ctypes.c_int64,
                                       ctypes.POINTER(_P)]),
    "yb_download_scene": (ctypes.c_int, [_P, ctypes.c_int32]),
    "yb_device_bytes": (ctypes.c_int, [_P, c_uint64_p]),
    "yb_scene_range": (ctypes.c_int, [_P, ctypes.c_int32, c_int32_p, c_int32_p]),
    "yb_export_bcc": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_int32]),
    "yb_export_obj": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "yb_export_fiber_mesh": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "yb_save_state": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "yb_read_bcc": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_float, c_float_p, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.POINTER(_P)]),
    "yb_read_obj": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_float, c_float_p, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.POINTER(_P)]),
    "yb_read_poly": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_float, c_float_p, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.POINTER(_P)]),
    "yb_build_from_json": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "yb_glue_endpoints": (ctypes.c_int, [_P, ctypes.c_float]),
    "yb_resample_cmr": (ctypes.c_int, [c_float_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       c_float_p, ctypes.c_int32, c_int32_p]),
    "yb_last_io_error": (ctypes.c_char_p, []),
    "yb_load_state": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "yb_set_pin_motion": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint8), ctypes.c_int32,
                                         ctypes.POINTER(YbPinMotion)]),
    "yb_set_stream": (ctypes.c_int, [_P, _P]),
    "yb_profile_advance": (ctypes.c_int, [_P, ctypes.c_float, c_double_p, c_uint64_p]),
    "yb_info": (ctypes.c_int, [_P, c_int32_p, c_int32_p, c_int32_p]),
    "yb_penetration_count": (ctypes.c_int, [_P, c_int64_p]),
    "yb_diagnostics": (ctypes.c_int, [_P, c_double_p]),
    "yb_step_residuals": (ctypes.c_int, [_P, c_double_p, ctypes.c_int32, c_int32_p]),
    "yb_min_pair_distance": (ctypes.c_int, [_P, c_double_p]),
    "yb_read_state_f64": (ctypes.c_int, [_P, c_double_p, c_double_p, c_double_p]),
    "yb_debug_contacts": (ctypes.c_int, [_P, c_int32_p, c_int32_p, c_float_p]),
    "yb_debug_dx": (ctypes.c_int, [_P, c_double_p]),
    "yb_debug_last_vel": (ctypes.c_int, [_P, c_double_p]),
    "yb_debug_packed_contacts": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint32), c_int32_p, ctypes.c_int64]),
    "yb_set_traversal": (ctypes.c_int, [_P, ctypes.c_int32]),
    "yb_set_small_path": (ctypes.c_int, [_P, ctypes.c_int32]),
    "yb_get_traversal": (ctypes.c_int, [_P, c_int32_p]),
    "yb_debug_phases": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_float]),
    "yb_debug_sort_pairs": (ctypes.c_int, [c_uint64_p, c_int32_p, ctypes.c_int32, ctypes.c_int32, c_uint64_p,
                                           c_int32_p]),
    "yb_sort_pairs_noalloc": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P]),
    "yb_scene_random_walks": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_int32, c_int32_p, ctypes.c_float,
                                             ctypes.c_float, ctypes.c_float, ctypes.c_float, c_float_p]),
    "yb_scene_random_walks_batch": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_int32, c_int32_p, c_int32_p,
                                                   ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                                   c_float_p, ctypes.c_int32]),
    "yb_rng_u64": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_int32]),
}

_LIB = None


def load():
    """Loads the engine library (once).  Raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "yarnball_b200: %s is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'`"
            % LIB_PATH
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def ptr(a, ctype):
    """ctypes pointer to the data of a contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class YarnBallError(RuntimeError):
    """A non-zero yb_status (the reference throws std::runtime_error for these)."""

    def __init__(self, status, where=""):
        self.status = int(status)
        msg = load().yb_status_string(int(status)).decode()
        super().__init__("%s%s (status %d)" % (where + ": " if where else "", msg, self.status))


def check(status, where=""):
    if status != 0:
        raise YarnBallError(status, where)
