"""ctypes binding of the C ABI in include/tccg_b200.h.

The CUDA library is the only compute path: if it cannot be loaded (or built),
every call raises ``NativeUnavailable`` -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

MAX_MODES = 12

OK = 0
ERR_INVALID = -1
ERR_UNSUPPORTED = -2
ERR_WORKSPACE = -3
ERR_CUDA = -4
ERR_ALIGNMENT = -5
ERR_DEVICE = -6

F32, F64, BF16 = 0, 1, 2
PREC_FP32, PREC_FP64, PREC_BF16, PREC_BF16X3 = 0, 1, 2, 3
METHOD_GETT, METHOD_TTGT, METHOD_LOG = 0, 1, 2

PRECISIONS = {"fp32": PREC_FP32, "fp64": PREC_FP64, "bf16": PREC_BF16, "bf16x3": PREC_BF16X3}
METHODS = {"gett": METHOD_GETT, "ttgt": METHOD_TTGT, "log": METHOD_LOG}

EXPORTED = [
    "tccg_version", "tccg_last_error", "tccg_plan_create", "tccg_plan_workspace",
    "tccg_plan_run", "tccg_plan_run_timed", "tccg_plan_run_events", "tccg_plan_describe", "tccg_plan_flops", "tccg_plan_destroy",
    "tccg_plan_status", "tccg_transpose", "tccg_group_create", "tccg_group_workspace",
    "tccg_group_bind", "tccg_group_run", "tccg_group_destroy", "tccg_gett_bf16x3_noalloc",
    "tccg_gett_bf16x3_noalloc_status", "tccg_debug_inject_timeout",
]


class NativeUnavailable(RuntimeError):
    pass


class TccgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("tccg error %d: %s" % (code, msg))
        self.code = code


_I64xM = ctypes.c_int64 * MAX_MODES


class Desc(ctypes.Structure):
    _fields_ = [("nm", ctypes.c_int32), ("nn", ctypes.c_int32), ("nk", ctypes.c_int32),
                ("swap_ab", ctypes.c_int32),
                ("m_ext", _I64xM), ("n_ext", _I64xM), ("k_ext", _I64xM),
                ("a_m_stride", _I64xM), ("a_k_stride", _I64xM),
                ("b_n_stride", _I64xM), ("b_k_stride", _I64xM),
                ("c_m_stride", _I64xM), ("c_n_stride", _I64xM)]


class Tuning(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("variant", ctypes.c_int32),
                ("ksplit", ctypes.c_int32), ("raster", ctypes.c_int32),
                ("max_ctas", ctypes.c_int32), ("pair", ctypes.c_int32),
                ("direct", ctypes.c_int32), ("shortk", ctypes.c_int32),
                ("simt_tile", ctypes.c_int32), ("tail_split", ctypes.c_int32),
                ("load", ctypes.c_int32), ("tile_n", ctypes.c_int32),
                ("skinny", ctypes.c_int32)]


_lib = None
_lock = threading.Lock()


def _declare(L):
    vp, sz, i32, i64p = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)
    L.tccg_version.restype = ctypes.c_char_p
    L.tccg_last_error.restype = ctypes.c_char_p
    L.tccg_plan_create.argtypes = [ctypes.POINTER(Desc), i32, i32, ctypes.POINTER(Tuning),
                                   ctypes.POINTER(vp)]
    L.tccg_plan_workspace.argtypes = [vp, ctypes.POINTER(sz)]
    L.tccg_plan_run.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, vp, sz, vp]
    L.tccg_plan_run_timed.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, vp, sz,
                                      vp, ctypes.POINTER(ctypes.c_float)]
    L.tccg_plan_run_events.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, vp, sz,
                                       vp, ctypes.POINTER(vp)]
    L.tccg_plan_describe.argtypes = [vp, ctypes.c_char_p, sz]
    L.tccg_plan_flops.argtypes = [vp, ctypes.c_double]
    L.tccg_plan_flops.restype = ctypes.c_double
    L.tccg_plan_destroy.argtypes = [vp]
    L.tccg_plan_status.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    L.tccg_transpose.argtypes = [i32, i32, ctypes.POINTER(ctypes.c_int32), i64p, i64p, i64p,
                                 ctypes.c_double, vp, ctypes.c_double, vp, vp]
    L.tccg_group_create.argtypes = [ctypes.POINTER(vp), i32, ctypes.POINTER(vp)]
    L.tccg_group_workspace.argtypes = [vp, ctypes.POINTER(sz)]
    L.tccg_group_bind.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                  vp, sz]
    L.tccg_group_run.argtypes = [vp, vp]
    L.tccg_group_destroy.argtypes = [vp]
    L.tccg_gett_bf16x3_noalloc.argtypes = [ctypes.POINTER(Desc), vp, vp, vp, ctypes.c_double,
                                           ctypes.c_double, vp]
    L.tccg_gett_bf16x3_noalloc_status.argtypes = [ctypes.POINTER(ctypes.c_int32)]
    L.tccg_debug_inject_timeout.argtypes = [i32, i32]
    for name in EXPORTED:
        if name not in ("tccg_version", "tccg_last_error", "tccg_plan_flops"):
            getattr(L, name).restype = ctypes.c_int


def lib(build_if_missing: bool = True):
    """Load (building first if needed) the native library."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB_PATH
        try:
            if build_if_missing and _build.needs_build():
                _build.build()
        except Exception as e:  # noqa: BLE001
            if not os.path.exists(path):
                raise NativeUnavailable("cannot build %s: %s" % (path, e)) from e
        if not os.path.exists(path):
            raise NativeUnavailable("%s is missing; run __graft_entry__.build()" % path)
        try:
            L = ctypes.CDLL(path)
        except OSError as e:
            raise NativeUnavailable("cannot load %s: %s" % (path, e)) from e
        _declare(L)
        _lib = L
        return L


def check(rc: int) -> None:
    if rc != OK:
        msg = lib().tccg_last_error().decode(errors="replace")
        raise TccgError(rc, msg)
