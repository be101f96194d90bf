"""ctypes binding of libtrj_sm100.so (the C ABI declared in include/trj_sm100.h).

There is no fallback: if the shared library is missing or cannot be loaded, the
import of the device layer raises, and every GPU operation fails loudly.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtrj_sm100.so")

TRJ_OK = 0
TRJ_ERR_INVALID = -1
TRJ_ERR_CUDA = -2
TRJ_ERR_NOMEM = -3
TRJ_ERR_CAPACITY = -4
TRJ_ERR_DATA = -5
TRJ_ERR_UNSUPPORTED = -6
TRJ_ERR_TIMEOUT = -7

TRJ_SQ_PLAIN_FP32 = 0
TRJ_SQ_SPLIT_BF16X3 = 1

EDGE_ULP, EDGE_FMA, EDGE_COUNTED, EDGE_TESTED = 0, 1, 2, 3

_ERRNAMES = {
    TRJ_ERR_INVALID: "TRJ_ERR_INVALID", TRJ_ERR_CUDA: "TRJ_ERR_CUDA", TRJ_ERR_NOMEM: "TRJ_ERR_NOMEM",
    TRJ_ERR_CAPACITY: "TRJ_ERR_CAPACITY", TRJ_ERR_DATA: "TRJ_ERR_DATA",
    TRJ_ERR_UNSUPPORTED: "TRJ_ERR_UNSUPPORTED", TRJ_ERR_TIMEOUT: "TRJ_ERR_TIMEOUT",
}

# Every exported entry point of include/trj_sm100.h with its ctypes signature.
c_int, c_int64, c_float, c_double = ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double
vp = ctypes.c_void_p
P = ctypes.POINTER
SIGNATURES = {
    "trj_abi_version": (c_int, []),
    "trj_ctx_create": (c_int, [c_int, P(vp)]),
    "trj_ctx_destroy": (c_int, [vp]),
    "trj_ctx_last_error": (ctypes.c_char_p, [vp]),
    "trj_ctx_check": (c_int, [vp, vp]),
    "trj_ctx_sm_count": (c_int, [vp]),
    "trj_ctx_set_timing": (c_int, [vp, c_int]),
    "trj_ctx_set_allocator": (c_int, [vp, vp, vp, vp]),
    "trj_ctx_launches": (c_int64, [vp]),
    "trj_ctx_set_sq_tile_cols": (c_int, [vp, c_int]),
    "trj_rdf_kernel_ms": (c_int, [vp, P(c_float)]),
    "trj_sq_kernel_ms": (c_int, [vp, P(c_float)]),
    "trj_frame_pack": (c_int, [vp, vp, vp, c_int64, c_int, P(c_float), vp, vp, vp]),
    "trj_frame_pack_static": (c_int, [vp, vp, vp, c_int64, c_int, P(c_float), vp, vp, vp]),
    "trj_frame_pack_charges": (c_int, [vp, vp, vp, vp, c_int64, c_int, P(c_float), vp, vp, vp, vp]),
    "trj_frame_pack_types": (c_int, [vp, vp, vp, vp, c_int, c_int64, c_int, P(c_float), vp, vp, vp]),
    "trj_rdf_plan_create": (c_int, [vp, c_int, c_float, c_float, P(c_float), c_int64, P(vp)]),
    "trj_rdf_plan_create_floor": (c_int, [vp, c_int, c_float, c_int, P(c_float), c_int64, P(vp)]),
    "trj_rdf_plan_create_2d": (c_int, [vp, c_int, c_float, c_float, P(c_float), c_int64, P(vp)]),
    "trj_rdf_plan_info": (c_int, [vp, P(c_int), P(c_int), P(c_int), P(c_float), P(c_float), P(c_int64)]),
    "trj_rdf_accumulate": (c_int, [vp, vp, c_int64, P(c_float), vp, vp, vp]),
    "trj_rdf_accumulate_charged": (c_int, [vp, vp, vp, c_int64, P(c_float), vp, vp, vp, vp]),
    "trj_rdf_plan_destroy": (c_int, [vp]),
    "trj_rdf_s2n": (c_int, [vp, c_int, vp, vp, vp, vp]),
    "trj_sq_plan_create": (c_int, [vp, c_int, c_int64, vp, vp, vp, vp, c_int, P(c_int64), P(vp)]),
    "trj_sq_plan_create_charged": (c_int, [vp, c_int, c_int64, vp, vp, vp, vp, c_int, P(c_int64), P(vp)]),
    "trj_sq_plan_info": (c_int, [vp, P(c_int64), P(c_int64), P(c_int64), P(c_int64)]),
    "trj_sq_plan_set_flush": (c_int, [vp, c_int]),
    "trj_sq_plan_set_pairs": (c_int, [vp, c_int]),
    "trj_sq_accumulate": (c_int, [vp, vp, c_int64, P(c_float), c_int, vp, vp]),
    "trj_sq_accumulate_charged": (c_int, [vp, vp, vp, c_int64, P(c_float), c_int, vp, vp]),
    "trj_sq_rho": (c_int, [vp, vp, vp]),
    "trj_sq_rho_groups": (c_int, [vp, vp, c_int64, P(c_float), c_int, vp, vp, vp]),
    "trj_sq_plan_set_z_from_y": (c_int, [vp, c_int]),
    "trj_rdf_plan_set_binning": (c_int, [vp, c_int]),
    "trj_rdf_plan_set_wait": (c_int, [vp, c_int64, c_int]),
    "trj_sq_plan_destroy": (c_int, [vp]),
    "trj_dyn_plan_create": (c_int, [vp, c_int, c_int64, c_int, c_int, c_int64, vp, vp, c_int, vp, P(vp)]),
    "trj_dyn_plan_info": (c_int, [vp, P(c_int64)]),
    "trj_dyn_accumulate": (c_int, [vp, vp, c_int64, P(c_float), vp, vp, vp]),
    "trj_dyn_flush": (c_int, [vp, vp, vp, vp, vp, vp]),
    "trj_dyn_kernel_ms": (c_int, [vp, P(c_float)]),
    "trj_dyn_plan_destroy": (c_int, [vp]),
    "trj_batch_create": (c_int, [vp, c_int, c_int64, c_int, P(vp)]),
    "trj_batch_staging": (c_int, [vp, c_int, P(vp), P(vp)]),
    "trj_batch_begin": (c_int, [vp, c_int]),
    "trj_batch_add": (c_int, [vp, c_int, vp, vp, c_int64, c_int64, P(c_float), vp, vp, vp]),
    "trj_batch_launch": (c_int, [vp, c_int, vp]),
    "trj_batch_info": (c_int, [vp, c_int, P(c_int), P(c_int64), P(c_int64)]),
    "trj_batch_kernel_ms": (c_int, [vp, P(c_float)]),
    "trj_batch_destroy": (c_int, [vp]),
}

_lib = None
_lock = threading.Lock()


class TrjError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the library once; raises if it is missing (no CPU fallback exists)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(f"{path} not found: build it with trj_analysis_b200/build.py "
                              "(the GPU path has no fallback)")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.trj_abi_version() != 1:
            raise ImportError("libtrj_sm100.so ABI version mismatch")
        _lib = lib
        return lib


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc == TRJ_OK:
        return
    msg = what
    if ctx is not None:
        m = load().trj_ctx_last_error(ctx)
        if m:
            msg = f"{what}: {m.decode()}" if what else m.decode()
    raise TrjError(rc, msg)


def box3(box) -> ctypes.Array:
    return (c_float * 3)(*[float(b) for b in box])
