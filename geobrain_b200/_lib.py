"""ctypes binding of the C ABI in include/geobrain_b200.h.

The CUDA library is built in-tree (``geobrain_b200/_so/libgeobrain_b200.so``,
see ``geobrain_b200.build``).  There is no fallback: if the library is
missing or no CUDA device is present, every call raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_so", "libgeobrain_b200.so")

GB_OK = 0
GB_E_ARG = -1
GB_E_CUDA = -2
GB_E_WORKSPACE = -3
GB_E_TIMEOUT = -4
GB_E_UNSUPPORTED = -5

CKPT_FORMATS = {"fp32": 0, "bf16": 1, "fp16": 2, "fp24": 3}
IMAGING_FORMATS = {"fp32": 0, "bf16": 1, "fp24": 3}


class GbError(RuntimeError):
    """A C-ABI call failed; ``code`` is the GB_E_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"geobrain_b200 error {code}: {msg}")
        self.code = code


class ModelDesc(ctypes.Structure):
    _fields_ = [
        ("nz", ctypes.c_int32), ("nx", ctypes.c_int32), ("nabc", ctypes.c_int32), ("nt", ctypes.c_int32),
        ("n_shots", ctypes.c_int32), ("n_rcv", ctypes.c_int32), ("half", ctypes.c_int32),
        ("free_surface", ctypes.c_int32), ("dt", ctypes.c_float), ("dx", ctypes.c_float),
    ]


class Desc3(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("nz", "ny", "nx", "nabc", "nt", "n_shots", "n_rcv", "free_surface")] + [
        (n, ctypes.c_float) for n in ("dt", "dx", "dy", "dz")]


class GradStore(ctypes.Structure):
    _fields_ = [("checkpoints", ctypes.c_void_p), ("checkpoint_every", ctypes.c_int32), ("format", ctypes.c_int32),
                ("imaging", ctypes.c_void_p), ("cached_steps", ctypes.c_int32), ("with_rho", ctypes.c_int32),
                ("imaging_format", ctypes.c_int32)]


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); every symbol include/geobrain_b200.h declares.
SIGNATURES = {
    "gb_plan_create": (ctypes.c_int, [ctypes.POINTER(ModelDesc), _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "gb_plan_destroy": (None, [_P]),
    "gb_plan_set_tiling": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "gb_plan_workspace_bytes": (_SZ, [_P, ctypes.c_int, ctypes.c_int]),
    "gb_plan_gradient_workspace_bytes": (_SZ, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gb_plan_checkpoint_bytes": (_SZ, [_P, ctypes.c_int, ctypes.c_int]),
    "gb_plan_imaging_bytes": (_SZ, [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gb_plan_set_group_streams": (ctypes.c_int, [_P, ctypes.c_int]),
    "gb_plan_set_graph_steps": (ctypes.c_int, [_P, ctypes.c_int]),
    "gb_plan_set_schedule": (ctypes.c_int, [_P, ctypes.c_int]),
    "gb_plan_schedule_items": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_int)]),
    "gb_plan_set_resident": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "gb_plan_launch_calls": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "gb_plan_get_resident": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    "gb_trace_misfit": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _P, _P, _P, _P]),
    "gb3_workspace_bytes": (_SZ, [ctypes.POINTER(Desc3)]),
    "gb3_forward": (ctypes.c_int, [ctypes.POINTER(Desc3)] + [_P] * 6 + [_P] * 4 + [_P] * 8 + [_P, _I32] +
                    [_P, _I32] + [_P, _SZ, _P]),
    "gb3_imaging_bytes": (_SZ, [ctypes.POINTER(Desc3), _I32]),
    "gb3_set_fused_step": (ctypes.c_int, [_I32]),
    "gb3_checkpoint_bytes": (_SZ, [ctypes.POINTER(Desc3), _I32]),
    "gb3_backward_workspace_bytes": (_SZ, [ctypes.POINTER(Desc3), _I32, _I32]),
    "gb3_backward": (ctypes.c_int, [ctypes.POINTER(Desc3)] + [_P] * 6 + [_P] * 4 + [_P] * 4 + [_P, _I32] +
                     [_P, _I32] + [_P, _P, _P, _P, _SZ, _P]),
    "gb_plan_autotune_workspace_bytes": (_SZ, [_P]),
    "gb_plan_get_config": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
    "gb_plan_set_streaming": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
    "gb_plan_set_absorbing": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_float]),
    "gb_plan_autotune": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _SZ, _I32, _P, ctypes.POINTER(ctypes.c_float)]),
    "gb_forward": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I32, _P, _P, _P, _SZ, _P]),
    "gb_backward": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "gb_workspace_status": (ctypes.c_int, [_P, _P]),
    "gb_selftest_bounded_wait": (ctypes.c_int, [_P, _SZ, _I32, _I32, _P]),
    "gb_plan_set_profiling": (ctypes.c_int, [_P, ctypes.c_int]),
    "gb_plan_profile": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong)]),
    "gb_static_scratch_bytes": (_SZ, []),
    "gb_forward_static_scratch": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I32, _P, _P]),
    "gb_batch_workspace_bytes": (_SZ, [_P, ctypes.c_int]),
    "gb_batch_forward": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _SZ, _P]),
    "gb_batch_backward": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _SZ, _P]),
    "gb_last_error": (ctypes.c_char_p, []),
    "gb_version": (ctypes.c_char_p, []),
}

_lib = None
_lock = threading.Lock()


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"geobrain_b200 CUDA library not built ({LIB_PATH}); run geobrain_b200.build.build()")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(rc: int) -> None:
    if rc != GB_OK:
        msg = load().gb_last_error()
        raise GbError(rc, msg.decode() if msg else "")


def ptr(t) -> int | None:
    """Device address of a tensor (None for None)."""
    return None if t is None else t.data_ptr()
