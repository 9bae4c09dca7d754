"""ctypes binding of libever_b200.so (include/ever_b200.h).

The library is built in-tree by ever_b200/build.py. Loading fails loudly when it is
missing: there is no CPU or PyTorch fallback for the trace.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

c_i32, c_i64, c_f32, c_p, c_sz = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_void_p, ctypes.c_size_t


class EverScene(ctypes.Structure):
    _fields_ = [("num_prims", c_i64), ("sh_coeffs", c_i32), ("num_nodes", c_i32), ("nodes", c_p),
                ("records", c_p), ("features", c_p), ("order", c_p), ("scratch", c_p)]


class EverTune(ctypes.Structure):
    _fields_ = [("kbuf", c_i32), ("block", c_i32), ("traversal", c_i32), ("regroup_min", c_i32),
                ("stack_depth", c_i32), ("reserved", c_i32 * 3)]


class EverForwardOut(ctypes.Structure):
    _fields_ = [("out", c_p), ("states", c_p), ("last_dirac", c_p), ("iters", c_p), ("event_log", c_p),
                ("log_cap", c_i32), ("touch_count", c_p), ("ray_stats", c_p), ("status", c_p)]


class EverBackwardOut(ctypes.Structure):
    _fields_ = [("dmean", c_p), ("dscale", c_p), ("dquat", c_p), ("ddensity", c_p), ("dfeatures", c_p),
                ("drayo", c_p), ("drayd", c_p), ("dmeans2d", c_p)]


class EverTraceArgs(ctypes.Structure):
    _fields_ = [("tmin", c_f32), ("tmax", c_f32), ("max_iters", c_i32), ("sh_degree", c_i32), ("depth_hint", c_p)]


class EverBatchView(ctypes.Structure):
    _fields_ = [("scene", c_i32), ("pad", c_i32), ("ray_offset", c_i64), ("ray_count", c_i64)]


class EverBatch(ctypes.Structure):
    _fields_ = [("num_scenes", c_i32), ("num_views", c_i32), ("num_slots", c_i64), ("num_rays", c_i64),
                ("scene_table", c_p), ("view_table", c_p), ("slot_ray", c_p), ("counters", c_p),
                ("order_scratch", c_p), ("sh_coeffs", c_i32 * 64), ("num_prims", c_i64 * 64),
                ("bwd_workspace", c_p * 64)]


class EverMlp(ctypes.Structure):
    _fields_ = [("params", c_p), ("w1", c_p), ("w2", c_p), ("w3", c_p), ("centre", c_f32 * 3), ("inv_scale", c_f32),
                ("wait_clocks", c_i64)]


class EverCamera(ctypes.Structure):
    _fields_ = [("width", c_i32), ("height", c_i32), ("fx", c_f32), ("fy", c_f32), ("cx", c_f32), ("cy", c_f32),
                ("c2w", c_f32 * 12)]


MLP_PARAMS = 9360

STATUS_STACK_OVERFLOW = 1
STATUS_LOG_OVERFLOW = 2
STATUS_INIT_OVERFLOW = 4

# name -> (restype, argtypes); every symbol of include/ever_b200.h
SIGNATURES = {
    "ever_last_error": (ctypes.c_char_p, []),
    "ever_abi_version": (ctypes.c_int, []),
    "ever_scene_workspace_bytes": (c_sz, [c_i64, c_i32]),
    "ever_scene_build": (ctypes.c_int, [c_p, c_p, c_p, c_p, c_p, c_i64, c_i32, c_p, c_sz,
                                        ctypes.POINTER(EverScene), c_p]),
    "ever_scene_build_dc": (ctypes.c_int, [c_p, c_p, c_p, c_p, c_p, c_i64, c_i32, c_p, c_sz,
                                        ctypes.POINTER(EverScene), c_p]),
    "ever_scene_refit": (ctypes.c_int, [c_p, c_p, c_p, c_p, c_p, c_p, c_sz, ctypes.POINTER(EverScene), c_p]),
    "ever_scene_set_features": (ctypes.c_int, [ctypes.POINTER(EverScene), c_p, c_p]),
    "ever_trace_forward": (ctypes.c_int, [ctypes.POINTER(EverScene), c_p, c_p, c_i64, ctypes.POINTER(EverTraceArgs),
                                          c_p, ctypes.POINTER(EverTune), ctypes.POINTER(EverForwardOut), c_p]),
    "ever_trace_forward_workspace_bytes": (c_sz, [c_i64]),
    "ever_trace_forward_regrouped": (ctypes.c_int, [ctypes.POINTER(EverScene), c_p, c_p, c_i64,
                                                    ctypes.POINTER(EverTraceArgs), c_p, ctypes.POINTER(EverTune),
                                                    ctypes.POINTER(EverForwardOut), c_p, c_sz, c_p]),
    "ever_backward_workspace_bytes": (c_sz, [c_i64, c_i32]),
    "ever_trace_backward": (ctypes.c_int, [ctypes.POINTER(EverScene), c_p, c_p, c_i64, ctypes.POINTER(EverTraceArgs),
                                           c_p, c_p, c_p, c_p, c_i32, c_p, c_i32, c_p, c_p, c_p, c_p, c_sz, c_p,
                                           ctypes.POINTER(EverTune), ctypes.POINTER(EverBackwardOut), c_p]),
    "ever_trace_backward_ordered": (ctypes.c_int, [ctypes.POINTER(EverScene), c_p, c_p, c_i64,
                                                   ctypes.POINTER(EverTraceArgs), c_p, c_p, c_p, c_p, c_i32, c_p,
                                                   c_i32, c_p, c_p, c_p, c_p, c_sz, c_p, c_p,
                                                   ctypes.POINTER(EverTune), ctypes.POINTER(EverBackwardOut), c_p]),
    "ever_backward_slot_order": (ctypes.c_int, [c_p, c_p, c_i64, c_i32, c_p, c_sz, c_p, c_p]),
    "ever_event_log_to_reference": (ctypes.c_int, [ctypes.POINTER(EverScene), c_p, c_i32, c_p, c_i64, c_p, c_p,
                                                   c_i32, c_p]),
    "ever_ray_order_workspace_bytes": (c_sz, [c_i64]),
    "ever_ray_order": (ctypes.c_int, [c_p, c_p, c_i64, c_p, c_sz, c_p, c_p]),
    "ever_ray_order_static": (ctypes.c_int, [c_p, c_p, c_i64, c_p, c_p]),
    "ever_batch_workspace_bytes": (c_sz, [c_i32, ctypes.POINTER(EverBatchView), c_i32, ctypes.POINTER(c_i64)]),
    "ever_batch_setup": (ctypes.c_int, [ctypes.POINTER(EverScene), ctypes.POINTER(c_p), c_i32,
                                        ctypes.POINTER(EverBatchView), c_i32, c_i64, c_p, c_sz,
                                        ctypes.POINTER(EverBatch)]),
    "ever_batch_order": (ctypes.c_int, [ctypes.POINTER(EverBatch), c_p, c_p, c_p]),
    "ever_trace_forward_batched": (ctypes.c_int, [ctypes.POINTER(EverBatch), c_p, c_p, ctypes.POINTER(EverTraceArgs),
                                                  ctypes.POINTER(EverTune), ctypes.POINTER(EverForwardOut), c_p]),
    "ever_trace_backward_batched": (ctypes.c_int, [ctypes.POINTER(EverBatch), c_p, c_p,
                                                   ctypes.POINTER(EverTraceArgs), c_p, c_p, c_p, c_p, c_i32, c_p,
                                                   c_p, ctypes.POINTER(EverTune), c_p]),
    "ever_scene_finalize_gradients": (ctypes.c_int, [ctypes.POINTER(EverScene), c_p, c_p, c_p, c_p, c_sz,
                                                     ctypes.POINTER(EverBackwardOut), c_p]),
    "ever_mlp_workspace_bytes": (c_sz, []),
    "ever_mlp_pack": (ctypes.c_int, [ctypes.POINTER(EverMlp), c_p]),
    "ever_mlp_predict": (ctypes.c_int, [ctypes.POINTER(EverMlp), c_p, c_p, c_p, c_i64, c_p, c_p,
                                        ctypes.POINTER(c_f32), c_p, c_p]),
    "ever_mlp_gradients": (ctypes.c_int, [ctypes.POINTER(EverMlp), c_p, c_p, c_p, c_p, c_i64, c_p, c_f32, c_f32,
                                          c_p, c_p, c_p, c_sz, c_p, c_p]),
    "ever_mlp_adam": (ctypes.c_int, [ctypes.POINTER(EverMlp), c_p, c_p, c_p, c_f32, c_f32, c_f32, c_f32, c_i32,
                                     c_p]),
    "ever_ply_count": (c_i64, [ctypes.c_char_p]),
    "ever_ply_read": (ctypes.c_int, [ctypes.c_char_p, c_i64, c_p, c_p, c_p, c_p, c_p]),
    "ever_sh_prepass": (ctypes.c_int, [c_p, c_p, c_i64, c_i32, c_i32, c_p, c_i32, c_p, c_p]),
    "ever_sh_prepass_backward": (ctypes.c_int, [c_p, c_p, c_i64, c_i32, c_i32, c_p, c_i32, c_p, c_p, c_p]),
    "ever_camera_rays": (ctypes.c_int, [ctypes.POINTER(EverCamera), c_p, c_p, c_p, c_p]),
    "ever_camera_slots": (c_i64, [ctypes.POINTER(EverCamera)]),
    "ever_camera_slot_pixels": (ctypes.c_int, [ctypes.POINTER(EverCamera), c_p, c_p]),
    "ever_trace_forward_camera": (ctypes.c_int, [ctypes.POINTER(EverScene), ctypes.POINTER(EverCamera), c_p,
                                                 ctypes.POINTER(EverTraceArgs), ctypes.POINTER(EverTune),
                                                 ctypes.POINTER(EverForwardOut), c_p]),
    "ever_trace_forward_camera_regrouped": (ctypes.c_int, [ctypes.POINTER(EverScene), ctypes.POINTER(EverCamera),
                                                           c_p, ctypes.POINTER(EverTraceArgs), ctypes.POINTER(EverTune),
                                                           ctypes.POINTER(EverForwardOut), c_p, c_sz, c_p]),
    "ever_trace_backward_camera": (ctypes.c_int, [ctypes.POINTER(EverScene), ctypes.POINTER(EverCamera), c_p,
                                                  ctypes.POINTER(EverTraceArgs), c_p, c_p, c_p, c_p, c_i32, c_p,
                                                  c_i32, c_p, c_p, c_p, c_p, c_sz, c_p, ctypes.POINTER(EverTune),
                                                  ctypes.POINTER(EverBackwardOut), c_p]),
    "ever_camera_backward_slot_order": (ctypes.c_int, [ctypes.POINTER(EverCamera), c_p, c_i32, c_p, c_sz, c_p,
                                                       c_p]),
    "ever_camera_event_log_to_reference": (ctypes.c_int, [ctypes.POINTER(EverScene), ctypes.POINTER(EverCamera),
                                                          c_p, c_i32, c_p, c_p, c_i32, c_p]),
    "ever_ray_order_binned": (ctypes.c_int, [c_p, c_p, c_p, c_i64, c_p, c_sz, c_p, c_p]),
    "ever_batch_order_binned": (ctypes.c_int, [ctypes.POINTER(EverBatch), c_p, c_p, c_p, c_p]),
}

_lock = threading.Lock()
_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Loads the library (building it first when nvcc is available and it is stale)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB
        if build_if_missing and not _build.up_to_date():
            try:
                _build.build()
            except Exception as e:  # no nvcc (e.g. a runtime-only box): use the prebuilt file
                if not os.path.exists(path):
                    raise RuntimeError(f"libever_b200.so missing and cannot be built: {e}") from e
        if not os.path.exists(path):
            raise RuntimeError(f"libever_b200.so not found at {path}; run ever_b200/build.py")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
        return L


def check(rc: int):
    if rc != 0:
        msg = load().ever_last_error().decode(errors="replace")
        raise RuntimeError(f"ever_b200 error {rc}: {msg}")


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())
