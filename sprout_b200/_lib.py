"""ctypes binding of libsprout_b200.so (the C ABI declared in include/sprout_b200.h).

The library is loaded from the package directory only.  If it is missing, loading fails
with an error: there is no CPU fallback for any entry point.
"""

from __future__ import annotations

import ctypes
import pathlib

_PACKAGE = pathlib.Path(__file__).resolve().parent
LIBRARY_PATH = _PACKAGE / "libsprout_b200.so"

SPB_OK = 0
SPB_ERROR_ARGUMENT = -1
SPB_ERROR_STATE = -2
SPB_ERROR_CUDA = -3
SPB_MISS = 0xFFFFFFFF

c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_i32 = ctypes.c_int32
c_f32 = ctypes.c_float
c_vp = ctypes.c_void_p


class TreeInfo(ctypes.Structure):
    _fields_ = [
        ("num_triangles", c_u32),
        ("num_nodes", c_u32),
        ("num_leaves", c_u32),
        ("max_depth", c_u32),
        ("device_bytes", c_u64),
        ("build_seconds", ctypes.c_double),
        ("sah_cost", ctypes.c_double),
    ]


class RenderStats(ctypes.Structure):
    _fields_ = [
        ("paths", c_u64),
        ("extension_rays", c_u64),
        ("shadow_rays", c_u64),
        ("device_seconds", ctypes.c_double),
        ("overflow", c_u32),
        ("guide_vertices", c_u64),
        ("guide_inference_seconds", ctypes.c_double),
        ("guide_training_samples", c_u64),
        ("guide_training_seconds", ctypes.c_double),
        ("wave_paths", c_u32),
        ("trace_blocks_per_sm", c_u32),
        ("graph_waves", c_u32),
        ("instances", c_u32),
        ("tracking_capped", c_u32),
        ("device_triangles", c_u64),
    ]


class View(ctypes.Structure):
    """spb_view: one camera of spb_render_views."""
    _fields_ = [
        ("width", c_u32),
        ("height", c_u32),
        ("fov", ctypes.c_float),
        ("transformation", ctypes.c_float * 16),
    ]


# name -> (restype, argtypes); mirrors include/sprout_b200.h one to one.
PROTOTYPES = {
    "spb_last_error": (ctypes.c_char_p, []),
    "spb_version": (ctypes.c_char_p, []),
    "spb_tree_create": (c_i32, [ctypes.POINTER(c_vp)]),
    "spb_tree_release": (c_i32, [c_vp]),
    "spb_tree_build": (c_i32, [c_vp, c_u32, c_u32, c_vp, c_vp, c_u32]),
    "spb_tree_info_get": (c_i32, [c_vp, ctypes.POINTER(TreeInfo)]),
    "spb_intersect_device": (c_i32, [c_vp, c_vp, c_u64, c_vp, c_vp, c_vp, c_vp]),
    "spb_intersect_p_device": (c_i32, [c_vp, c_vp, c_u64, c_vp, c_vp]),
    "spb_intersect_host": (c_i32, [c_vp, c_vp, c_u64, c_vp, c_vp, c_vp]),
    "spb_intersect_p_host": (c_i32, [c_vp, c_vp, c_u64, c_vp]),
    "spb_tree_status": (c_i32, [c_vp, ctypes.POINTER(c_u32)]),
    "spb_synth_sphere_mesh": (c_i32, [c_u32, c_f32, c_u32, ctypes.POINTER(c_u32),
                                      ctypes.POINTER(c_u32), c_vp, c_vp]),
    "spb_synth_rays": (c_i32, [c_u64, c_u64, c_u32, c_f32, c_vp, c_u32]),
    "spb_ggx_albedo_table": (c_i32, [c_vp]),
    "spb_render_last_stats": (c_i32, [ctypes.POINTER(RenderStats)]),
    "spb_render_views": (c_i32, [c_u32, ctypes.POINTER(View), c_u32, c_vp]),
    "spb_guide_parameter_count": (c_i32, [ctypes.POINTER(ctypes.c_uint32)]),
    "spb_guide_forward": (c_i32, [c_vp, c_vp, ctypes.c_uint64, c_vp]),
    "spb_guide_gradients": (c_i32, [c_vp, c_vp, c_vp, c_vp, ctypes.c_uint64, c_vp]),
    "spb_intersect_host_static": (c_i32, [c_vp, c_vp, c_u64, c_vp, c_vp]),
    "spb_cast_stats_device": (c_i32, [c_vp, c_vp, c_u64, c_vp, c_vp, c_vp, ctypes.POINTER(c_u64),
                                      ctypes.POINTER(c_u64)]),
}

_lib = None


class SproutError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with `python -m sprout_b200.build` "
                "(nvcc, sm_100a); there is no CPU fallback")
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != SPB_OK:
        msg = load().spb_last_error().decode(errors="replace")
        raise SproutError(status, msg)
