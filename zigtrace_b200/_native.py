"""ctypes binding of the C ABI in include/zigtrace_b200.h.

The shared library is built in-tree (``zigtrace_b200/libzt_b200.so``).  There
is no fallback: if the library is missing or fails to load, every entry point
raises, so nothing silently renders on the CPU.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libzt_b200.so"

# ---- data layouts (must match include/zigtrace_b200.h) -------------------
VEC3_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8")])
SHAPE_DTYPE = np.dtype([("kind", "<u4"), ("material", "<u4"), ("p", "<f8", (9,))])
MATERIAL_DTYPE = np.dtype([("kind", "<u4"), ("reserved", "<u4"), ("color", "<f8", (3,)), ("param", "<f8")])
CAMERA_DTYPE = np.dtype([("look_from", "<f8", (3,)), ("look_at", "<f8", (3,)), ("up", "<f8", (3,)),
                         ("vfov", "<f8"), ("aperture", "<f8"), ("focus_dist", "<f8"),
                         ("has_focus_dist", "<u4"), ("reserved", "<u4")])
BACKGROUND_DTYPE = np.dtype([("kind", "<u4"), ("reserved", "<u4"), ("a", "<f8", (3,)), ("b", "<f8", (3,))])
OPTIONS_DTYPE = np.dtype([("width", "<u8"), ("height", "<u8"), ("spp", "<u8"), ("max_depth", "<u8"),
                          ("threads", "<u8"), ("seed", "<u8"), ("tile_size", "<u8"),
                          ("light_sampling", "<u4"), ("reserved", "<u4")])
BVH_NODE_DTYPE = np.dtype([("bmin", "<f8", (3,)), ("bmax", "<f8", (3,)), ("first", "<u4"), ("count", "<u4")])
LIGHT_DTYPE = np.dtype([("shape", SHAPE_DTYPE), ("radiance", "<f8", (3,)), ("weight", "<f8")])
GPU_CONFIG_DTYPE = np.dtype([("mode", "<u4"), ("block_size", "<u4"), ("queue_capacity", "<u4"),
                             ("precision", "<u4")])

assert SHAPE_DTYPE.itemsize == 80 and MATERIAL_DTYPE.itemsize == 40
assert CAMERA_DTYPE.itemsize == 104 and BACKGROUND_DTYPE.itemsize == 56
assert OPTIONS_DTYPE.itemsize == 64 and BVH_NODE_DTYPE.itemsize == 56
assert LIGHT_DTYPE.itemsize == 112

ZT_OK = 0
ERRORS = {
    -1: "InvalidOptions",
    -2: "OutOfMemory",
    -3: "TooManyPrimitives",
    -4: "UnboundedShape",
    -5: "InvalidArgument",
    -6: "CudaError",
    -7: "Timeout",
    -8: "NotBuilt",
}

# Every exported entry point with (restype, argtypes); the ABI test checks
# this list against the header.
_P = C.c_void_p
_u64 = C.c_uint64
_u32 = C.c_uint32
_i32 = C.c_int32
SIGNATURES = {
    "zt_scene_create": (_i32, [C.POINTER(_P)]),
    "zt_scene_destroy": (None, [_P]),
    "zt_scene_add_material": (_i32, [_P, _P, C.POINTER(_u32)]),
    "zt_scene_add_materials": (_i32, [_P, _P, C.c_size_t, C.POINTER(_u32)]),
    "zt_scene_add_shapes": (_i32, [_P, _P, C.c_size_t]),
    "zt_scene_add_quad": (_i32, [_P, _P, _P, _P, _u32]),
    "zt_scene_set_camera": (_i32, [_P, _P]),
    "zt_scene_set_background": (_i32, [_P, _P]),
    "zt_scene_build": (_i32, [_P]),
    "zt_scene_build_device": (_i32, [_P, C.POINTER(_u32), C.POINTER(C.c_double)]),
    "zt_scene_set_bvh": (_i32, [_P, _P, C.c_size_t, _P, C.c_size_t]),
    "zt_scene_counts": (_i32, [_P, C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64),
                               C.POINTER(_u64)]),
    "zt_scene_bvh": (_i32, [_P, _P, _P]),
    "zt_scene_lights": (_i32, [_P, _P, _P, C.POINTER(C.c_double)]),
    "zt_scene_bvh_depth": (_i32, [_P, C.POINTER(_u64)]),
    "zt_scene_upload": (_i32, [_P]),
    "zt_scene_release_device": (_i32, [_P]),
    "zt_scene_upload_bytes": (_i32, [_P, C.POINTER(_u64)]),
    "zt_render": (_i32, [_P, _P, _P]),
    "zt_render_ex": (_i32, [_P, _P, _P, _P]),
    "zt_render_rows": (_i32, [_P, _P, _u64, _u64, _P]),
    "zt_render_device": (_i32, [_P, _P, _P, _P, _P]),
    "zt_render_rows_device": (_i32, [_P, _P, _u64, _u64, _P, _P, _P]),
    "zt_set_wavefront_iteration_limit": (_i32, [_u64]),
    "zt_render_debug": (_i32, [_P, _P, _P, _P]),
    "zt_render_noalloc": (_i32, [_P, _P, _P, _P]),
    "zt_forward": (_i32, [_P, _P, _P, _P]),
    "zt_backward": (_i32, [_P, _P, _P, _P, _P]),
    "zt_forward_rows": (_i32, [_P, _P, _u64, _u64, _P, _P]),
    "zt_backward_rows": (_i32, [_P, _P, _u64, _u64, _P, _P, _P]),
    "zt_scene_set_primal_cache_limit": (_i32, [_P, _u64]),
    "zt_batch_create": (_i32, [_P, _P, _u64, _P, _P, _u32, C.POINTER(_P)]),
    "zt_batch_launch": (_i32, [_P, _P]),
    "zt_batch_destroy": (None, [_P]),
    "zt_render_batch": (_i32, [_P, _P, _u64, _P, _P]),
    "zt_trace_paths": (_i32, [_P, _P, _P, _P, _u64, _u64, _u32, _P]),
    "zt_rng_streams": (_i32, [_u64, _u64, _u64, _u64, _P]),
    "zt_image_to_rgb8": (_i32, [_P, _u64, _u32, C.c_double, C.c_double, _P]),
    "zt_image_to_rgb8_device": (_i32, [_P, _u64, _u32, C.c_double, C.c_double, _P, _P]),
    "zt_png_size": (_i32, [_u64, _u64, C.POINTER(_u64)]),
    "zt_png_encode": (_i32, [_P, _u64, _u64, _P, _u64]),
    "zt_png_encode_device": (_i32, [_P, _u64, _u64, _P, _u64, _P]),
    "zt_render_rgb8": (_i32, [_P, _P, _P, _u32, C.c_double, C.c_double, _P]),
    "zt_render_png": (_i32, [_P, _P, _P, _u32, C.c_double, C.c_double, _P, _u64]),
    "zt_last_error": (C.c_char_p, []),
    "zt_version": (C.c_char_p, []),
}


class ZigtraceError(RuntimeError):
    """A zt_status other than ZT_OK; ``name`` is the reference's error name."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.name = ERRORS.get(status, f"status {status}")
        super().__init__(f"{self.name}: {message}")


_lib = None


def lib() -> C.CDLL:
    """Loads the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run zigtrace_b200._build.build() (needs nvcc)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int) -> None:
    if status != ZT_OK:
        msg = lib().zt_last_error()
        raise ZigtraceError(status, msg.decode() if msg else "")


def ptr(a: np.ndarray) -> C.c_void_p:
    """Pointer to the array's data that keeps the array alive for the call."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)
