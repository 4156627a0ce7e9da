"""Loads libmcrt.so (include/mcrt.h) with ctypes. There is no fallback: if the
library is missing or a CUDA call fails, the call raises."""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmcrt.so")

MCRT_OK = 0
MCRT_ERR_INVALID = 1
MCRT_ERR_CUDA = 2
MCRT_ERR_NO_SCENE = 3
MCRT_ERR_TEXTURE = 4
MCRT_ERR_LIMIT = 5
MCRT_ERR_WALK = 6  # a BVH walk reached a bound (stack depth, see-through list, step budget)

# Rays per call of mcrt_intersect_closest_noalloc (its fixed per-device array holds this many).
NOALLOC_MAX_RAYS = 1 << 16


class McrtError(RuntimeError):
    """A failed libmcrt call: `code` is the MCRT_ERR_* status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class WalkLimitError(McrtError):
    """A call whose BVH walks reached one of their bounds (MCRT_ERR_WALK): its result
    may differ from the reference's, so none is returned."""


class mcrt_stats(C.Structure):
    _fields_ = [
        ("closest_rays", C.c_uint64), ("any_rays", C.c_uint64), ("samples", C.c_uint64),
        ("launches", C.c_uint64), ("ms_total", C.c_double), ("ms_raygen", C.c_double),
        ("ms_extend", C.c_double), ("ms_shade", C.c_double), ("ms_shadow", C.c_double),
        ("ms_resolve", C.c_double), ("ms_accumulate", C.c_double), ("n_raygen", C.c_uint64),
        ("n_extend", C.c_uint64), ("n_shade", C.c_uint64), ("n_shadow", C.c_uint64),
        ("n_resolve", C.c_uint64), ("n_accumulate", C.c_uint64), ("path_bytes", C.c_uint64),
        ("scene_bytes", C.c_uint64), ("status", C.c_uint32), ("pad_", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad_"}


# Every function include/mcrt.h declares, with its ctypes signature.
_P = C.POINTER
_i32, _u32, _f, _d, _u8, _vp = C.c_int32, C.c_uint32, C.c_float, C.c_double, C.c_uint8, C.c_void_p
SIGNATURES = {
    "mcrt_last_error": (C.c_char_p, []),
    "mcrt_version": (_i32, []),
    "mcrt_device_count": (_i32, [_P(_i32)]),
    "mcrt_executor_create": (_i32, [_i32, _P(_vp)]),
    "mcrt_executor_destroy": (_i32, [_vp]),
    "mcrt_send_geometry": (_i32, [_vp, _i32, _P(abi.mcrt_geometry)]),
    "mcrt_send_textures": (_i32, [_vp, _i32, _P(abi.mcrt_texture)]),
    "mcrt_send_shading": (_i32, [_vp, _i32, _P(abi.mcrt_shading)]),
    "mcrt_render_tile": (_i32, [_vp, _i32, _i32, _P(abi.mcrt_camera), _P(abi.mcrt_settings), _P(abi.mcrt_tile),
                                _i32, _i32, _i32, _i32, _P(_f)]),
    "mcrt_raytrace": (_i32, [_vp, _i32, _i32, _P(abi.mcrt_camera), _P(abi.mcrt_settings), _i32, _i32, _i32, _i32,
                             _P(_u8)]),
    "mcrt_raytrace_device": (_i32, [_vp, _i32, _i32, _P(abi.mcrt_camera), _P(abi.mcrt_settings), _i32, _i32, _i32,
                                    _i32, _vp]),
    "mcrt_render_pixels": (_i32, [_vp, _i32, _i32, _P(abi.mcrt_camera), _P(abi.mcrt_settings), _i32, _i32, _i32,
                                  _i32, _i32, _P(_i32), _P(_i32), _P(_u8), _P(_f)]),
    "mcrt_trace_primary": (_i32, [_vp, _i32, _P(abi.mcrt_camera), _i32, _i32, _i32, _u32, _i32, _P(_i32), _P(_i32),
                                  _P(_i32), _P(_f), _P(_i32)]),
    "mcrt_intersect_closest": (_i32, [_vp, _i32, _i32, _P(_f), _i32, _P(_i32), _P(_f), _P(_f), _P(_i32)]),
    "mcrt_intersect_closest_noalloc": (_i32, [_vp, _i32, _i32, _P(_f), _i32, _P(_i32), _P(_f), _P(_f),
                                              _P(_i32)]),
    "mcrt_intersect_any_count": (_i32, [_vp, _i32, _i32, _P(_f), _P(_i32)]),
    "mcrt_batch_create": (_i32, [_i32, _i32, C.c_int64, _i32, _P(_vp)]),
    "mcrt_batch_destroy": (_i32, [_vp]),
    "mcrt_batch_set_chunk": (_i32, [_vp, _i32]),
    "mcrt_batch_submit": (_i32, [_vp, _vp, _P(C.c_int64)]),
    "mcrt_batch_cancel": (_i32, [_vp, C.c_int64]),
    "mcrt_batch_step": (_i32, [_vp, _vp, _i32, _P(_i32), _P(_i32)]),
    "mcrt_batch_render": (_i32, [_vp, _i32, _vp]),
    "mcrt_batch_get_stats": (_i32, [_vp, _vp]),
    "mcrt_build_bvh": (_i32, [_vp, _P(_f), _i32, _P(_f), _P(_i32), _P(_u32), _P(_i32)]),
    "mcrt_compile_geometry": (_i32, [_vp, _i32, _P(_d), _P(_d), _P(_d), _P(_d), _P(_u8), _P(_u32), _P(_u8), _P(_u8),
                                     _P(_f), _P(_f), _P(_f), _P(_f), _P(_f), _P(_u32), _P(_u8), _P(_u8), _P(_f),
                                     _P(_i32), _P(_u32), _P(_i32), _P(_d), _P(_i32)]),
    "mcrt_upload_meshes": (_i32, [_vp, _i32, _P(abi.mcrt_mesh)]),
    "mcrt_compile_instances": (_i32, [_vp, _i32, _i32, _P(abi.mcrt_instance), _i32, _P(abi.mcrt_build_info),
                                      _P(abi.mcrt_compiled_out)]),
    "mcrt_set_timing": (_i32, [_vp, _i32]),
    "mcrt_set_capacity": (_i32, [_vp, _i32]),
    "mcrt_traversal_variants": (_i32, [_i32, _P(_i32), _P(_i32), _P(_i32)]),
    "mcrt_set_traversal": (_i32, [_vp, _i32, _i32]),
    "mcrt_batch_set_traversal": (_i32, [_vp, _i32, _i32]),
    "mcrt_get_stats": (_i32, [_vp, _P(mcrt_stats)]),
    "mcrt_reset_stats": (_i32, [_vp]),
    "mcrt_set_step_limit": (_i32, [_vp, _i32]),
}

_lib: Optional[C.CDLL] = None


def load() -> C.CDLL:
    """The loaded library, with signatures set. Raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run `python -m meercadraytracer_b200.build` "
                               "(the ray tracer has no CPU path)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def call(name: str, *args) -> None:
    """Calls an mcrt_* function and raises McrtError on a non-zero status."""
    lib = load()
    code = getattr(lib, name)(*args)
    if code != MCRT_OK:
        message = lib.mcrt_last_error().decode(errors="replace") or f"{name} failed ({code})"
        raise (WalkLimitError if code == MCRT_ERR_WALK else McrtError)(code, message)


def traversal_variants() -> list:
    """The (threads per block, short-stack entries) pairs the traversal kernels were compiled for."""
    n = C.c_int32()
    call("mcrt_traversal_variants", 0, None, None, C.byref(n))
    blocks = (C.c_int32 * max(1, n.value))()
    stacks = (C.c_int32 * max(1, n.value))()
    call("mcrt_traversal_variants", n.value, blocks, stacks, C.byref(n))
    return [(int(blocks[i]), int(stacks[i])) for i in range(n.value)]
