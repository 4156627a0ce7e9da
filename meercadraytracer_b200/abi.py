"""ctypes mirror of include/mcrt_types.h and marshaling from the compiled types.

The C structs are the boundary's data contract (they mirror src/types.ts of the
reference); this module turns the Python dataclasses of `types.py` into those
structs without copying the large arrays. Every `to_c_*` function returns the
struct and a list of objects that must stay alive while the struct is in use.
"""
from __future__ import annotations

import ctypes as C
from typing import Any, List, Sequence, Tuple

import numpy as np

from .types import (
    BACKGROUND_KINDS,
    LIGHT_TYPES,
    MATERIAL_MODELS,
    SHADOW_MODES,
    CompiledCamera,
    CompiledGeometry,
    CompiledScene,
    CompiledTexture,
    Tile,
    TraceSettings,
)

c_double3 = C.c_double * 3
c_double9 = C.c_double * 9
c_double16 = C.c_double * 16


class mcrt_texture(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("format", C.c_int32), ("srgb", C.c_int32),
        ("flip_y", C.c_int32), ("wrap_s", C.c_int32), ("wrap_t", C.c_int32), ("id", C.c_int32),
        ("matrix", c_double9), ("data", C.c_void_p),
    ]


class mcrt_environment(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("faces", C.c_int32 * 6), ("texture", C.c_int32), ("flip_x", C.c_int32),
        ("rotation", c_double9), ("intensity", C.c_double),
    ]


class mcrt_material(C.Structure):
    _fields_ = [
        ("model", C.c_int32), ("side", C.c_int32), ("color", c_double3), ("opacity", C.c_double),
        ("transparent", C.c_int32), ("vertex_colors", C.c_int32), ("alpha_test", C.c_double),
        ("flat_shading", C.c_int32), ("tone_mapped", C.c_int32), ("map", C.c_int32),
        ("alpha_map", C.c_int32), ("emissive_map", C.c_int32), ("normal_map", C.c_int32),
        ("ao_map", C.c_int32), ("roughness_map", C.c_int32), ("metalness_map", C.c_int32),
        ("physical", C.c_int32), ("emissive", c_double3), ("normal_scale", C.c_double * 2),
        ("ao_map_intensity", C.c_double), ("roughness", C.c_double), ("metalness", C.c_double),
        ("ior", C.c_double), ("specular_intensity", C.c_double), ("specular_color", c_double3),
        ("transmission", C.c_double), ("thickness", C.c_double), ("attenuation", c_double3),
        ("shininess", C.c_double), ("specular", c_double3), ("env_map", C.c_int32),
        ("combine", C.c_int32), ("env_map_intensity", C.c_double), ("reflectivity", C.c_double),
    ]


class mcrt_light(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("cast_shadow", C.c_int32), ("color", c_double3),
        ("ground_color", c_double3), ("direction", c_double3), ("position", c_double3),
        ("distance", C.c_double), ("decay", C.c_double), ("cone_cos", C.c_double),
        ("penumbra_cos", C.c_double),
    ]


class mcrt_fog(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("pad_", C.c_int32), ("color", c_double3), ("near_", C.c_double),
        ("far_", C.c_double), ("density", C.c_double),
    ]


class mcrt_background(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("texture", C.c_int32), ("environment", C.c_int32), ("pad_", C.c_int32),
        ("color", c_double3), ("intensity", C.c_double),
    ]


class mcrt_geometry(C.Structure):
    _fields_ = [
        ("triangle_count", C.c_int32), ("node_count", C.c_int32),
        ("triangles", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
        ("uvs", C.POINTER(C.c_float)), ("tangents", C.POINTER(C.c_float)),
        ("colors", C.POINTER(C.c_float)), ("materials", C.POINTER(C.c_uint32)),
        ("flags", C.POINTER(C.c_uint8)), ("sides", C.POINTER(C.c_uint8)),
        ("bvh_bounds", C.POINTER(C.c_float)), ("bvh_nodes", C.POINTER(C.c_int32)),
        ("epsilon", C.c_double),
    ]


class mcrt_shading(C.Structure):
    _fields_ = [
        ("material_count", C.c_int32), ("texture_count", C.c_int32),
        ("environment_count", C.c_int32), ("light_count", C.c_int32),
        ("materials", C.POINTER(mcrt_material)), ("textures", C.POINTER(mcrt_texture)),
        ("environments", C.POINTER(mcrt_environment)), ("lights", C.POINTER(mcrt_light)),
        ("background", mcrt_background), ("fog", mcrt_fog), ("environment", C.c_int32),
        ("pad_", C.c_int32),
    ]


class mcrt_camera(C.Structure):
    _fields_ = [
        ("projection_inverse", c_double16), ("world", c_double16), ("orthographic", C.c_int32),
        ("pad_", C.c_int32), ("forward", c_double3), ("position", c_double3),
    ]


class mcrt_settings(C.Structure):
    _fields_ = [
        ("max_bounces", C.c_int32), ("shadows", C.c_int32), ("global_illumination", C.c_int32),
        ("tone_mapping", C.c_int32), ("tone_mapping_exposure", C.c_double),
        ("clear_color", c_double3), ("clear_alpha", C.c_double), ("seed", C.c_uint32),
        ("pad_", C.c_int32),
    ]


class mcrt_tile(C.Structure):
    _fields_ = [("x", C.c_int32), ("y", C.c_int32), ("width", C.c_int32), ("height", C.c_int32)]


class mcrt_request(C.Structure):
    """A batched render request (include/mcrt.h)."""

    _fields_ = [
        ("scene", C.c_void_p), ("geometry_version", C.c_int32), ("shading_version", C.c_int32),
        ("camera", mcrt_camera), ("settings", mcrt_settings), ("width", C.c_int32), ("height", C.c_int32),
        ("samples", C.c_int32), ("preview_block", C.c_int32), ("srgb", C.c_int32),
        ("image", C.POINTER(C.c_uint8)), ("preview_image", C.POINTER(C.c_uint8)),
        ("progress_image", C.POINTER(C.c_uint8)),
    ]


class mcrt_batch_event(C.Structure):
    _fields_ = [("id", C.c_int64), ("kind", C.c_int32), ("samples", C.c_int32)]


class mcrt_batch_stats(C.Structure):
    _fields_ = [
        ("closest_rays", C.c_uint64), ("any_rays", C.c_uint64), ("samples", C.c_uint64), ("chunks", C.c_uint64),
        ("graph_launches", C.c_uint64), ("gpu_ms", C.c_double), ("arena_bytes", C.c_uint64),
        ("arena_used", C.c_uint64), ("path_bytes", C.c_uint64), ("status", C.c_uint32), ("pad_", C.c_uint32),
    ]


class mcrt_mesh(C.Structure):
    _fields_ = [
        ("vertex_count", C.c_int32), ("index_count", C.c_int32), ("position", C.POINTER(C.c_float)),
        ("normal", C.POINTER(C.c_float)), ("uv", C.POINTER(C.c_float)), ("index", C.POINTER(C.c_uint32)),
    ]


class mcrt_instance(C.Structure):
    _fields_ = [
        ("world", C.c_double * 16), ("mesh", C.c_int32), ("material", C.c_uint32), ("flags", C.c_uint8),
        ("side", C.c_uint8), ("flat_shading", C.c_uint8), ("pad_", C.c_uint8 * 5),
    ]


class mcrt_build_info(C.Structure):
    _fields_ = [
        ("flatten_ms", C.c_double), ("build_ms", C.c_double), ("finish_ms", C.c_double), ("total_ms", C.c_double),
        ("triangle_count", C.c_int32), ("node_count", C.c_int32), ("levels", C.c_int32), ("bins", C.c_int32),
        ("geometry_bytes", C.c_uint64), ("build_bytes", C.c_uint64),
    ]


class mcrt_compiled_out(C.Structure):
    _fields_ = [
        ("triangles", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)), ("uvs", C.POINTER(C.c_float)),
        ("tangents", C.POINTER(C.c_float)), ("materials", C.POINTER(C.c_uint32)), ("flags", C.POINTER(C.c_uint8)),
        ("sides", C.POINTER(C.c_uint8)), ("bounds", C.POINTER(C.c_float)), ("nodes", C.POINTER(C.c_int32)),
        ("order", C.POINTER(C.c_uint32)), ("epsilon", C.c_double), ("triangle_count", C.c_int32),
        ("node_count", C.c_int32),
    ]


def ptr(array: np.ndarray, ctype: Any) -> Any:
    """Pointer to a C-contiguous numpy array's data, or NULL for an empty array."""
    if array is None or array.size == 0:
        return C.cast(None, C.POINTER(ctype))
    assert array.flags["C_CONTIGUOUS"], "arrays passed to C must be contiguous"
    return array.ctypes.data_as(C.POINTER(ctype))


def to_uint32(value: float) -> int:
    """ECMAScript ToUint32: what the reference's integer hash sees of a seed."""
    if value != value or value in (float("inf"), float("-inf")):
        return 0
    return int(value) % (1 << 32)  # int() truncates toward zero, as ToUint32 does


def _contiguous(array: np.ndarray, dtype: Any) -> np.ndarray:
    return np.ascontiguousarray(array, dtype=dtype)


def to_c_geometry(g: CompiledGeometry) -> Tuple[mcrt_geometry, List[Any]]:
    keep = [
        _contiguous(g.triangles, np.float32), _contiguous(g.normals, np.float32),
        _contiguous(g.uvs, np.float32), _contiguous(g.tangents, np.float32),
        _contiguous(g.colors, np.float32), _contiguous(g.materials, np.uint32),
        _contiguous(g.flags, np.uint8), _contiguous(g.sides, np.uint8),
        _contiguous(g.bvh.bounds, np.float32), _contiguous(g.bvh.nodes, np.int32),
    ]
    s = mcrt_geometry()
    s.triangle_count = g.triangle_count
    s.node_count = g.bvh.node_count
    s.triangles = ptr(keep[0], C.c_float)
    s.normals = ptr(keep[1], C.c_float)
    s.uvs = ptr(keep[2], C.c_float)
    s.tangents = ptr(keep[3], C.c_float)
    s.colors = ptr(keep[4], C.c_float)
    s.materials = ptr(keep[5], C.c_uint32)
    s.flags = ptr(keep[6], C.c_uint8)
    s.sides = ptr(keep[7], C.c_uint8)
    s.bvh_bounds = ptr(keep[8], C.c_float)
    s.bvh_nodes = ptr(keep[9], C.c_int32)
    s.epsilon = float(g.epsilon)
    return s, keep


def to_c_texture(t: CompiledTexture, texture_id: int = 0, with_data: bool = True) -> Tuple[mcrt_texture, List[Any]]:
    if t.data.dtype == np.float32:
        fmt, data = 1, _contiguous(t.data, np.float32)
    else:
        fmt, data = 0, _contiguous(t.data, np.uint8)
    if data.size != t.width * t.height * 4:
        raise ValueError(f"texture data has {data.size} values, expected {t.width * t.height * 4}")
    s = mcrt_texture()
    s.width, s.height, s.format = t.width, t.height, fmt
    s.srgb, s.flip_y = int(bool(t.srgb)), int(bool(t.flip_y))
    s.wrap_s, s.wrap_t, s.id = int(t.wrap_s), int(t.wrap_t), int(texture_id)
    s.matrix = c_double9(*[float(x) for x in t.matrix])
    s.data = data.ctypes.data if with_data else None
    return s, [data]


def to_c_shading(scene: CompiledScene, texture_ids: Sequence[int] = (), with_texture_data: bool = True
                 ) -> Tuple[mcrt_shading, List[Any]]:
    keep: List[Any] = []
    nm = len(scene.materials)
    mats = (mcrt_material * max(1, nm))()
    for i, m in enumerate(scene.materials):
        c = mats[i]
        c.model = MATERIAL_MODELS.index(m.model)
        c.side = int(m.side)
        c.color = c_double3(*m.color)
        c.opacity = float(m.opacity)
        c.transparent = int(bool(m.transparent))
        c.vertex_colors = int(bool(m.vertex_colors))
        c.alpha_test = float(m.alpha_test)
        c.flat_shading = int(bool(m.flat_shading))
        c.tone_mapped = int(bool(m.tone_mapped))
        c.map, c.alpha_map, c.emissive_map = int(m.map), int(m.alpha_map), int(m.emissive_map)
        c.normal_map, c.ao_map = int(m.normal_map), int(m.ao_map)
        c.roughness_map, c.metalness_map = int(m.roughness_map), int(m.metalness_map)
        c.physical = int(bool(m.physical))
        c.emissive = c_double3(*m.emissive)
        c.normal_scale = (C.c_double * 2)(*m.normal_scale)
        c.ao_map_intensity = float(m.ao_map_intensity)
        c.roughness, c.metalness = float(m.roughness), float(m.metalness)
        c.ior, c.specular_intensity = float(m.ior), float(m.specular_intensity)
        c.specular_color = c_double3(*m.specular_color)
        c.transmission, c.thickness = float(m.transmission), float(m.thickness)
        c.attenuation = c_double3(*m.attenuation)
        c.shininess = float(m.shininess)
        c.specular = c_double3(*m.specular)
        c.env_map, c.combine = int(m.env_map), int(m.combine)
        c.env_map_intensity, c.reflectivity = float(m.env_map_intensity), float(m.reflectivity)
    keep.append(mats)

    nt = len(scene.textures)
    texs = (mcrt_texture * max(1, nt))()
    for i, t in enumerate(scene.textures):
        tid = texture_ids[i] if i < len(texture_ids) else i + 1
        texs[i], k = to_c_texture(t, tid, with_texture_data)
        keep.extend(k)
    keep.append(texs)

    ne = len(scene.environments)
    envs = (mcrt_environment * max(1, ne))()
    for i, e in enumerate(scene.environments):
        c = envs[i]
        c.kind = 0 if e.kind == "cube" else 1
        c.faces = (C.c_int32 * 6)(*e.faces)
        c.texture = int(e.texture)
        c.flip_x = int(bool(e.flip_x))
        c.rotation = c_double9(*e.rotation)
        c.intensity = float(e.intensity)
    keep.append(envs)

    nl = len(scene.lights)
    lights = (mcrt_light * max(1, nl))()
    for i, l in enumerate(scene.lights):
        c = lights[i]
        c.type = LIGHT_TYPES.index(l.type)
        c.cast_shadow = int(bool(l.cast_shadow))
        c.color = c_double3(*l.color)
        c.ground_color = c_double3(*l.ground_color)
        c.direction = c_double3(*l.direction)
        c.position = c_double3(*l.position)
        c.distance, c.decay = float(l.distance), float(l.decay)
        c.cone_cos, c.penumbra_cos = float(l.cone_cos), float(l.penumbra_cos)
    keep.append(lights)

    s = mcrt_shading()
    s.material_count, s.texture_count, s.environment_count, s.light_count = nm, nt, ne, nl
    s.materials, s.textures, s.environments, s.lights = mats, texs, envs, lights
    b = scene.background
    s.background.kind = BACKGROUND_KINDS.index(b.kind)
    s.background.texture = int(b.texture)
    s.background.environment = int(b.environment)
    s.background.color = c_double3(*b.color)
    s.background.intensity = float(b.intensity)
    if scene.fog is None:
        s.fog.kind = 0
    else:
        f = scene.fog
        s.fog.kind = 1 if f.kind == "linear" else 2
        s.fog.color = c_double3(*f.color)
        s.fog.near_, s.fog.far_, s.fog.density = float(f.near), float(f.far), float(f.density)
    s.environment = int(scene.environment)
    return s, keep


def to_c_camera(cam: CompiledCamera) -> mcrt_camera:
    c = mcrt_camera()
    c.projection_inverse = c_double16(*[float(x) for x in cam.projection_inverse])
    c.world = c_double16(*[float(x) for x in cam.world])
    c.orthographic = int(bool(cam.orthographic))
    c.forward = c_double3(*cam.forward)
    c.position = c_double3(*cam.position)
    return c


def to_c_settings(s: TraceSettings) -> mcrt_settings:
    c = mcrt_settings()
    c.max_bounces = int(s.max_bounces)
    if s.shadows not in SHADOW_MODES:
        raise ValueError(f"unknown shadows mode {s.shadows!r}")
    c.shadows = SHADOW_MODES.index(s.shadows)
    c.global_illumination = int(bool(s.global_illumination))
    c.tone_mapping = int(s.tone_mapping)
    c.tone_mapping_exposure = float(s.tone_mapping_exposure)
    c.clear_color = c_double3(*s.clear_color)
    c.clear_alpha = float(s.clear_alpha)
    c.seed = to_uint32(s.seed)
    return c


def to_c_tile(t: Tile) -> mcrt_tile:
    return mcrt_tile(int(t.x), int(t.y), int(t.width), int(t.height))
