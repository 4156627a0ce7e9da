"""ctypes binding of the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY.

Only the test suite, the smoke check and the benchmark's CPU-baseline leg use
this module, as the checker for the CUDA path. It restates the reference's hot
path on the CPU (see oracle.cpp) and exposes it over the same compiled-scene
types the product consumes.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Any, Dict, Optional, Sequence, Tuple

import numpy as np

from meercadraytracer_b200 import abi
from meercadraytracer_b200.compile import TriangleSink
from meercadraytracer_b200.types import (
    CompiledBvh,
    CompiledCamera,
    CompiledGeometry,
    CompiledScene,
    CompiledTexture,
    CompiledEnvironment,
    Tile,
    TraceSettings,
)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class oracle_hit(C.Structure):
    _fields_ = [("triangle", C.c_int32), ("front", C.c_int32), ("t", C.c_double), ("u", C.c_double),
                ("v", C.c_double)]


class oracle_counters(C.Structure):
    _fields_ = [("closest_queries", C.c_int64), ("closest_boxes", C.c_int64), ("closest_tris", C.c_int64),
                ("any_queries", C.c_int64), ("any_boxes", C.c_int64), ("any_tris", C.c_int64),
                ("samples", C.c_int64)]

    def as_dict(self) -> Dict[str, int]:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


def build() -> str:
    """Compiles liboracle.so with its Makefile if it is missing or stale."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        d, i32, u32, P = C.c_double, C.c_int32, C.c_uint32, C.POINTER
        L.oracle_hash.restype = u32
        L.oracle_hash.argtypes = [u32]
        L.oracle_seed.restype = u32
        L.oracle_seed.argtypes = [u32, u32, u32, u32]
        L.oracle_random_next.restype = d
        L.oracle_random_next.argtypes = [P(u32)]
        for name in ("oracle_srgb_to_linear", "oracle_linear_to_srgb", "oracle_fresnel_weight"):
            getattr(L, name).restype = d
            getattr(L, name).argtypes = [d]
        L.oracle_half_to_float.restype = d
        L.oracle_half_to_float.argtypes = [u32]
        L.oracle_tone_map.argtypes = [P(d), C.c_int, d]
        L.oracle_uint8_clamp.restype = C.c_uint8
        L.oracle_uint8_clamp.argtypes = [d]
        L.oracle_dfg.argtypes = [d, d, P(d)]
        for name in ("oracle_visibility_ggx", "oracle_smoothstep", "oracle_distance_attenuation"):
            getattr(L, name).restype = d
            getattr(L, name).argtypes = [d, d, d]
        for name in ("oracle_distribution_ggx", "oracle_blinn_phong"):
            getattr(L, name).restype = d
            getattr(L, name).argtypes = [d, d]
        L.oracle_sample_texture.argtypes = [P(abi.mcrt_texture), d, d, P(d)]
        L.oracle_sample_environment.argtypes = [P(abi.mcrt_environment), P(abi.mcrt_texture), d, d, d, P(d)]
        L.oracle_plant_draw_mistake.argtypes = [i32]
        L.oracle_build_bvh.restype = i32
        L.oracle_build_bvh.argtypes = [P(C.c_float), i32, P(C.c_float), P(i32), P(u32)]
        L.oracle_build_bvh_bins.restype = i32
        L.oracle_build_bvh_bins.argtypes = [P(C.c_float), i32, i32, P(C.c_float), P(i32), P(u32)]
        L.oracle_intersect_closest.restype = i32
        L.oracle_intersect_closest.argtypes = [P(C.c_float), P(C.c_uint8), P(C.c_float), P(i32), i32, P(d), P(d),
                                               d, d, i32, P(oracle_hit), P(oracle_counters)]
        L.oracle_intersect_any_count.restype = i32
        L.oracle_intersect_any_count.argtypes = [P(C.c_float), P(C.c_float), P(i32), i32, P(d), P(d), d, d,
                                                 P(oracle_counters)]
        L.oracle_compile_geometry.restype = i32
        L.oracle_compile_geometry.argtypes = [
            i32, P(d), P(d), P(d), P(d), P(C.c_uint8), P(u32), P(C.c_uint8), P(C.c_uint8),
            P(C.c_float), P(C.c_float), P(C.c_float), P(C.c_float), P(C.c_float), P(u32), P(C.c_uint8),
            P(C.c_uint8), P(C.c_float), P(i32), P(u32), P(i32), P(d), P(i32), i32]
        L.oracle_camera_ray.argtypes = [P(abi.mcrt_camera), d, d, P(d)]
        L.oracle_render_tile.restype = i32
        L.oracle_render_tile.argtypes = [P(abi.mcrt_geometry), P(abi.mcrt_shading), P(abi.mcrt_camera),
                                         P(abi.mcrt_settings), P(abi.mcrt_tile), i32, i32, i32, i32,
                                         P(C.c_float), P(oracle_counters)]
        L.oracle_encode_tile.argtypes = [P(C.c_uint8), i32, P(abi.mcrt_tile), P(C.c_float), P(C.c_float), i32, i32]
        L.oracle_render_pixels.restype = i32
        L.oracle_render_pixels.argtypes = [P(abi.mcrt_geometry), P(abi.mcrt_shading), P(abi.mcrt_camera),
                                           P(abi.mcrt_settings), i32, i32, i32, i32, i32, P(i32), P(i32),
                                           P(C.c_uint8), P(C.c_float), i32, P(oracle_counters)]
        L.oracle_raytrace.restype = i32
        L.oracle_raytrace.argtypes = [P(abi.mcrt_geometry), P(abi.mcrt_shading), P(abi.mcrt_camera),
                                      P(abi.mcrt_settings), i32, i32, i32, i32, P(C.c_uint8), i32,
                                      P(oracle_counters)]
        L.oracle_trace_primary.restype = i32
        L.oracle_trace_primary.argtypes = [P(abi.mcrt_geometry), P(abi.mcrt_camera), i32, i32, i32, u32, i32,
                                           P(i32), P(i32), P(i32), P(d), P(d), P(d), P(i32), P(d), i32]
        _lib = L
    return _lib


def _p(a: np.ndarray, t: Any) -> Any:
    return abi.ptr(a, t)


# ----------------------------------------------------------- scalar functions
def hash32(x: int) -> int:
    return int(lib().oracle_hash(x & 0xFFFFFFFF))


def seed(a: int, b: int, c: int, d: int) -> int:
    m = 0xFFFFFFFF
    return int(lib().oracle_seed(a & m, b & m, c & m, d & m))


def random_sequence(state: int, n: int) -> Tuple[list, int]:
    s = C.c_uint32(state)
    values = [lib().oracle_random_next(C.byref(s)) for _ in range(n)]
    return values, int(s.value)


def srgb_to_linear(c: float) -> float:
    return lib().oracle_srgb_to_linear(c)


def linear_to_srgb(c: float) -> float:
    return lib().oracle_linear_to_srgb(c)


def half_to_float(h: int) -> float:
    return lib().oracle_half_to_float(h)


def tone_map(c: Sequence[float], mapping: int, exposure: float = 1.0) -> list:
    arr = (C.c_double * 3)(*c)
    lib().oracle_tone_map(arr, mapping, exposure)
    return list(arr)


def uint8_clamp(v: float) -> int:
    return int(lib().oracle_uint8_clamp(v))


def dfg(roughness: float, dot_nv: float) -> Tuple[float, float]:
    out = (C.c_double * 2)()
    lib().oracle_dfg(roughness, dot_nv, out)
    return out[0], out[1]


def fresnel_weight(x: float) -> float:
    return lib().oracle_fresnel_weight(x)


def visibility_ggx(alpha: float, nl: float, nv: float) -> float:
    return lib().oracle_visibility_ggx(alpha, nl, nv)


def distribution_ggx(alpha: float, nh: float) -> float:
    return lib().oracle_distribution_ggx(alpha, nh)


def blinn_phong(shininess: float, nh: float) -> float:
    return lib().oracle_blinn_phong(shininess, nh)


def smoothstep(e0: float, e1: float, x: float) -> float:
    return lib().oracle_smoothstep(e0, e1, x)


def distance_attenuation(d: float, cutoff: float, decay: float) -> float:
    return lib().oracle_distance_attenuation(d, cutoff, decay)


def sample_texture(texture: CompiledTexture, u: float, v: float) -> list:
    t, keep = abi.to_c_texture(texture)
    out = (C.c_double * 4)()
    lib().oracle_sample_texture(C.byref(t), u, v, out)
    return list(out)


def sample_environment(env: CompiledEnvironment, textures: Sequence[CompiledTexture], d: Sequence[float]) -> list:
    scene = CompiledScene(geometry=None, textures=list(textures), environments=[env])  # type: ignore[arg-type]
    sh, keep = abi.to_c_shading(scene)
    out = (C.c_double * 3)()
    lib().oracle_sample_environment(sh.environments, sh.textures, d[0], d[1], d[2], out)
    return list(out)


def plant_draw_mistake(which: int) -> None:
    """Test only: reorders one of the path loop's random draws in the oracle (1-6, see
    oracle.cpp); 0 restores the reference's order."""
    lib().oracle_plant_draw_mistake(int(which))


# ------------------------------------------------------------------------ bvh
def build_bvh(triangles: np.ndarray, count: int, bins: int = 16) -> Tuple[CompiledBvh, np.ndarray]:
    """buildBvh, src/bvh.ts:16-178, with `bins` SAH bins per axis (the reference's BINS is 16)."""
    tris = np.ascontiguousarray(triangles, np.float32)
    cap = max(1, 2 * count - 1)
    bounds = np.zeros(cap * 6, np.float32)
    nodes = np.zeros(cap * 3, np.int32)
    order = np.zeros(max(1, count), np.uint32)
    n = lib().oracle_build_bvh_bins(_p(tris, C.c_float), count, int(bins), _p(bounds, C.c_float),
                                    _p(nodes, C.c_int32), _p(order, C.c_uint32))
    return CompiledBvh(bounds[: n * 6].copy(), nodes[: n * 3].copy(), int(n)), order[:count].copy()


def intersect_closest(triangles: np.ndarray, sides: np.ndarray, bvh: CompiledBvh, o: Sequence[float],
                      d: Sequence[float], t_min: float = 0.0, t_max: float = float("inf"), cull: bool = True,
                      counters: Optional[oracle_counters] = None) -> Tuple[bool, oracle_hit]:
    hit = oracle_hit()
    tris = np.ascontiguousarray(triangles, np.float32)
    sd = np.ascontiguousarray(sides, np.uint8)
    found = lib().oracle_intersect_closest(
        _p(tris, C.c_float), _p(sd, C.c_uint8), _p(bvh.bounds, C.c_float), _p(bvh.nodes, C.c_int32),
        bvh.node_count, (C.c_double * 3)(*o), (C.c_double * 3)(*d), t_min, t_max, int(cull), C.byref(hit),
        C.byref(counters) if counters is not None else None)
    return bool(found), hit


def intersect_any_count(triangles: np.ndarray, bvh: CompiledBvh, o: Sequence[float], d: Sequence[float],
                        t_min: float = 0.0, t_max: float = float("inf")) -> int:
    tris = np.ascontiguousarray(triangles, np.float32)
    return int(lib().oracle_intersect_any_count(
        _p(tris, C.c_float), _p(bvh.bounds, C.c_float), _p(bvh.nodes, C.c_int32), bvh.node_count,
        (C.c_double * 3)(*o), (C.c_double * 3)(*d), t_min, t_max, None))


# -------------------------------------------------------------------- compile
def compile_sink(sink: TriangleSink, bins: int = 16) -> CompiledGeometry:
    """compileGeometry after the flatten (src/compile.ts:359-403): the oracle's geometry builder,
    with `bins` SAH bins per axis in the BVH build (16 as the reference)."""
    n = sink.count
    cap = max(1, 2 * n - 1)
    f32, u8, u32 = np.float32, np.uint8, np.uint32
    tris, nrm = np.zeros(n * 9, f32), np.zeros(n * 9, f32)
    uvs, tan = np.zeros(n * 6, f32), np.zeros(n * 4, f32)
    colors = np.zeros(n * 12, f32)
    mats, flags, sides = np.zeros(n, u32), np.zeros(n, u8), np.zeros(n, u8)
    bounds, nodes, order = np.zeros(cap * 6, f32), np.zeros(cap * 3, np.int32), np.zeros(max(1, n), u32)
    node_count, eps, any_colors = C.c_int32(), C.c_double(), C.c_int32()
    c = lambda a, dt: np.ascontiguousarray(a, dt)  # noqa: E731
    p, nn, uv, col = c(sink.p, np.float64), c(sink.n, np.float64), c(sink.uv, np.float64), c(sink.colors, np.float64)
    hc, sm, sf, ss = c(sink.has_color, u8), c(sink.materials, u32), c(sink.flags, u8), c(sink.sides, u8)
    D = C.c_double
    lib().oracle_compile_geometry(
        n, _p(p, D), _p(nn, D), _p(uv, D), _p(col, D), _p(hc, C.c_uint8), _p(sm, C.c_uint32), _p(sf, C.c_uint8),
        _p(ss, C.c_uint8), _p(tris, C.c_float), _p(nrm, C.c_float), _p(uvs, C.c_float), _p(tan, C.c_float),
        _p(colors, C.c_float), _p(mats, C.c_uint32), _p(flags, C.c_uint8), _p(sides, C.c_uint8),
        _p(bounds, C.c_float), _p(nodes, C.c_int32), _p(order, C.c_uint32), C.byref(node_count), C.byref(eps),
        C.byref(any_colors), int(bins))
    m = int(node_count.value)
    return CompiledGeometry(
        triangle_count=n, triangles=tris, normals=nrm, uvs=uvs, tangents=tan,
        colors=colors if any_colors.value else np.zeros(0, f32), materials=mats, flags=flags, sides=sides,
        bvh=CompiledBvh(bounds[: m * 6].copy(), nodes[: m * 3].copy(), m), epsilon=float(eps.value),
        order=order[:n].copy())


# --------------------------------------------------------------------- tracer
class _Views:
    """C views of a compiled scene, kept alive together."""

    def __init__(self, scene: CompiledScene, camera: CompiledCamera, settings: TraceSettings):
        self.geometry, k1 = abi.to_c_geometry(scene.geometry)
        self.shading, k2 = abi.to_c_shading(scene)
        self.camera = abi.to_c_camera(camera)
        self.settings = abi.to_c_settings(settings)
        self.keep = (k1, k2)


def camera_ray(camera: CompiledCamera, x: float, y: float) -> list:
    c = abi.to_c_camera(camera)
    out = (C.c_double * 6)()
    lib().oracle_camera_ray(C.byref(c), x, y, out)
    return list(out)


def render_tile(scene: CompiledScene, camera: CompiledCamera, settings: TraceSettings, tile: Tile, width: int,
                height: int, pass_: int, block: int = 1) -> np.ndarray:
    """Tracer.renderTile, src/tracer.ts:62-89: premultiplied RGBA floats."""
    v = _Views(scene, camera, settings)
    out = np.zeros(tile.width * tile.height * 4, np.float32)
    t = abi.to_c_tile(tile)
    lib().oracle_render_tile(C.byref(v.geometry), C.byref(v.shading), C.byref(v.camera), C.byref(v.settings),
                             C.byref(t), width, height, pass_, block, _p(out, C.c_float), None)
    return out


def encode_tile(image: np.ndarray, width: int, tile: Tile, data: np.ndarray, sum_: Optional[np.ndarray], count: int,
                srgb: bool) -> None:
    """writeTile / encodeTile, src/progressive.ts:288-313, in place."""
    t = abi.to_c_tile(tile)
    lib().oracle_encode_tile(_p(image, C.c_uint8), width, C.byref(t), _p(np.ascontiguousarray(data, np.float32),
                             C.c_float), _p(sum_, C.c_float) if sum_ is not None else None, count, int(srgb))


def render_pixels(scene: CompiledScene, camera: CompiledCamera, settings: TraceSettings, width: int, height: int,
                  samples: int, srgb: bool, px: np.ndarray, py: np.ndarray, threads: int = 1,
                  counters: Optional[oracle_counters] = None) -> Tuple[np.ndarray, np.ndarray]:
    """raytraceCompiled restricted to listed pixels: (rgba uint8 [n,4], float sums [n,4])."""
    v = _Views(scene, camera, settings)
    px = np.ascontiguousarray(px, np.int32)
    py = np.ascontiguousarray(py, np.int32)
    n = px.size
    rgba = np.zeros(n * 4, np.uint8)
    sums = np.zeros(n * 4, np.float32)
    lib().oracle_render_pixels(C.byref(v.geometry), C.byref(v.shading), C.byref(v.camera), C.byref(v.settings),
                               width, height, samples, int(srgb), n, _p(px, C.c_int32), _p(py, C.c_int32),
                               _p(rgba, C.c_uint8), _p(sums, C.c_float), threads,
                               C.byref(counters) if counters is not None else None)
    return rgba.reshape(n, 4), sums.reshape(n, 4)


def raytrace_compiled(scene: CompiledScene, camera: CompiledCamera, width: int, height: int,
                      settings: TraceSettings, samples: int = 16, srgb: bool = True, threads: int = 1,
                      counters: Optional[oracle_counters] = None) -> np.ndarray:
    """raytraceCompiled, src/raytrace.ts:69-82: RGBA8 image, top row first."""
    v = _Views(scene, camera, settings)
    out = np.zeros(width * height * 4, np.uint8)
    lib().oracle_raytrace(C.byref(v.geometry), C.byref(v.shading), C.byref(v.camera), C.byref(v.settings), width,
                          height, max(1, samples), int(srgb), _p(out, C.c_uint8), threads,
                          C.byref(counters) if counters is not None else None)
    return out


def trace_primary(scene: CompiledScene, camera: CompiledCamera, width: int, height: int, pass_: int, seed_: int,
                  px: np.ndarray, py: np.ndarray, threads: int = 1) -> Dict[str, np.ndarray]:
    """The first closest-hit query of each listed pixel's sample for one pass."""
    g, keep = abi.to_c_geometry(scene.geometry)
    cam = abi.to_c_camera(camera)
    px = np.ascontiguousarray(px, np.int32)
    py = np.ascontiguousarray(py, np.int32)
    n = px.size
    tri = np.zeros(n, np.int32)
    t, u, v = np.zeros(n), np.zeros(n), np.zeros(n)
    front = np.zeros(n, np.int32)
    rays = np.zeros(n * 6)
    D = C.c_double
    lib().oracle_trace_primary(C.byref(g), C.byref(cam), width, height, pass_, abi.to_uint32(seed_), n,
                               _p(px, C.c_int32), _p(py, C.c_int32), _p(tri, C.c_int32), _p(t, D), _p(u, D),
                               _p(v, D), _p(front, C.c_int32), _p(rays, D), threads)
    return {"tri": tri, "t": t, "u": u, "v": v, "front": front, "rays": rays.reshape(n, 6)}
