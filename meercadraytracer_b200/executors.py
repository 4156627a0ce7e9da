"""The GPU tile executor: the TileExecutor interface of src/executors.ts:4-14
backed by an executor of libmcrt (include/mcrt.h) on one CUDA device.

Messages are the reference's RequestMessage (src/protocol.ts:29-45) as dicts
with snake_case keys:

  {"type": "geometry", "version": v, "geometry": CompiledGeometry}
  {"type": "textures", "items": [{"id": i, "data": ndarray}, ...]}
  {"type": "shading", "version": v, "shading": ShadingPayload}
  {"type": "tile", "job": j, "geometry_version": g, "shading_version": s,
   "camera": CompiledCamera, "settings": TraceSettings, "tile": Tile,
   "width": w, "height": h, "pass": p, "block": b}

`render` resolves with the tile's premultiplied RGBA float32 samples, as the
worker's Tracer.renderTile does; a tile that refers to a scene the executor
has not received, or any GPU failure, rejects it with an Error, as
createTileHandler answers {type: 'error'} (src/protocol.ts:75-104). There is
no CPU fallback: failures surface to the caller.
"""
from __future__ import annotations

import ctypes as C
import threading
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence, Set, Tuple

import numpy as np

from . import abi
from ._lib import NOALLOC_MAX_RAYS, McrtError, call, load, mcrt_stats
from .types import (
    CompiledBvh,
    CompiledCamera,
    CompiledGeometry,
    CompiledScene,
    CompiledTexture,
    Tile,
    TraceSettings,
)


@dataclass
class ShadingPayload:
    """ShadingPayload, src/protocol.ts:19-27: everything but geometry and texture pixels."""

    materials: list
    textures: list  # CompiledTexture metadata; `texture_ids[i]` names the pixels of textures[i]
    texture_ids: List[int]
    environments: list
    lights: list
    background: Any
    environment: int
    fog: Any

    @staticmethod
    def of(scene: CompiledScene, texture_ids: Sequence[int]) -> "ShadingPayload":
        return ShadingPayload(scene.materials, scene.textures, list(texture_ids), scene.environments, scene.lights,
                              scene.background, scene.environment, scene.fog)


class GpuExecutor:
    """One CUDA device as a TileExecutor: the scene stays resident in HBM."""

    # One render at a time per executor: whole frames already fill the GPU.
    concurrency = 1

    def __init__(self, device: int = 0):
        load()
        handle = C.c_void_p()
        call("mcrt_executor_create", int(device), C.byref(handle))
        self._h = handle
        self.device = device
        self.textures: Set[int] = set()  # texture ids this executor holds (TileExecutor.textures)
        self._pending_pixels: Dict[int, np.ndarray] = {}
        self._lock = threading.Lock()
        self._worker = ThreadPoolExecutor(max_workers=1, thread_name_prefix=f"mcrt{device}")
        self._disposed = False
        self._geometry_version: Optional[int] = None
        self._shading_version: Optional[int] = None
        self._versions = 0
        self._scene_ref: Optional[CompiledScene] = None
        self._geometry_ref: Optional[CompiledGeometry] = None
        self._slots: Tuple[int, int] = (0, 0)

    # ------------------------------------------------------------ messages
    def send(self, message: Dict[str, Any], transfer: Any = None) -> None:
        """TileExecutor.send: messages are processed in the order they are sent."""
        self._check()
        kind = message["type"]
        with self._lock:
            if kind == "geometry":
                g, keep = abi.to_c_geometry(message["geometry"])
                call("mcrt_send_geometry", self._h, int(message["version"]), C.byref(g))
                self._geometry_version = int(message["version"])
            elif kind == "textures":
                for item in message["items"]:
                    self._pending_pixels[int(item["id"])] = item["data"]
                    self.textures.add(int(item["id"]))
            elif kind == "shading":
                sh: ShadingPayload = message["shading"]
                self._send_shading(int(message["version"]), sh)
            else:
                raise ValueError(f"unknown message type {kind!r}")

    def _send_shading(self, version: int, sh: ShadingPayload) -> None:
        scene = CompiledScene(geometry=None, materials=sh.materials, textures=[], environments=sh.environments,  # type: ignore[arg-type]
                              lights=sh.lights, background=sh.background, environment=sh.environment, fog=sh.fog)
        s, keep = abi.to_c_shading(scene)
        arr = (abi.mcrt_texture * max(1, len(sh.textures)))()
        fresh = []
        for i, (t, tid) in enumerate(zip(sh.textures, sh.texture_ids)):
            # Pixels travel once per executor (src/progressive.ts:140-148); a
            # texture without them here refers to pixels uploaded before.
            data = self._pending_pixels.get(tid)
            meta = CompiledTexture(t.width, t.height, data if data is not None else t.data, t.srgb, t.flip_y,
                                   t.wrap_s, t.wrap_t, t.matrix)
            arr[i], k = abi.to_c_texture(meta, tid, with_data=data is not None)
            keep.extend(k)
            if data is not None:
                fresh.append(tid)
        s.texture_count = len(sh.textures)
        s.textures = arr
        keep.append(arr)
        call("mcrt_send_shading", self._h, version, C.byref(s))
        for tid in fresh:
            self._pending_pixels.pop(tid, None)
        self._shading_version = version

    def render(self, message: Dict[str, Any]) -> "Future[np.ndarray]":
        """TileExecutor.render: resolves with the tile's premultiplied RGBA floats."""
        fut: Future = Future()
        if self._disposed:
            fut.set_exception(RuntimeError("the renderer was disposed"))
            return fut
        return self._worker.submit(self._render_tile, message)

    def _render_tile(self, m: Dict[str, Any]) -> np.ndarray:
        tile: Tile = m["tile"]
        out = np.zeros(tile.width * tile.height * 4, np.float32)
        cam = abi.to_c_camera(m["camera"])
        st = abi.to_c_settings(m["settings"])
        t = abi.to_c_tile(tile)
        with self._lock:
            call("mcrt_render_tile", self._h, int(m["geometry_version"]), int(m["shading_version"]), C.byref(cam),
                 C.byref(st), C.byref(t), int(m["width"]), int(m["height"]), int(m["pass"]), int(m.get("block", 1)),
                 abi.ptr(out, C.c_float))
        return out

    def dispose(self) -> None:
        """TileExecutor.dispose: frees the device state."""
        if self._disposed:
            return
        self._disposed = True
        self._worker.shutdown(wait=True)
        call("mcrt_executor_destroy", self._h)
        self._h = None

    def __del__(self):  # pragma: no cover - best effort
        try:
            if not self._disposed and self._h is not None:
                self.dispose()
        except Exception:
            pass

    def _check(self) -> None:
        if self._disposed:
            raise RuntimeError("the renderer was disposed")

    # ---------------------------------------------------- whole-scene calls
    def load_scene(self, scene: CompiledScene) -> Tuple[int, int]:
        """Makes `scene` resident (geometry, texture pixels, shading) unless it already is."""
        self._check()
        # Hold the scene itself: comparing id()s alone could match a new scene
        # allocated where a freed one was.
        if self._scene_ref is scene and self._geometry_ref is scene.geometry and self._geometry_version is not None:
            return self._slots
        self._versions += 1
        gv = sv = self._versions
        self.send({"type": "geometry", "version": gv, "geometry": scene.geometry})
        ids = [self._versions * 100000 + i for i in range(len(scene.textures))]
        self.send({"type": "textures", "items": [{"id": i, "data": t.data} for i, t in zip(ids, scene.textures)]})
        self.send({"type": "shading", "version": sv, "shading": ShadingPayload.of(scene, ids)})
        self._scene_ref = scene
        self._geometry_ref = scene.geometry
        self._slots = (gv, sv)
        return gv, sv

    def raytrace(self, scene: CompiledScene, camera: CompiledCamera, width: int, height: int,
                 settings: TraceSettings, samples: int = 16, srgb: bool = True) -> np.ndarray:
        """raytraceCompiled (src/raytrace.ts:69-82) on the device: RGBA8 bytes."""
        gv, sv = self.load_scene(scene)
        out = np.zeros(width * height * 4, np.uint8)
        cam, st = abi.to_c_camera(camera), abi.to_c_settings(settings)
        with self._lock:
            call("mcrt_raytrace", self._h, gv, sv, C.byref(cam), C.byref(st), int(width), int(height), int(samples),
                 int(bool(srgb)), abi.ptr(out, C.c_uint8))
        return out

    def raytrace_device(self, scene: CompiledScene, camera: CompiledCamera, width: int, height: int,
                        settings: TraceSettings, samples: int, srgb: bool, device_ptr: int) -> None:
        """As raytrace, leaving the image in device memory at `device_ptr`."""
        gv, sv = self.load_scene(scene)
        cam, st = abi.to_c_camera(camera), abi.to_c_settings(settings)
        with self._lock:
            call("mcrt_raytrace_device", self._h, gv, sv, C.byref(cam), C.byref(st), int(width), int(height),
                 int(samples), int(bool(srgb)), C.c_void_p(device_ptr))

    def raytrace_resident(self, versions: Tuple[int, int], camera: CompiledCamera, width: int, height: int,
                          settings: TraceSettings, samples: int, srgb: bool = True,
                          device_ptr: Optional[int] = None) -> Optional[np.ndarray]:
        """raytraceCompiled on the geometry and shading versions this executor holds (for
        geometry made by compile_instances): RGBA8 bytes, or into `device_ptr`."""
        cam, st = abi.to_c_camera(camera), abi.to_c_settings(settings)
        gv, sv = int(versions[0]), int(versions[1])
        with self._lock:
            if device_ptr is not None:
                call("mcrt_raytrace_device", self._h, gv, sv, C.byref(cam), C.byref(st), int(width), int(height),
                     int(samples), int(bool(srgb)), C.c_void_p(device_ptr))
                return None
            out = np.zeros(width * height * 4, np.uint8)
            call("mcrt_raytrace", self._h, gv, sv, C.byref(cam), C.byref(st), int(width), int(height), int(samples),
                 int(bool(srgb)), abi.ptr(out, C.c_uint8))
            return out

    def render_pixels(self, scene: CompiledScene, camera: CompiledCamera, width: int, height: int,
                      settings: TraceSettings, samples: int, srgb: bool, px: np.ndarray, py: np.ndarray
                      ) -> Tuple[np.ndarray, np.ndarray]:
        """raytraceCompiled for listed pixels: (rgba uint8 [n, 4], sums float32 [n, 4])."""
        gv, sv = self.load_scene(scene)
        px = np.ascontiguousarray(px, np.int32)
        py = np.ascontiguousarray(py, np.int32)
        n = px.size
        rgba = np.zeros(n * 4, np.uint8)
        sums = np.zeros(n * 4, np.float32)
        cam, st = abi.to_c_camera(camera), abi.to_c_settings(settings)
        with self._lock:
            call("mcrt_render_pixels", self._h, gv, sv, C.byref(cam), C.byref(st), int(width), int(height),
                 int(samples), int(bool(srgb)), n, abi.ptr(px, C.c_int32), abi.ptr(py, C.c_int32),
                 abi.ptr(rgba, C.c_uint8), abi.ptr(sums, C.c_float))
        return rgba.reshape(n, 4), sums.reshape(n, 4)

    def trace_primary(self, scene: CompiledScene, camera: CompiledCamera, width: int, height: int, pass_: int,
                      seed: float, px: np.ndarray, py: np.ndarray) -> Dict[str, np.ndarray]:
        gv, _ = self.load_scene(scene)
        px = np.ascontiguousarray(px, np.int32)
        py = np.ascontiguousarray(py, np.int32)
        n = px.size
        tri = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        front = np.zeros(n, np.int32)
        cam = abi.to_c_camera(camera)
        with self._lock:
            call("mcrt_trace_primary", self._h, gv, C.byref(cam), int(width), int(height), int(pass_),
                 abi.to_uint32(seed), n, abi.ptr(px, C.c_int32), abi.ptr(py, C.c_int32), abi.ptr(tri, C.c_int32),
                 abi.ptr(t, C.c_float), abi.ptr(front, C.c_int32))
        return {"tri": tri, "t": t, "front": front}

    def intersect_closest(self, geometry_version: int, rays: np.ndarray, cull: bool = True
                          ) -> Dict[str, np.ndarray]:
        """intersectClosest for rays [n, 8] (origin, -, direction, -) on the resident geometry."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        tri = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        u = np.zeros(n, np.float32)
        front = np.zeros(n, np.int32)
        with self._lock:
            call("mcrt_intersect_closest", self._h, int(geometry_version), n, abi.ptr(rays, C.c_float), int(cull),
                 abi.ptr(tri, C.c_int32), abi.ptr(t, C.c_float), abi.ptr(u, C.c_float), abi.ptr(front, C.c_int32))
        return {"tri": tri, "t": t, "u": u, "front": front}

    def intersect_closest_noalloc(self, geometry_version: int, rays: np.ndarray, cull: bool = True
                                  ) -> Dict[str, np.ndarray]:
        """intersect_closest through mcrt_intersect_closest_noalloc: no device memory is allocated
        during the call (working memory is the library's fixed per-device array), at most
        NOALLOC_MAX_RAYS rays. The array is shared by every executor on the device, so calls from
        different executors must not overlap; this executor's lock serialises its own calls."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        tri = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        u = np.zeros(n, np.float32)
        front = np.zeros(n, np.int32)
        with self._lock:
            call("mcrt_intersect_closest_noalloc", self._h, int(geometry_version), n, abi.ptr(rays, C.c_float),
                 int(cull), abi.ptr(tri, C.c_int32), abi.ptr(t, C.c_float), abi.ptr(u, C.c_float),
                 abi.ptr(front, C.c_int32))
        return {"tri": tri, "t": t, "u": u, "front": front}

    def intersect_any_count(self, geometry_version: int, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        counts = np.zeros(n, np.int32)
        with self._lock:
            call("mcrt_intersect_any_count", self._h, int(geometry_version), n, abi.ptr(rays, C.c_float),
                 abi.ptr(counts, C.c_int32))
        return counts

    # ------------------------------------------------------------ compile
    def build_bvh(self, triangles: np.ndarray, count: int) -> Tuple[CompiledBvh, np.ndarray]:
        """buildBvh (src/bvh.ts:16-178) on the GPU."""
        tris = np.ascontiguousarray(triangles, np.float32)
        cap = max(1, 2 * count - 1)
        bounds = np.zeros(cap * 6, np.float32)
        nodes = np.zeros(cap * 3, np.int32)
        order = np.zeros(max(1, count), np.uint32)
        m = C.c_int32()
        with self._lock:
            call("mcrt_build_bvh", self._h, abi.ptr(tris, C.c_float), int(count), abi.ptr(bounds, C.c_float),
                 abi.ptr(nodes, C.c_int32), abi.ptr(order, C.c_uint32), C.byref(m))
        k = int(m.value)
        return CompiledBvh(bounds[: k * 6].copy(), nodes[: k * 3].copy(), k), order[:count].copy()

    def compile_sink(self, sink: Any) -> CompiledGeometry:
        """compileGeometry after the flatten (src/compile.ts:359-403) on the GPU."""
        n = sink.count
        cap = max(1, 2 * n - 1)
        f32, u8, u32 = np.float32, np.uint8, np.uint32
        tris, nrm = np.zeros(n * 9, f32), np.zeros(n * 9, f32)
        uvs, tan = np.zeros(n * 6, f32), np.zeros(n * 4, f32)
        colors = np.zeros(max(1, n * 12), f32)
        mats, flags, sides = np.zeros(n, u32), np.zeros(n, u8), np.zeros(n, u8)
        bounds, nodes, order = np.zeros(cap * 6, f32), np.zeros(cap * 3, np.int32), np.zeros(max(1, n), u32)
        node_count, eps, any_colors = C.c_int32(), C.c_double(), C.c_int32()
        c = lambda a, dt: np.ascontiguousarray(a, dt)  # noqa: E731
        p, nn, uv, col = c(sink.p, np.float64), c(sink.n, np.float64), c(sink.uv, np.float64), c(sink.colors, np.float64)
        hc, sm, sf, ss = c(sink.has_color, u8), c(sink.materials, u32), c(sink.flags, u8), c(sink.sides, u8)
        P, D = abi.ptr, C.c_double
        with self._lock:
            call("mcrt_compile_geometry", self._h, n, P(p, D), P(nn, D), P(uv, D), P(col, D), P(hc, C.c_uint8),
                 P(sm, C.c_uint32), P(sf, C.c_uint8), P(ss, C.c_uint8), P(tris, C.c_float), P(nrm, C.c_float),
                 P(uvs, C.c_float), P(tan, C.c_float), P(colors, C.c_float), P(mats, C.c_uint32), P(flags, C.c_uint8),
                 P(sides, C.c_uint8), P(bounds, C.c_float), P(nodes, C.c_int32), P(order, C.c_uint32),
                 C.byref(node_count), C.byref(eps), C.byref(any_colors))
        m = int(node_count.value)
        return CompiledGeometry(
            triangle_count=n, triangles=tris, normals=nrm, uvs=uvs, tangents=tan,
            colors=colors[: n * 12].copy() if any_colors.value else np.zeros(0, f32), materials=mats, flags=flags,
            sides=sides, bvh=CompiledBvh(bounds[: m * 6].copy(), nodes[: m * 3].copy(), m), epsilon=float(eps.value),
            order=order[:n].copy())

    # ----------------------------------------------------- instanced geometry
    def upload_meshes(self, meshes: Sequence[Any]) -> None:
        """Meshes for compile_instances: BufferGeometry-like objects with `position` (and
        optionally `normal`, `uv`, `index`) arrays, kept on the device."""
        arr = (abi.mcrt_mesh * max(1, len(meshes)))()
        keep = []
        for i, g in enumerate(meshes):
            pos = np.ascontiguousarray(np.asarray(g.position, np.float32).reshape(-1))
            nrm = None if g.normal is None else np.ascontiguousarray(np.asarray(g.normal, np.float32).reshape(-1))
            uv = None if g.uv is None else np.ascontiguousarray(np.asarray(g.uv, np.float32).reshape(-1))
            idx = None if g.index is None else np.ascontiguousarray(np.asarray(g.index, np.uint32).reshape(-1))
            keep += [pos, nrm, uv, idx]
            arr[i].vertex_count = pos.size // 3
            arr[i].index_count = 0 if idx is None else idx.size
            arr[i].position = abi.ptr(pos, C.c_float)
            arr[i].normal = abi.ptr(nrm, C.c_float)
            arr[i].uv = abi.ptr(uv, C.c_float)
            arr[i].index = abi.ptr(idx, C.c_uint32)
        with self._lock:
            call("mcrt_upload_meshes", self._h, len(meshes), arr)
        self._mesh_tris = [(arr[i].index_count or arr[i].vertex_count) // 3 for i in range(len(meshes))]

    def compile_instances(self, instances: Sequence[Tuple[Any, int, int, int, int, bool]], bins: int = 16,
                          download: bool = False) -> Tuple[Dict[str, Any], Optional[CompiledGeometry]]:
        """compileGeometry of instances of the uploaded meshes, on the GPU: each instance is
        (world matrix [16] column-major, mesh, material, flags, side, flat_shading). The result
        is resident (geometry version returned in the info); with `download` the compiled arrays
        come back as a CompiledGeometry too."""
        arr = (abi.mcrt_instance * max(1, len(instances)))()
        for i, (world, mesh, material, flags, side, flat) in enumerate(instances):
            w = np.asarray(world, np.float64).reshape(16)
            for k in range(16):
                arr[i].world[k] = float(w[k])
            arr[i].mesh, arr[i].material = int(mesh), int(material)
            arr[i].flags, arr[i].side, arr[i].flat_shading = int(flags), int(side), int(bool(flat))
        self._versions += 1
        version = self._versions
        info = abi.mcrt_build_info()
        out = None
        out_c = None
        if download:
            n = self._instance_triangles(instances)
            cap = max(1, 2 * n - 1)
            f32 = np.float32
            out = {"triangles": np.zeros(9 * n, f32), "normals": np.zeros(9 * n, f32), "uvs": np.zeros(6 * n, f32),
                   "tangents": np.zeros(4 * n, f32), "materials": np.zeros(n, np.uint32), "flags": np.zeros(n, np.uint8),
                   "sides": np.zeros(n, np.uint8), "bounds": np.zeros(6 * cap, f32), "nodes": np.zeros(3 * cap, np.int32),
                   "order": np.zeros(max(1, n), np.uint32)}
            out_c = abi.mcrt_compiled_out()
            types = {"triangles": C.c_float, "normals": C.c_float, "uvs": C.c_float, "tangents": C.c_float,
                     "materials": C.c_uint32, "flags": C.c_uint8, "sides": C.c_uint8, "bounds": C.c_float,
                     "nodes": C.c_int32, "order": C.c_uint32}
            for k, t in types.items():
                setattr(out_c, k, abi.ptr(out[k], t))
        with self._lock:
            call("mcrt_compile_instances", self._h, version, len(instances), arr, int(bins), C.byref(info),
                 C.byref(out_c) if out_c is not None else None)
            self._geometry_version = version
            self._scene_ref = None
            self._geometry_ref = None
        d = {name: getattr(info, name) for name, _ in info._fields_}
        d["version"] = version
        geometry = None
        if out is not None:
            m = int(out_c.node_count)
            n = int(out_c.triangle_count)
            geometry = CompiledGeometry(
                triangle_count=n, triangles=out["triangles"], normals=out["normals"], uvs=out["uvs"],
                tangents=out["tangents"], colors=np.zeros(0, np.float32), materials=out["materials"],
                flags=out["flags"], sides=out["sides"],
                bvh=CompiledBvh(out["bounds"][: 6 * m].copy(), out["nodes"][: 3 * m].copy(), m),
                epsilon=float(out_c.epsilon), order=out["order"][:n].copy())
        return d, geometry

    def _instance_triangles(self, instances: Sequence[Any]) -> int:
        if not hasattr(self, "_mesh_tris"):
            raise RuntimeError("upload_meshes first")
        return int(sum(self._mesh_tris[int(inst[1])] for inst in instances))

    def send_shading_only(self, scene: CompiledScene) -> int:
        """Sends a scene's textures and shading (materials, lights, ...) without geometry;
        returns the shading version, for geometry made by compile_instances."""
        self._versions += 1
        sv = self._versions
        ids = [sv * 100000 + i for i in range(len(scene.textures))]
        self.send({"type": "textures", "items": [{"id": i, "data": t.data} for i, t in zip(ids, scene.textures)]})
        self.send({"type": "shading", "version": sv, "shading": ShadingPayload.of(scene, ids)})
        return sv

    # -------------------------------------------------------------- tuning
    def set_timing(self, enabled: bool) -> None:
        call("mcrt_set_timing", self._h, int(bool(enabled)))

    def set_capacity(self, paths: int) -> None:
        call("mcrt_set_capacity", self._h, int(paths))

    def set_traversal(self, block: int, stack: int) -> None:
        """Traversal kernels by threads per block and short-stack depth (_lib.traversal_variants())."""
        call("mcrt_set_traversal", self._h, int(block), int(stack))

    def set_step_limit(self, steps: int) -> None:
        """Test and debugging hook: node visits plus leaves one BVH query may take (0: the
        default, 2N + 64 for N triangles); a query that runs out fails its call."""
        call("mcrt_set_step_limit", self._h, int(steps))

    def stats(self) -> Dict[str, Any]:
        s = mcrt_stats()
        call("mcrt_get_stats", self._h, C.byref(s))
        return s.as_dict()

    def reset_stats(self) -> None:
        call("mcrt_reset_stats", self._h)


_default: Dict[int, GpuExecutor] = {}
_default_lock = threading.Lock()


def default_executor(device: int = 0) -> GpuExecutor:
    """A process-wide executor per device, created on first use."""
    with _default_lock:
        ex = _default.get(device)
        if ex is None or ex._disposed:
            ex = GpuExecutor(device)
            _default[device] = ex
        return ex
