"""Progressive rendering with the accumulation on the GPU: the reference's
SceneSync, makeTiles and ProgressiveRenderer (src/progressive.ts:53-282).

The reference's ProgressiveRenderer hands tiles (one sample per tile per pass)
to tile executors and keeps the Float32 running sum and the RGBA8 image on the
host (writeTile, src/progressive.ts:288-313). Here the executors are GPUs and
the whole image is one tile: a block preview, then the passes, accumulate and
encode on the device (the batch engine of include/mcrt.h, mcrt_batch_*), and
the host receives RGBA8 frames. Frames, samples, restarts and results keep the
reference's meaning:

  * `render` reports ProgressiveFrame updates at most every frame_interval ms
    (the last one always) and returns True when every pixel has `samples`
    samples, False when stopped or superseded first;
  * starting a render or calling stop() ends the one in progress (generation
    counter, src/progressive.ts:178-188);
  * SceneSync recompiles geometry only when the geometry key changes, shading
    only when its payload changes, and sends each executor texture pixels
    once (src/progressive.ts:80-157).

There is no CPU fallback (the reference falls back to tracing in the page when
every worker fails, src/progressive.ts:240-255): a GPU failure raises.
"""
from __future__ import annotations

import math
import threading
import time
import weakref
from dataclasses import dataclass, fields, is_dataclass
from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import scene as S
from .batch import EVENT_DONE, EVENT_PREVIEW, EVENT_PROGRESS, BatchRenderer
from .compile import GeometryBuilder, SceneShading, compile_camera, compile_geometry, compile_shading
from .executors import GpuExecutor, ShadingPayload
from .types import CompiledGeometry, Tile, TraceSettings


@dataclass
class ProgressiveFrame:
    """ProgressiveFrame, src/progressive.ts:12-21."""

    image: np.ndarray  # RGBA8, top row first, straight alpha
    width: int
    height: int
    samples: int  # samples every pixel has; 0 while only the preview shows
    max_samples: int
    done: bool


@dataclass
class ProgressiveOptions:
    """ProgressiveOptions, src/progressive.ts:23-38."""

    width: int
    height: int
    settings: TraceSettings
    output_color_space: str = S.SRGBColorSpace
    samples: int = 64
    preview_block: int = 4
    tile_size: int = 64  # kept for the interface: the GPU renders the image as one tile
    filter: Optional[Callable[[Any], bool]] = None
    frame_interval: float = 100.0  # ms
    fit_aspect: bool = False


# ---------------------------------------------------------------- scene sync
_texture_ids: Dict[int, Tuple[Any, int]] = {}
_next_texture_id = [1]
_texture_lock = threading.Lock()


def texture_id(data: Any) -> int:
    """textureId, src/progressive.ts:40-49: one id per pixel array, for as long as it lives."""
    with _texture_lock:
        entry = _texture_ids.get(id(data))
        if entry is not None and entry[0]() is data:
            return entry[1]
        tid = _next_texture_id[0]
        _next_texture_id[0] += 1
        try:
            ref = weakref.ref(data)
        except TypeError:  # objects without weak references are kept alive instead
            ref = (lambda d: (lambda: d))(data)
        _texture_ids[id(data)] = (ref, tid)
        return tid


def geometry_key(meshes: Sequence[Any]) -> str:
    """geometryKey, src/progressive.ts:53-73: changes whenever a mesh's triangles,
    transform, shadow flags or the triangle-relevant parts of its materials would.
    BufferGeometry.version stands for three.js's attribute versions (bump it after
    editing arrays in place)."""
    parts: List[str] = []
    for mesh in meshes:
        g = mesh.geometry
        world = ",".join(repr(float(v)) for v in np.asarray(mesh.matrix_world).reshape(-1))
        parts.append(f"{id(mesh)}:{id(g)}:{getattr(g, 'version', 0)}:{getattr(g, 'draw_start', 0)}:"
                     f"{getattr(g, 'draw_count', 0)}:{len(getattr(g, 'groups', []) or [])}:"
                     f"{int(bool(mesh.cast_shadow))}{int(bool(mesh.receive_shadow))}:{world}")
        if isinstance(mesh, S.InstancedMesh):
            parts.append(f"i{mesh.count}:{getattr(mesh, 'instance_version', 0)}")
        for m in (mesh.material if isinstance(mesh.material, (list, tuple)) else [mesh.material]):
            if m is None:
                continue
            parts.append(f"{id(m)}:{m.side}:{int(bool(m.transparent))}:{int(m.alpha_test > 0)}:"
                         f"{int(getattr(m, 'transmission', 0) > 0)}:{int(bool(m.wireframe))}:{int(bool(m.visible))}:"
                         f"{int(bool(m.vertex_colors))}:{int(bool(m.flat_shading))}")
    return "|".join(parts)


def _plain(v: Any) -> Any:
    """A comparable form of shading data (JSON.stringify's role in SceneSync.update)."""
    if is_dataclass(v):
        return (type(v).__name__,) + tuple((f.name, _plain(getattr(v, f.name))) for f in fields(v))
    if isinstance(v, (list, tuple)):
        return tuple(_plain(x) for x in v)
    if isinstance(v, np.ndarray):
        return ("ndarray", v.dtype.str, v.shape, v.tobytes())
    if isinstance(v, float) and math.isnan(v):
        return "nan"
    return v


class SceneSync:
    """SceneSync, src/progressive.ts:80-157: compiled scene state and what each
    executor has been sent."""

    def __init__(self, builder: Optional[GeometryBuilder] = None):
        self.geometry: Optional[CompiledGeometry] = None
        self.geometry_version = 0
        self.shading_version = 0
        self._builder = builder
        self._shading: Optional[ShadingPayload] = None
        self._textures: list = []
        self._texture_ids: List[int] = []
        self._geometry_key = ""
        self._shading_key: Any = None
        self._sent: Dict[int, Tuple[Any, Dict[str, int]]] = {}

    def update(self, scene: S.Scene, camera: S.Camera, filter: Optional[Callable[[Any], bool]] = None,
               builder: Optional[GeometryBuilder] = None) -> None:
        """Recompiles what changed since the last update."""
        shading, meshes = compile_shading(scene, filter)
        key = geometry_key(meshes)
        indices = {id(m): i for i, m in enumerate(shading.material_objects)}
        if self.geometry is None or key != self._geometry_key:
            self.geometry = compile_geometry(meshes, lambda m: indices.get(id(m), 0), builder or self._builder)
            self._geometry_key = key
            self.geometry_version += 1
        payload = self._payload(shading)
        shading_key = _plain((payload.materials, [(t.width, t.height, t.srgb, t.flip_y, t.wrap_s, t.wrap_t,
                                                   tuple(t.matrix)) for t in payload.textures], payload.texture_ids,
                              payload.environments, payload.lights, payload.background, payload.environment,
                              payload.fog))
        if shading_key != self._shading_key:
            self._shading = payload
            self._shading_key = shading_key
            self._textures = shading.textures
            self.shading_version += 1

    def _payload(self, shading: SceneShading) -> ShadingPayload:
        # Ids follow the source texture's pixel array (the compiled copy is a new view each time).
        self._texture_ids = [texture_id(getattr(k, "data", k)) for k in shading.texture_keys]
        return ShadingPayload(shading.materials, shading.textures, list(self._texture_ids), shading.environments,
                              shading.lights, shading.background, shading.environment, shading.fog)

    def sync(self, executor: GpuExecutor) -> None:
        """Sends an executor whatever it is missing of the current scene."""
        entry = self._sent.get(id(executor))
        if entry is None or entry[0] is not executor:
            entry = (executor, {"geometry": 0, "shading": 0})
            self._sent[id(executor)] = entry
        state = entry[1]
        if state["geometry"] != self.geometry_version and self.geometry is not None:
            executor.send({"type": "geometry", "version": self.geometry_version, "geometry": self.geometry})
            state["geometry"] = self.geometry_version
        if state["shading"] != self.shading_version and self._shading is not None:
            items = []
            for t, tid in zip(self._textures, self._texture_ids):
                if tid not in executor.textures:
                    items.append({"id": tid, "data": t.data})
                    executor.textures.add(tid)
            if items:
                executor.send({"type": "textures", "items": items})
            executor.send({"type": "shading", "version": self.shading_version, "shading": self._shading})
            state["shading"] = self.shading_version

    def forget(self, executor: GpuExecutor) -> None:
        self._sent.pop(id(executor), None)


def make_tiles(width: int, height: int, size: int) -> List[Tile]:
    """makeTiles, src/progressive.ts:160-170: tiles ordered from the centre outwards
    (a stable sort by the distance of the tile centre to the image centre)."""
    tiles = [Tile(x, y, min(size, width - x), min(size, height - y))
             for y in range(0, height, size) for x in range(0, width, size)]
    cx, cy = width / 2, height / 2
    return sorted(tiles, key=lambda t: math.hypot(t.x + t.width / 2 - cx, t.y + t.height / 2 - cy))


# ------------------------------------------------------- progressive renders
class ProgressiveRenderer:
    """ProgressiveRenderer, src/progressive.ts:177-282, on GPU executors.

    One render runs at a time; its block preview and passes go through a batch
    engine on the first executor's device, so the image accumulates in HBM and
    only RGBA8 frames come back. `capacity` is the engine's path pool and
    `memory_budget` the device memory for the running image's buffers."""

    def __init__(self, executors: Sequence[GpuExecutor], capacity: int = 1 << 22, memory_budget: int = 1 << 30,
                 builder: Optional[GeometryBuilder] = None):
        self.executors: List[GpuExecutor] = list(executors)
        self._generation = 0
        self._lock = threading.Lock()
        self._capacity = capacity
        self._budget = memory_budget
        self._batch: Optional[BatchRenderer] = None
        self.sync = SceneSync(builder if builder is not None else self._gpu_builder)

    def _gpu_builder(self, sink: Any) -> CompiledGeometry:
        if not self.executors:
            raise RuntimeError("the renderer has no executors")
        return self.executors[0].compile_sink(sink)

    def stop(self) -> None:
        """Stops the current render; its render() returns False."""
        self._generation += 1

    def _engine(self) -> BatchRenderer:
        if self._batch is None:
            self._batch = BatchRenderer(self.executors[0].device, self._capacity, self._budget)
        return self._batch

    def render(self, scene: S.Scene, camera: S.Camera, options: ProgressiveOptions,
               on_frame: Callable[[ProgressiveFrame], None]) -> bool:
        """Renders `scene` from `camera`, calling on_frame as the image improves. Returns True
        when every pixel has options.samples samples, False if stopped or superseded first."""
        self._generation += 1
        generation = self._generation
        width, height = int(options.width), int(options.height)
        if width <= 0 or height <= 0 or not self.executors:
            return False
        live = lambda: generation == self._generation  # noqa: E731
        with self._lock:
            if not live():
                return False
            self.sync.update(scene, camera, options.filter)
            cam = compile_camera(camera, width / height if options.fit_aspect else None)
            executor = self.executors[0]
            self.sync.sync(executor)
            srgb = options.output_color_space == S.SRGBColorSpace
            max_samples = max(1, int(math.floor(options.samples)))
            block = int(math.floor(options.preview_block)) if options.preview_block > 1 else 0
            engine = self._engine()
            rid = engine.submit_to(executor, (self.sync.geometry_version, self.sync.shading_version), cam,
                                   options.settings, width, height, max_samples, block, srgb, progress=True)
            image = np.zeros(width * height * 4, np.uint8)
            samples = 0
            last_frame = [0.0]

            def emit(force: bool, done: bool) -> None:
                now = time.monotonic() * 1000.0
                if not force and now - last_frame[0] < options.frame_interval:
                    return
                last_frame[0] = now
                on_frame(ProgressiveFrame(image, width, height, samples, max_samples, done))

            try:
                while True:
                    if not live():
                        engine.cancel(rid)
                        self._drain(engine)
                        return False
                    events, idle = engine.step()
                    for eid, kind, n in events:
                        if eid != rid or not live():
                            continue
                        if kind == EVENT_PREVIEW and samples == 0:
                            image[:] = engine.preview(rid)
                            emit(False, False)
                        elif kind == EVENT_PROGRESS:
                            samples = max(samples, int(n))
                            image[:] = engine.progress(rid)
                            emit(False, False)
                        elif kind == EVENT_DONE:
                            samples = max_samples
                            image[:] = engine.result(rid)
                            if not live():
                                return False
                            emit(True, True)
                            return True
                    if idle:
                        return False
            finally:
                engine.forget(rid)

    @staticmethod
    def _drain(engine: BatchRenderer) -> None:
        """Runs the engine until the cancelled work in flight has returned its buffers."""
        for _ in range(1 << 20):
            _, idle = engine.step()
            if idle:
                return

    def dispose(self) -> None:
        self.stop()
        with self._lock:
            if self._batch is not None:
                self._batch.dispose()
                self._batch = None
            for ex in self.executors:
                ex.dispose()
            self.executors = []
