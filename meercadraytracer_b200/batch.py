"""Batched and served rendering over libmcrt's batch engine (mcrt_batch_* in
include/mcrt.h).

The reference renders one progressive image at a time (ProgressiveRenderer,
src/progressive.ts:177-282): a block preview, then one sample per pass,
accumulated. BatchRenderer runs many such renders (different scenes,
cameras, sizes and sample counts) together in one wavefront on one GPU:

    renderer = BatchRenderer(capacity=1 << 22, memory_budget=4 << 30)
    images = renderer.render([RenderRequest(scene, camera, 512, 512, settings, 16), ...])

or, as a serving loop, submit() / step() / cancel() with preview, progress
and done events. Each request's final image equals raytrace_compiled's for the same
inputs, alone or in any mix. Scenes stay resident: each distinct
CompiledScene is uploaded once, to its own GpuExecutor.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import abi
from ._lib import call, load
from .executors import GpuExecutor
from .types import CompiledCamera, CompiledScene, TraceSettings

EVENT_PREVIEW = 1
EVENT_DONE = 2
EVENT_PROGRESS = 3


@dataclass
class RenderRequest:
    """One render: raytraceCompiled's arguments plus a block preview size."""

    scene: CompiledScene
    camera: CompiledCamera
    width: int
    height: int
    settings: TraceSettings
    samples: int = 16
    preview_block: int = 0  # > 1: ProgressiveOptions.previewBlock
    srgb: bool = True
    progress: bool = False  # copy the image to the host after every completed pass (scheduled pass by pass)


class BatchRenderer:
    """A batch engine on one device with the scenes it has seen kept resident."""

    def __init__(self, device: int = 0, capacity: int = 1 << 22, memory_budget: int = 2 << 30,
                 use_graph: bool = True):
        load()
        handle = C.c_void_p()
        call("mcrt_batch_create", int(device), int(capacity), int(memory_budget), int(bool(use_graph)),
             C.byref(handle))
        self._h = handle
        self.device = device
        self.capacity = int(capacity)
        self._executors: Dict[int, Tuple[CompiledScene, GpuExecutor]] = {}
        self._buffers: Dict[int, Tuple[np.ndarray, Optional[np.ndarray], Optional[np.ndarray]]] = {}
        self._adopted: set = set()

    # ----------------------------------------------------------- scenes
    def executor(self, scene: CompiledScene) -> GpuExecutor:
        """The executor holding `scene` resident (created and loaded on first use)."""
        entry = self._executors.get(id(scene))
        if entry is None or entry[0] is not scene:
            ex = GpuExecutor(self.device)
            ex.load_scene(scene)
            entry = (scene, ex)
            self._executors[id(scene)] = entry
        return entry[1]

    def adopt(self, scene: CompiledScene, executor: GpuExecutor) -> None:
        """Uses `executor` (already holding `scene`) for requests on `scene`; the caller keeps
        ownership (dispose() leaves it alone)."""
        self._executors[id(scene)] = (scene, executor)
        self._adopted.add(id(executor))

    # ---------------------------------------------------------- requests
    @staticmethod
    def _c_fields(ex: GpuExecutor, versions: Tuple[int, int], camera: CompiledCamera, settings: TraceSettings,
                  width: int, height: int, samples: int, preview_block: int, srgb: bool, image: np.ndarray,
                  preview: Optional[np.ndarray], progress: Optional[np.ndarray]) -> abi.mcrt_request:
        c = abi.mcrt_request()
        c.scene = ex._h.value
        c.geometry_version, c.shading_version = int(versions[0]), int(versions[1])
        c.camera = abi.to_c_camera(camera)
        c.settings = abi.to_c_settings(settings)
        c.width, c.height = int(width), int(height)
        c.samples = int(samples)
        c.preview_block = int(preview_block)
        c.srgb = int(bool(srgb))
        none = C.cast(None, C.POINTER(C.c_uint8))
        c.image = abi.ptr(image, C.c_uint8)
        c.preview_image = abi.ptr(preview, C.c_uint8) if preview is not None else none
        c.progress_image = abi.ptr(progress, C.c_uint8) if progress is not None else none
        return c

    def _c_request(self, r: RenderRequest, image: np.ndarray, preview: Optional[np.ndarray],
                   progress: Optional[np.ndarray] = None) -> abi.mcrt_request:
        ex = self.executor(r.scene)
        versions = ex.load_scene(r.scene)
        return self._c_fields(ex, versions, r.camera, r.settings, r.width, r.height, r.samples, r.preview_block,
                              r.srgb, image, preview, progress)

    def _submit_c(self, c: abi.mcrt_request, buffers: Tuple[np.ndarray, Optional[np.ndarray], Optional[np.ndarray]]
                  ) -> int:
        rid = C.c_int64()
        call("mcrt_batch_submit", self._h, C.byref(c), C.byref(rid))
        self._buffers[rid.value] = buffers
        return rid.value

    def submit(self, r: RenderRequest) -> int:
        """Queues a request; returns its id. Its images are result(id) / preview(id) / progress(id)."""
        image = np.zeros(r.width * r.height * 4, np.uint8)
        preview = np.zeros(r.width * r.height * 4, np.uint8) if r.preview_block > 1 else None
        progress = np.zeros(r.width * r.height * 4, np.uint8) if r.progress else None
        return self._submit_c(self._c_request(r, image, preview, progress), (image, preview, progress))

    def submit_to(self, executor: GpuExecutor, versions: Tuple[int, int], camera: CompiledCamera,
                  settings: TraceSettings, width: int, height: int, samples: int, preview_block: int = 0,
                  srgb: bool = True, progress: bool = False) -> int:
        """As submit, for a scene that `executor` already holds under `versions` (geometry, shading),
        as SceneSync.sync leaves it."""
        image = np.zeros(width * height * 4, np.uint8)
        preview = np.zeros(width * height * 4, np.uint8) if preview_block > 1 else None
        prog = np.zeros(width * height * 4, np.uint8) if progress else None
        c = self._c_fields(executor, versions, camera, settings, width, height, samples, preview_block, srgb, image,
                           preview, prog)
        return self._submit_c(c, (image, preview, prog))

    def cancel(self, rid: int) -> None:
        call("mcrt_batch_cancel", self._h, int(rid))

    def step(self, max_events: int = 256) -> Tuple[List[Tuple[int, int, int]], bool]:
        """One scheduling step: ([(id, kind, samples)], idle)."""
        events = (abi.mcrt_batch_event * max(1, max_events))()
        n = C.c_int32()
        idle = C.c_int32()
        call("mcrt_batch_step", self._h, events, int(max_events), C.byref(n), C.byref(idle))
        return [(events[i].id, events[i].kind, events[i].samples) for i in range(n.value)], bool(idle.value)

    def result(self, rid: int) -> np.ndarray:
        return self._buffers[rid][0]

    def preview(self, rid: int) -> Optional[np.ndarray]:
        return self._buffers[rid][1]

    def progress(self, rid: int) -> Optional[np.ndarray]:
        """The image after the last completed pass (requests submitted with progress=True)."""
        return self._buffers[rid][2]

    def forget(self, rid: int) -> None:
        """Drops the host buffers of a finished or cancelled request."""
        self._buffers.pop(rid, None)

    def render(self, requests: Sequence[RenderRequest]) -> List[np.ndarray]:
        """Renders every request to completion in one batch (mcrt_batch_render)."""
        images = [np.zeros(r.width * r.height * 4, np.uint8) for r in requests]
        arr = (abi.mcrt_request * max(1, len(requests)))()
        for i, r in enumerate(requests):
            arr[i] = self._c_request(r, images[i], None)
        call("mcrt_batch_render", self._h, int(len(requests)), arr)
        return images

    def set_chunk(self, paths: int) -> None:
        call("mcrt_batch_set_chunk", self._h, int(paths))

    def set_traversal(self, block: int, stack: int) -> None:
        """Traversal kernels by threads per block and short-stack depth (_lib.traversal_variants())."""
        call("mcrt_batch_set_traversal", self._h, int(block), int(stack))

    def stats(self) -> Dict[str, float]:
        s = abi.mcrt_batch_stats()
        call("mcrt_batch_get_stats", self._h, C.byref(s))
        return {name: getattr(s, name) for name, _ in s._fields_ if name != "pad_"}

    def dispose(self) -> None:
        if self._h is not None:
            call("mcrt_batch_destroy", self._h)
            self._h = None
        for _, ex in self._executors.values():
            if id(ex) not in self._adopted:
                ex.dispose()
        self._executors.clear()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.dispose()
        except Exception:
            pass
