"""RaytracingRenderer without a canvas: the reference's WebGLRenderer look-alike
(src/RaytracingRenderer.ts:58-321) drawing into an RGBA8 buffer in host
memory, over GPU executors.

The parts of the interface applications use stay: set_size / get_size,
set_pixel_ratio, set_clear_color, tone_mapping, tone_mapping_exposure,
output_color_space, samples, max_bounces, shadows, global_illumination,
preview_block, fit_aspect, filter, seed, render (starts or restarts a
progressive render and returns at once; calls made before the render starts
are merged, as requestAnimationFrame merges them), render_async, when_done,
stop, progress, on_progress, clear, copy_settings_from and dispose.
`image` replaces the canvas: width * height * 4 bytes, top row first,
straight alpha, refreshed with every frame. Renders run on a background
thread instead of the browser's event loop; a failure is reported through
progress.error, as the reference does (src/RaytracingRenderer.ts:289-304).
"""
from __future__ import annotations

import math
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, replace
from typing import Any, Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import scene as S
from .executors import GpuExecutor
from .progressive import ProgressiveFrame, ProgressiveOptions, ProgressiveRenderer
from .raytrace import trace_settings


@dataclass
class RaytracingProgress:
    """RaytracingProgress, src/RaytracingRenderer.ts:33-46."""

    samples: int = 0
    max_samples: int = 0
    done: bool = True
    stopped: bool = False
    elapsed: float = 0.0  # ms since the render started
    error: Optional[str] = None


def _srgb_decode(c: float) -> float:
    return c / 12.92 if c < 0.04045 else math.pow((c + 0.055) / 1.055, 2.4)


class RaytracingRenderer:
    """Headless RaytracingRenderer on GPU executors (one per device in `devices`)."""

    def __init__(self, width: int = 300, height: int = 150, samples: int = 64, max_bounces: int = 4,
                 shadows: str = "all", global_illumination: bool = False, preview_block: int = 4,
                 fit_aspect: bool = False, filter: Optional[Callable[[Any], bool]] = None, tile_size: int = 64,
                 frame_interval: float = 100.0, seed: float = 0, tone_mapping: Optional[int] = None,
                 tone_mapping_exposure: Optional[float] = None, output_color_space: Optional[str] = None,
                 clear_color: Optional[Sequence[float]] = None, clear_alpha: Optional[float] = None,
                 devices: Sequence[int] = (0,), executors: Optional[Sequence[GpuExecutor]] = None):
        self.tone_mapping = S.NoToneMapping if tone_mapping is None else tone_mapping
        self.tone_mapping_exposure = 1.0 if tone_mapping_exposure is None else tone_mapping_exposure
        self.output_color_space = S.SRGBColorSpace if output_color_space is None else output_color_space
        self.samples = samples
        self.max_bounces = max_bounces
        self.shadows = shadows
        self.global_illumination = global_illumination
        self.preview_block = preview_block
        self.fit_aspect = fit_aspect
        self.filter = filter
        self._tile_size = tile_size
        self._frame_interval = frame_interval
        self._seed = seed
        self._clear_color: Tuple[float, float, float] = tuple(clear_color) if clear_color else (0.0, 0.0, 0.0)
        self._clear_alpha = 0.0 if clear_alpha is None else clear_alpha
        self._pixel_ratio = 1.0
        self._css_width, self._css_height = width, height
        self.width, self.height = int(width), int(height)
        self.image = np.zeros(self.width * self.height * 4, np.uint8)
        self._listeners: List[Callable[[RaytracingProgress], None]] = []
        self._last = RaytracingProgress()
        self._start_time = 0.0
        self._disposed = False
        self._pending: Optional[Tuple[Any, Any]] = None
        self._scheduled = False
        self._state = threading.Lock()
        self._current: "Future[bool]" = Future()
        self._current.set_result(True)
        self._runner_lock = threading.Lock()
        exs = list(executors) if executors is not None else [GpuExecutor(d) for d in devices]
        self._progressive = ProgressiveRenderer(exs)

    # ------------------------------------------------------------ settings
    def copy_settings_from(self, renderer: Any) -> "RaytracingRenderer":
        """copySettingsFrom: tone mapping, exposure, colour space, clear colour and alpha, pixel ratio."""
        for name in ("tone_mapping", "tone_mapping_exposure", "output_color_space"):
            if getattr(renderer, name, None) is not None:
                setattr(self, name, getattr(renderer, name))
        if hasattr(renderer, "get_clear_color"):
            c = renderer.get_clear_color()
            self._clear_color = (float(c[0]), float(c[1]), float(c[2]))
        if hasattr(renderer, "get_clear_alpha"):
            self._clear_alpha = float(renderer.get_clear_alpha())
        if hasattr(renderer, "get_pixel_ratio"):
            self.set_pixel_ratio(renderer.get_pixel_ratio())
        return self

    def set_pixel_ratio(self, value: float) -> None:
        self._pixel_ratio = float(value)
        self.set_size(self._css_width, self._css_height)

    def get_pixel_ratio(self) -> float:
        return self._pixel_ratio

    def set_size(self, width: float, height: float, update_style: bool = True) -> None:
        """The image is width x pixel ratio by height x pixel ratio pixels."""
        self._css_width, self._css_height = width, height
        self.width = max(0, int(math.floor(width * self._pixel_ratio)))
        self.height = max(0, int(math.floor(height * self._pixel_ratio)))
        self.image = np.zeros(self.width * self.height * 4, np.uint8)

    def get_size(self) -> Tuple[float, float]:
        return self._css_width, self._css_height

    def set_clear_color(self, color: Any, alpha: Optional[float] = None) -> None:
        """A hex colour is sRGB (stored linear); a sequence or an object with r, g, b is linear."""
        if isinstance(color, (list, tuple)):
            self._clear_color = (float(color[0]), float(color[1]), float(color[2]))
        elif hasattr(color, "r"):
            self._clear_color = (float(color.r), float(color.g), float(color.b))
        elif isinstance(color, int):
            self._clear_color = (_srgb_decode(((color >> 16) & 255) / 255), _srgb_decode(((color >> 8) & 255) / 255),
                                 _srgb_decode((color & 255) / 255))
        if alpha is not None:
            self._clear_alpha = float(alpha)

    def get_clear_color(self) -> Tuple[float, float, float]:
        return self._clear_color

    def get_clear_alpha(self) -> float:
        return self._clear_alpha

    def set_clear_alpha(self, alpha: float) -> None:
        self._clear_alpha = float(alpha)

    # ------------------------------------------------------------- renders
    def render(self, scene: Any, camera: Any) -> None:
        """Starts, or restarts, a progressive render; returns at once. Calls made before the
        render thread picks the job up are merged into the last one."""
        if self._disposed:
            return
        with self._state:
            self._pending = (scene, camera)
            if self._scheduled:
                return
            self._scheduled = True
        self._progressive.stop()  # a running render ends now
        threading.Thread(target=self._start_pending, daemon=True).start()

    def _start_pending(self) -> None:
        with self._state:
            self._scheduled = False
            job, self._pending = self._pending, None
        if job is not None and not self._disposed:
            self._run(job[0], job[1])

    def render_async(self, scene: Any, camera: Any) -> "Future[bool]":
        """Renders on a background thread; the future resolves to True when all samples completed,
        False if restarted or stopped."""
        with self._state:
            self._pending = None
        self._progressive.stop()
        fut: "Future[bool]" = Future()
        self._current = fut
        threading.Thread(target=self._run, args=(scene, camera, fut), daemon=True).start()
        return fut

    def when_done(self) -> "Future[bool]":
        return self._current

    def stop(self) -> None:
        """Stops rendering; `image` keeps what has been drawn."""
        with self._state:
            self._pending = None
        self._progressive.stop()
        if not self._last.done and not self._last.stopped:
            self._report(replace(self._last, stopped=True, elapsed=self._elapsed()))

    @property
    def progress(self) -> RaytracingProgress:
        return self._last

    def on_progress(self, listener: Callable[[RaytracingProgress], None]) -> Callable[[], None]:
        """Calls the listener as the render progresses; returns a function that removes it."""
        self._listeners.append(listener)
        return lambda: self._listeners.remove(listener) if listener in self._listeners else None

    def clear(self) -> None:
        self.image[:] = 0

    def dispose(self) -> None:
        self._disposed = True
        self.stop()
        with self._runner_lock:
            self._progressive.dispose()
        self._listeners.clear()

    # ------------------------------------------------------------ internals
    def _elapsed(self) -> float:
        return (time.monotonic() - self._start_time) * 1000.0

    def _run(self, scene: Any, camera: Any, fut: Optional["Future[bool]"] = None) -> None:
        if fut is None:
            fut = Future()
            self._current = fut
        with self._runner_lock:  # one render at a time; a superseded one has been stopped
            if self._disposed:
                fut.set_result(False)
                return
            self._start_time = time.monotonic()
            max_samples = max(1, int(math.floor(self.samples)))
            self._report(RaytracingProgress(0, max_samples, False, False, 0.0))
            settings = trace_settings({"max_bounces": self.max_bounces, "shadows": self.shadows,
                                       "global_illumination": self.global_illumination,
                                       "tone_mapping": self.tone_mapping,
                                       "tone_mapping_exposure": self.tone_mapping_exposure,
                                       "clear_color": self._clear_color, "clear_alpha": self._clear_alpha,
                                       "seed": self._seed})
            colour = S.LinearSRGBColorSpace if self.output_color_space == S.LinearSRGBColorSpace else S.SRGBColorSpace
            options = ProgressiveOptions(self.width, self.height, settings, colour, self.samples, self.preview_block,
                                         self._tile_size, self.filter, self._frame_interval, self.fit_aspect)
            try:
                ok = self._progressive.render(scene, camera, options, self._draw)
            except Exception as error:  # reported, as the reference reports a failed render
                self._report(replace(self._last, done=False, stopped=True, error=str(error), elapsed=self._elapsed()))
                ok = False
            fut.set_result(ok)

    def _report(self, progress: RaytracingProgress) -> None:
        self._last = progress
        for listener in list(self._listeners):
            listener(progress)

    def _draw(self, frame: ProgressiveFrame) -> None:
        if frame.width != self.width or frame.height != self.height:
            return
        self.image[:] = frame.image
        self._report(RaytracingProgress(frame.samples, frame.max_samples, frame.done, False, self._elapsed()))
