"""Headless entry points: `raytrace` and `raytrace_compiled` (src/raytrace.ts).

Both run on the GPU through the C-ABI library (`_lib.py`): the compiled scene
is uploaded to HBM once per geometry / shading version and every sample,
accumulation and the RGBA8 encode happen on the device. There is no CPU path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Callable, Optional, Tuple

import numpy as np

from .types import CompiledCamera, CompiledScene, TraceSettings

SRGB_COLOR_SPACE = "srgb"
LINEAR_SRGB_COLOR_SPACE = "srgb-linear"


@dataclass
class RaytraceOptions:
    """RaytraceOptions, src/raytrace.ts:9-35 (None means the reference's default)."""

    samples: Optional[float] = None
    max_bounces: Optional[float] = None
    shadows: Optional[str] = None
    global_illumination: Optional[bool] = None
    tone_mapping: Optional[int] = None
    tone_mapping_exposure: Optional[float] = None
    output_color_space: Optional[str] = None
    clear_color: Optional[Tuple[float, float, float]] = None
    clear_alpha: Optional[float] = None
    filter: Optional[Callable[[Any], bool]] = None
    seed: Optional[float] = None


@dataclass
class RaytraceResult:
    """RaytraceResult, src/raytrace.ts:37-42: RGBA8, top row first, straight alpha."""

    width: int
    height: int
    data: np.ndarray = field(repr=False)


def as_options(options: Any = None, **kw: Any) -> RaytraceOptions:
    if options is None:
        options = RaytraceOptions()
    elif isinstance(options, dict):
        options = RaytraceOptions(**options)
    for k, v in kw.items():
        setattr(options, k, v)
    return options


def trace_settings(options: Any = None) -> TraceSettings:
    """traceSettings, src/raytrace.ts:45-56: fills in the defaults."""
    o = as_options(options)
    max_bounces = 4 if o.max_bounces is None else o.max_bounces
    return TraceSettings(
        max_bounces=max(0, int(math.floor(max_bounces))),
        shadows=o.shadows if o.shadows is not None else "all",
        global_illumination=bool(o.global_illumination) if o.global_illumination is not None else False,
        tone_mapping=o.tone_mapping if o.tone_mapping is not None else 0,
        tone_mapping_exposure=o.tone_mapping_exposure if o.tone_mapping_exposure is not None else 1.0,
        clear_color=tuple(o.clear_color) if o.clear_color is not None else (0.0, 0.0, 0.0),
        clear_alpha=o.clear_alpha if o.clear_alpha is not None else 0.0,
        seed=o.seed if o.seed is not None else 0,
    )


def sample_count(options: Any = None) -> int:
    """`Math.max(1, Math.floor(options.samples ?? 16))`, src/raytrace.ts:73."""
    o = as_options(options)
    return max(1, int(math.floor(16 if o.samples is None else o.samples)))


def output_srgb(options: Any = None) -> bool:
    """src/raytrace.ts:77: sRGB unless the output colour space is linear."""
    o = as_options(options)
    return (o.output_color_space or SRGB_COLOR_SPACE) != LINEAR_SRGB_COLOR_SPACE


def raytrace_compiled(scene: CompiledScene, camera: CompiledCamera, width: int, height: int,
                      options: Any = None, executor: Any = None) -> RaytraceResult:
    """raytraceCompiled, src/raytrace.ts:69-82, on the GPU.

    `executor` is a GpuExecutor to reuse (its resident scene is replaced only if
    `scene` differs from the one it holds); by default a shared one on device 0.
    """
    from .executors import default_executor

    ex = executor or default_executor()
    data = ex.raytrace(scene, camera, width, height, trace_settings(options), sample_count(options),
                       output_srgb(options))
    return RaytraceResult(width, height, data)


def raytrace(scene: Any, camera: Any, width: int, height: int, options: Any = None,
             executor: Any = None) -> RaytraceResult:
    """raytrace, src/raytrace.ts:63-66: compile the scene description, then trace it."""
    from .compile import compile_camera, compile_scene

    o = as_options(options)
    compiled = compile_scene(scene, o.filter)
    return raytrace_compiled(compiled, compile_camera(camera), width, height, o, executor)
