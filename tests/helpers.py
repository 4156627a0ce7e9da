"""Test helpers in the shape of the reference's tests/helpers.ts.

`render` traces with the oracle (CPU) or the CUDA path, with linear output and
1 sample unless asked, so values are easy to predict, as the reference does.
"""
from __future__ import annotations

import math
from typing import Any, Dict, Optional, Tuple

import numpy as np

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200.compile import compile_camera, compile_scene
from meercadraytracer_b200.raytrace import as_options, output_srgb, sample_count, trace_settings

# tests/helpers.ts:45 -- one 8-bit level.
ONE_LEVEL = 1 / 255 + 1e-6


def top_camera() -> S.OrthographicCamera:
    """Orthographic camera at z = 10 looking down -z at the square -1..1 (tests/helpers.ts:5-11)."""
    camera = S.OrthographicCamera(-1, 1, 1, -1, 0.1, 100)
    camera.position.set(0, 0, 10)
    camera.look_at(0, 0, 0)
    camera.update_matrix_world()
    return camera


def floor(material: S.Material, size: float = 4) -> S.Mesh:
    """A size x size plane in z = 0 facing +z (tests/helpers.ts:14-16)."""
    return S.Mesh(S.plane_geometry(size, size), material)


def overhead_light(intensity: float) -> S.DirectionalLight:
    """Directional light shining straight down -z (tests/helpers.ts:39-43)."""
    light = S.DirectionalLight(0xffffff, intensity)
    light.position.set(0, 0, 10)
    return light


def compile_with_oracle(scene: S.Scene, filter=None):
    from oracle import cpu

    return compile_scene(scene, filter, builder=cpu.compile_sink)


class Rendered:
    def __init__(self, data: np.ndarray, width: int, height: int):
        self.data = data
        self.width = width
        self.height = height

    def at(self, x: int, y: int) -> Tuple[float, float, float, float]:
        i = (y * self.width + x) * 4
        return tuple(float(self.data[i + c]) / 255 for c in range(4))  # type: ignore[return-value]


def raytrace_oracle(scene: S.Scene, camera: S.Camera, width: int, height: int, options: Any = None,
                    threads: int = 1) -> np.ndarray:
    """The reference's `raytrace`, run by the oracle."""
    from oracle import cpu

    o = as_options(options)
    compiled = compile_with_oracle(scene, o.filter)
    return cpu.raytrace_compiled(compiled, compile_camera(camera), width, height, trace_settings(o),
                                 sample_count(o), output_srgb(o), threads)


def render(scene: S.Scene, camera: S.Camera, options: Optional[Dict[str, Any]] = None, width: int = 16,
           height: int = 16, impl: str = "oracle") -> Rendered:
    """tests/helpers.ts:26-36: linear output and 1 sample unless asked."""
    opts: Dict[str, Any] = {"output_color_space": "srgb-linear", "samples": 1}
    opts.update(options or {})
    if impl == "oracle":
        data = raytrace_oracle(scene, camera, width, height, opts)
    else:
        from meercadraytracer_b200.raytrace import raytrace

        data = raytrace(scene, camera, width, height, opts).data
    return Rendered(data, width, height)


def centre(r: Rendered) -> Tuple[float, float, float, float]:
    return r.at(8, 8)
