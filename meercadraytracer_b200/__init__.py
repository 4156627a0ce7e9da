"""B200-native ray/path tracer with the API of VJigouline/MeerCADRaytracer's hot path.

The compiled scene (src/types.ts of the reference) lives in HBM; BVH build,
ray generation, traversal, shading, shadow rays, accumulation and RGBA8
encoding are hand-written sm_100a CUDA kernels behind a C-ABI library
(include/mcrt.h). This package is the host side: scene description and
compilation, the `raytrace` entry points and the GPU tile executor.
"""
from .types import (  # noqa: F401
    TRI_CAST_SHADOW,
    TRI_OPAQUE,
    TRI_RECEIVE_SHADOW,
    CompiledBackground,
    CompiledBvh,
    CompiledCamera,
    CompiledEnvironment,
    CompiledFog,
    CompiledGeometry,
    CompiledLight,
    CompiledMaterial,
    CompiledScene,
    CompiledTexture,
    Tile,
    TraceSettings,
)
from .raytrace import (  # noqa: F401
    RaytraceOptions,
    RaytraceResult,
    raytrace,
    raytrace_compiled,
    trace_settings,
)

__version__ = "0.1.0"
