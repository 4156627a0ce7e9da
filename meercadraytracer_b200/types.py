"""Plain-data form of a compiled scene: the reference's data contract.

Mirrors src/types.ts of the reference (VJigouline/MeerCADRaytracer) field for
field, in snake_case. Typed arrays are numpy arrays of the same element types
and strides (float32 triangles with 9 floats each, int32 BVH nodes with 3 ints
each, and so on), so a compiled scene carries over unchanged; JavaScript
numbers are Python floats (doubles).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

RGB = Tuple[float, float, float]

# Triangle flags, src/types.ts:133-135.
TRI_OPAQUE = 1
TRI_CAST_SHADOW = 2
TRI_RECEIVE_SHADOW = 4

# CompiledMaterial.model, src/types.ts:41.
MATERIAL_MODELS = ("physical", "phong", "lambert", "toon", "basic")
# CompiledLight.type, src/types.ts:91-113.
LIGHT_TYPES = ("ambient", "hemisphere", "directional", "point", "spot")
# CompiledBackground.kind, src/types.ts:123-127.
BACKGROUND_KINDS = ("clear", "color", "screen", "environment")
# TraceSettings.shadows, src/types.ts:195.
SHADOW_MODES = ("all", "castShadow", "none")


@dataclass
class CompiledTexture:
    """src/types.ts:8-21. `data` is uint8 or float32 RGBA, first row first."""

    width: int
    height: int
    data: np.ndarray
    srgb: bool = False
    flip_y: bool = False
    wrap_s: int = 1001
    wrap_t: int = 1001
    matrix: Tuple[float, ...] = (1, 0, 0, 0, 1, 0, 0, 0, 1)


@dataclass
class CompiledEnvironment:
    """src/types.ts:23-39: kind 'cube' (faces, flip_x) or 'equirect' (texture)."""

    kind: str
    rotation: Tuple[float, ...] = (1, 0, 0, 0, 1, 0, 0, 0, 1)
    intensity: float = 1.0
    faces: Tuple[int, ...] = (-1, -1, -1, -1, -1, -1)
    flip_x: bool = True
    texture: int = -1


@dataclass
class CompiledMaterial:
    """src/types.ts:43-89, with the defaults compileMaterial gives (src/compile.ts:111-146)."""

    model: str = "physical"
    side: int = 0
    color: RGB = (1.0, 1.0, 1.0)
    opacity: float = 1.0
    transparent: bool = False
    alpha_test: float = 0.0
    vertex_colors: bool = False
    flat_shading: bool = False
    tone_mapped: bool = True
    map: int = -1
    alpha_map: int = -1
    emissive_map: int = -1
    normal_map: int = -1
    ao_map: int = -1
    roughness_map: int = -1
    metalness_map: int = -1
    emissive: RGB = (0.0, 0.0, 0.0)
    normal_scale: Tuple[float, float] = (1.0, 1.0)
    ao_map_intensity: float = 1.0
    roughness: float = 1.0
    metalness: float = 0.0
    physical: bool = False
    ior: float = 1.5
    specular_intensity: float = 1.0
    specular_color: RGB = (1.0, 1.0, 1.0)
    transmission: float = 0.0
    thickness: float = 0.0
    attenuation: RGB = (0.0, 0.0, 0.0)
    shininess: float = 30.0
    specular: RGB = (0.0666, 0.0666, 0.0666)
    env_map: int = -1
    env_map_intensity: float = 1.0
    reflectivity: float = 1.0
    combine: int = 0


@dataclass
class CompiledLight:
    """src/types.ts:91-113. Fields a light type does not have stay at their defaults."""

    type: str
    color: RGB = (1.0, 1.0, 1.0)
    ground_color: RGB = (0.0, 0.0, 0.0)
    direction: RGB = (0.0, 0.0, 1.0)
    position: RGB = (0.0, 0.0, 0.0)
    distance: float = 0.0
    decay: float = 2.0
    cone_cos: float = 0.0
    penumbra_cos: float = 0.0
    cast_shadow: bool = False


@dataclass
class CompiledFog:
    """src/types.ts:115-121."""

    kind: str
    color: RGB = (1.0, 1.0, 1.0)
    near: float = 0.0
    far: float = 0.0
    density: float = 0.0


@dataclass
class CompiledBackground:
    """src/types.ts:123-127."""

    kind: str = "clear"
    color: RGB = (0.0, 0.0, 0.0)
    texture: int = -1
    environment: int = -1
    intensity: float = 1.0


@dataclass
class CompiledBvh:
    """src/types.ts:158-167: bounds float32[6 * node_count], nodes int32[3 * node_count]."""

    bounds: np.ndarray
    nodes: np.ndarray
    node_count: int


@dataclass
class CompiledGeometry:
    """src/types.ts:137-156. Per-triangle arrays are in BVH order."""

    triangle_count: int
    triangles: np.ndarray
    normals: np.ndarray
    uvs: np.ndarray
    tangents: np.ndarray
    colors: np.ndarray
    materials: np.ndarray
    flags: np.ndarray
    sides: np.ndarray
    bvh: CompiledBvh
    epsilon: float
    # Original (pre-BVH) index of each triangle: the `order` buildBvh returns.
    # Not part of the reference's message; kept for mapping hits back to input triangles.
    order: Optional[np.ndarray] = None


@dataclass
class CompiledScene:
    """src/types.ts:169-179."""

    geometry: CompiledGeometry
    materials: List[CompiledMaterial] = field(default_factory=list)
    textures: List[CompiledTexture] = field(default_factory=list)
    environments: List[CompiledEnvironment] = field(default_factory=list)
    lights: List[CompiledLight] = field(default_factory=list)
    background: CompiledBackground = field(default_factory=CompiledBackground)
    environment: int = -1
    fog: Optional[CompiledFog] = None


@dataclass
class CompiledCamera:
    """src/types.ts:181-190: column-major matrices."""

    projection_inverse: Tuple[float, ...]
    world: Tuple[float, ...]
    orthographic: bool
    forward: RGB
    position: RGB


@dataclass
class TraceSettings:
    """src/types.ts:193-204."""

    max_bounces: int = 4
    shadows: str = "all"
    global_illumination: bool = False
    tone_mapping: int = 0
    tone_mapping_exposure: float = 1.0
    clear_color: RGB = (0.0, 0.0, 0.0)
    clear_alpha: float = 0.0
    seed: float = 0


@dataclass
class Tile:
    """src/types.ts:206-211."""

    x: int
    y: int
    width: int
    height: int


def empty_geometry() -> CompiledGeometry:
    """A geometry with no triangles, as compileGeometry returns for an empty scene."""
    return CompiledGeometry(
        triangle_count=0,
        triangles=np.zeros(0, np.float32),
        normals=np.zeros(0, np.float32),
        uvs=np.zeros(0, np.float32),
        tangents=np.zeros(0, np.float32),
        colors=np.zeros(0, np.float32),
        materials=np.zeros(0, np.uint32),
        flags=np.zeros(0, np.uint8),
        sides=np.zeros(0, np.uint8),
        bvh=CompiledBvh(np.zeros(0, np.float32), np.zeros(0, np.int32), 0),
        epsilon=1e-7,
        order=np.zeros(0, np.uint32),
    )
