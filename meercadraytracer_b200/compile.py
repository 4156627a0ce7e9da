"""Scene compilation: scene description -> CompiledScene, as src/compile.ts does.

The scene-graph walk, material, light, background and fog compilation
(src/compile.ts:29-306, 434-527) run on the host in Python, because their
input is the host-side object model. The per-triangle flatten (addMesh,
src/compile.ts:212-306) is vectorised with numpy into "sink" arrays. What
follows it -- BVH build, reorder into BVH order, tangents and epsilon
(src/compile.ts:327-432) -- is done by a geometry builder: the product's is the
GPU one, `GpuExecutor.compile_sink` (libmcrt's `mcrt_compile_geometry`).
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass
from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import scene as S
from .types import (
    TRI_CAST_SHADOW,
    TRI_OPAQUE,
    TRI_RECEIVE_SHADOW,
    CompiledBackground,
    CompiledCamera,
    CompiledEnvironment,
    CompiledFog,
    CompiledGeometry,
    CompiledLight,
    CompiledMaterial,
    CompiledScene,
    CompiledTexture,
)

_warned: set = set()


def warn_once(message: str) -> None:
    """warnOnce, src/compile.ts:29-34."""
    if message in _warned:
        return
    _warned.add(message)
    warnings.warn(f"meercad-raytracer: {message}")


def is_helper(obj: Any) -> bool:
    """isHelper, src/compile.ts:37-41."""
    return obj.type.endswith("Helper") or obj.user_data.get("raytrace") is False


def _normalize(v: Sequence[float]) -> Tuple[float, float, float]:
    """normalize, src/compile.ts:52-55."""
    length = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return (v[0] / length, v[1] / length, v[2] / length) if length > 0 else (0.0, 0.0, 1.0)


def collect_objects(scene: S.Scene, filter: Optional[Callable[[Any], bool]] = None) -> Tuple[list, list]:
    """collectObjects, src/compile.ts:64-80 (camera layers are not modelled)."""
    meshes: list = []
    lights: list = []

    def visit(obj: Any) -> None:
        if not obj.visible or is_helper(obj):
            return
        if filter is not None and not filter(obj):
            return
        if isinstance(obj, S.Light):
            lights.append(obj)
        elif isinstance(obj, S.Mesh):
            meshes.append(obj)
        for child in obj.children:
            visit(child)

    visit(scene)
    return meshes, lights


_IDENTITY3 = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)


def _texture_pixels(texture: Any, data: Any) -> np.ndarray:
    """readImage's decode of one RGBA image (src/textures.ts:60-110): 8-bit data
    kept, half floats widened, anything else as float32."""
    data = np.asarray(data)
    channels = data.size // max(1, texture.width * texture.height)
    if channels != 4:
        raise ValueError("only RGBA data textures are supported")
    if texture.type == S.HalfFloatType:
        data = data.astype(np.uint16).view(np.float16).astype(np.float32)
    elif data.dtype != np.uint8:
        data = data.astype(np.float32)
    return data.reshape(-1)


def _to_compiled(texture: Any, pixels: np.ndarray, flip_y: bool, matrix: Sequence[float]) -> CompiledTexture:
    """toCompiled, src/textures.ts:113-127."""
    srgb = pixels.dtype == np.uint8 and texture.color_space == S.SRGBColorSpace
    return CompiledTexture(texture.width, texture.height, pixels, bool(srgb), bool(flip_y), texture.wrap_s,
                           texture.wrap_t, tuple(matrix))


class _Face:
    """The source of one cube face in the texture table: its pixel array, which
    identifies the face when pixels are shipped to an executor."""

    def __init__(self, data: Any) -> None:
        self.data = data


class TextureTable:
    """TextureTable, src/textures.ts:134-198: each texture stored once."""

    def __init__(self) -> None:
        self.textures: List[CompiledTexture] = []
        self.environments: List[CompiledEnvironment] = []
        self.keys: List[Any] = []  # source object of each texture, for identity-based ids
        self._index: Dict[int, int] = {}
        self._environment_index: Dict[Tuple[Any, ...], int] = {}

    def add(self, texture: Optional[S.DataTexture]) -> int:
        """add, src/textures.ts:141-157: a material map or screen background; cube
        textures are environments only."""
        if texture is None or isinstance(texture, S.CubeTexture):
            return -1
        key = id(texture)
        if key in self._index:
            return self._index[key]
        index = len(self.textures)
        self.textures.append(_to_compiled(texture, _texture_pixels(texture, texture.data), bool(texture.flip_y),
                                          texture.matrix()))
        self.keys.append(texture)
        self._index[key] = index
        return index

    def add_environment(self, texture: Any, intensity: float, rotation: Any) -> int:
        """addEnvironment, src/textures.ts:164-197: cube textures (six faces, x
        mirrored unless a render target) and equirectangular textures, each
        (texture, version, intensity, rotation) compiled once."""
        if texture is None:
            return -1
        matrix = _euler_to_matrix_transposed(rotation)
        key = (id(texture), getattr(texture, "version", 0), float(intensity), tuple(matrix))
        if key in self._environment_index:
            return self._environment_index[key]
        environment: Optional[CompiledEnvironment] = None
        mapping = texture.mapping
        if isinstance(texture, S.CubeTexture) or mapping in (S.CubeReflectionMapping, S.CubeRefractionMapping):
            images = list(getattr(texture, "images", []))
            faces: List[int] = []
            if len(images) == 6:
                for image in images:
                    self.textures.append(_to_compiled(texture, _texture_pixels(texture, image), False, _IDENTITY3))
                    self.keys.append(_Face(image))
                    faces.append(len(self.textures) - 1)
            if len(faces) == 6:
                environment = CompiledEnvironment("cube", matrix, float(intensity), faces=tuple(faces),
                                                  flip_x=not getattr(texture, "is_render_target_texture", False))
            else:
                warn_once("a cube texture without six readable images is ignored")
        elif mapping in (S.EquirectangularReflectionMapping, S.EquirectangularRefractionMapping):
            index = self.add(texture)
            if index >= 0:
                environment = CompiledEnvironment("equirect", matrix, float(intensity), texture=index)
        else:
            warn_once(f"environment textures with mapping {mapping} are not supported and are ignored")
        index = -1
        if environment is not None:
            self.environments.append(environment)
            index = len(self.environments) - 1
        self._environment_index[key] = index
        return index


def _euler_to_matrix_transposed(euler: Any) -> Tuple[float, ...]:
    """eulerToMatrixTransposed, src/textures.ts:204-217 (XYZ order)."""
    if euler is None or (euler.x == 0 and euler.y == 0 and euler.z == 0):
        return (1, 0, 0, 0, 1, 0, 0, 0, 1)
    x, y, z = euler.x, euler.y, euler.z
    rx = np.array([[1, 0, 0], [0, math.cos(x), -math.sin(x)], [0, math.sin(x), math.cos(x)]])
    ry = np.array([[math.cos(y), 0, math.sin(y)], [0, 1, 0], [-math.sin(y), 0, math.cos(y)]])
    rz = np.array([[math.cos(z), -math.sin(z), 0], [math.sin(z), math.cos(z), 0], [0, 0, 1]])
    m = rx @ ry @ rz
    return tuple(float(v) for v in m.reshape(9))  # transpose, read column-major


def _volume_attenuation(m: Any) -> Tuple[float, float, float]:
    """volumeAttenuation, src/compile.ts:86-92."""
    distance = getattr(m, "attenuation_distance", math.inf)
    colour = getattr(m, "attenuation_color", None)
    if colour is None or not (distance > 0) or distance == math.inf:
        return (0.0, 0.0, 0.0)
    coef = lambda c: -math.log(min(max(c, 1e-6), 1)) / distance  # noqa: E731
    return (coef(colour.r), coef(colour.g), coef(colour.b))


def compile_material(m: S.Material, table: TextureTable) -> CompiledMaterial:
    """compileMaterial, src/compile.ts:94-147."""
    kind = m.kind
    model = {"standard": "physical", "physical": "physical", "phong": "phong", "lambert": "lambert",
             "toon": "toon", "basic": "basic"}.get(kind)
    if model is None:
        warn_once(f"{type(m).__name__} is not supported and is shaded as a Lambert material")
        model = "lambert"
    physical = kind == "physical"
    env_map = -1
    if m.env_map is not None:
        env_map = table.add_environment(m.env_map, m.env_map_intensity if m.env_map_intensity is not None else 1,
                                        getattr(m, "env_map_rotation", None))
    emissive = m.emissive.tuple(m.emissive_intensity) if m.emissive is not None else (0.0, 0.0, 0.0)
    return CompiledMaterial(
        model=model,
        side=m.side,
        color=m.color.tuple() if m.color is not None else (1.0, 1.0, 1.0),
        opacity=m.opacity,
        transparent=bool(m.transparent),
        alpha_test=m.alpha_test,
        vertex_colors=bool(m.vertex_colors),
        flat_shading=bool(m.flat_shading),
        tone_mapped=m.tone_mapped is not False,
        map=table.add(m.map),
        alpha_map=table.add(m.alpha_map),
        emissive_map=table.add(m.emissive_map),
        normal_map=table.add(m.normal_map),
        ao_map=table.add(m.ao_map),
        roughness_map=table.add(m.roughness_map),
        metalness_map=table.add(m.metalness_map),
        emissive=emissive,
        normal_scale=tuple(m.normal_scale),
        ao_map_intensity=m.ao_map_intensity,
        roughness=getattr(m, "roughness", 1.0),
        metalness=getattr(m, "metalness", 0.0),
        physical=physical,
        ior=getattr(m, "ior", 1.5),
        specular_intensity=getattr(m, "specular_intensity", 1.0),
        specular_color=m.specular_color.tuple() if physical else (1.0, 1.0, 1.0),
        transmission=getattr(m, "transmission", 0.0) if physical else 0.0,
        thickness=getattr(m, "thickness", 0.0) if physical else 0.0,
        attenuation=_volume_attenuation(m) if physical else (0.0, 0.0, 0.0),
        shininess=getattr(m, "shininess", 30.0),
        specular=m.specular.tuple() if getattr(m, "specular", None) is not None else (0.0666, 0.0666, 0.0666),
        env_map=env_map,
        env_map_intensity=m.env_map_intensity if m.env_map_intensity is not None else 1.0,
        reflectivity=m.reflectivity if m.reflectivity is not None else 1.0,
        combine=m.combine if m.combine is not None else 0,
    )


def compile_light(light: S.Light) -> Optional[CompiledLight]:
    """compileLight, src/compile.ts:149-177."""
    color = light.color.tuple(light.intensity)
    pos = tuple(float(v) for v in light.matrix_world[12:15])
    if type(light) is S.AmbientLight:
        return CompiledLight("ambient", color=color)
    if isinstance(light, S.HemisphereLight):
        return CompiledLight("hemisphere", color=color, ground_color=light.ground_color.tuple(light.intensity),
                             direction=_normalize(pos))
    if isinstance(light, (S.DirectionalLight, S.SpotLight)):
        target = light.target
        if target.parent is None:
            target.update_matrix_world()
        tpos = target.matrix_world[12:15]
        direction = _normalize((pos[0] - tpos[0], pos[1] - tpos[1], pos[2] - tpos[2]))
        if isinstance(light, S.DirectionalLight):
            return CompiledLight("directional", color=color, direction=direction, cast_shadow=light.cast_shadow)
        return CompiledLight("spot", color=color, position=pos, direction=direction, distance=light.distance,
                             decay=light.decay, cone_cos=math.cos(light.angle),
                             penumbra_cos=math.cos(light.angle * (1 - light.penumbra)),
                             cast_shadow=light.cast_shadow)
    if isinstance(light, S.PointLight):
        return CompiledLight("point", color=color, position=pos, distance=light.distance, decay=light.decay,
                             cast_shadow=light.cast_shadow)
    warn_once(f"{type(light).__name__} is not supported and is left out")
    return None


def compile_background(scene: S.Scene, table: TextureTable) -> CompiledBackground:
    """compileBackground, src/compile.ts:434-449."""
    bg = scene.background
    if bg is None:
        return CompiledBackground("clear")
    if isinstance(bg, S.Color):
        return CompiledBackground("color", color=bg.tuple())
    if isinstance(bg, (S.DataTexture, S.CubeTexture)):
        if isinstance(bg, S.CubeTexture) or bg.mapping in (301, 302, 303, 304):
            env = table.add_environment(bg, scene.background_intensity, scene.background_rotation)
            return CompiledBackground("environment", environment=env, intensity=scene.background_intensity) \
                if env >= 0 else CompiledBackground("clear")
        tex = table.add(bg)
        return CompiledBackground("screen", texture=tex, intensity=scene.background_intensity) \
            if tex >= 0 else CompiledBackground("clear")
    return CompiledBackground("clear")


def compile_fog(fog: Any) -> Optional[CompiledFog]:
    """compileFog, src/compile.ts:451-456."""
    if fog is None:
        return None
    if isinstance(fog, S.FogExp2):
        return CompiledFog("exp2", fog.color.tuple(), 0.0, 0.0, fog.density)
    return CompiledFog("linear", fog.color.tuple(), fog.near, fog.far, 0.0)


@dataclass
class SceneShading:
    """SceneShading, src/compile.ts:463-473."""

    materials: List[CompiledMaterial]
    textures: List[CompiledTexture]
    environments: List[CompiledEnvironment]
    lights: List[CompiledLight]
    background: CompiledBackground
    environment: int
    fog: Optional[CompiledFog]
    material_objects: List[Any]
    texture_keys: List[Any]


def compile_shading(scene: S.Scene, filter: Optional[Callable[[Any], bool]] = None) -> Tuple[SceneShading, list]:
    """compileShading, src/compile.ts:476-510."""
    scene.update_matrix_world()
    meshes, lights = collect_objects(scene, filter)
    table = TextureTable()
    material_objects: List[Any] = []
    materials: List[CompiledMaterial] = []
    seen: Dict[int, int] = {}
    for mesh in meshes:
        for m in (mesh.material if isinstance(mesh.material, (list, tuple)) else [mesh.material]):
            if m is None or id(m) in seen:
                continue
            seen[id(m)] = len(materials)
            material_objects.append(m)
            materials.append(compile_material(m, table))
    background = compile_background(scene, table)
    environment = table.add_environment(scene.environment, scene.environment_intensity,
                                        scene.environment_rotation) if scene.environment is not None else -1
    compiled_lights = [l for l in (compile_light(x) for x in lights) if l is not None]
    shading = SceneShading(materials, table.textures, table.environments, compiled_lights, background,
                           environment, compile_fog(scene.fog), material_objects, table.keys)
    return shading, meshes


# ---------------------------------------------------------------- the flatten
@dataclass
class TriangleSink:
    """Flattened world-space triangles, as compileGeometry's sink receives them
    (src/compile.ts:335-356): doubles before any float32 rounding."""

    p: np.ndarray  # (n, 9) float64 vertex positions
    n: np.ndarray  # (n, 9) float64 vertex normals
    uv: np.ndarray  # (n, 6) float64
    colors: np.ndarray  # (n, 12) float64
    has_color: np.ndarray  # (n,) uint8
    materials: np.ndarray  # (n,) uint32
    flags: np.ndarray  # (n,) uint8
    sides: np.ndarray  # (n,) uint8

    @property
    def count(self) -> int:
        return int(self.p.shape[0])


def _normal_matrix(m: np.ndarray) -> Tuple[np.ndarray, float]:
    """normalMatrix, src/compile.ts:192-205: cofactors / det, column-major, and det."""
    a, b, c, d, e, f, g, h, i = m[0], m[4], m[8], m[1], m[5], m[9], m[2], m[6], m[10]
    A, B, Cc = e * i - f * h, -(d * i - f * g), d * h - e * g
    det = a * A + b * B + c * Cc
    s = 1 / det if det != 0 else 0.0
    n = np.array([A * s, -(b * i - c * h) * s, (b * f - c * e) * s,
                  B * s, (a * i - c * g) * s, -(a * f - c * d) * s,
                  Cc * s, -(a * h - b * g) * s, (a * e - b * d) * s], np.float64)
    return n, det


def js_hypot_rows(v: np.ndarray) -> np.ndarray:
    """Math.hypot(x, y, z) of each row as V8 computes it: the values scaled by the
    largest magnitude, their squares summed with Kahan compensation, then
    sqrt(sum) * largest. Rows with an infinity give infinity, rows with a NaN NaN."""
    a = np.abs(v)
    mx = a.max(axis=1)
    safe = np.where(mx > 0, mx, 1.0)
    total = np.zeros(v.shape[0])
    comp = np.zeros(v.shape[0])
    with np.errstate(invalid="ignore", over="ignore"):
        for k in range(3):
            n = a[:, k] / safe
            summand = n * n - comp
            prelim = total + summand
            comp = (prelim - total) - summand
            total = prelim
        out = np.sqrt(total) * mx
    out = np.where(mx == 0, 0.0, out)
    out = np.where(np.isnan(a).any(axis=1), np.nan, out)
    return np.where(np.isinf(a).any(axis=1), np.inf, out)


def _normalise_rows(v: np.ndarray) -> np.ndarray:
    """`Math.hypot(nx, ny, nz) || 1` and the divisions of addMesh (src/compile.ts:268-270)."""
    length = js_hypot_rows(v)
    length = np.where((length > 0) | np.isnan(length), length, 1.0)
    length = np.where(np.isnan(length), 1.0, length)
    return v / length[:, None]


def flatten_meshes(meshes: Sequence[S.Mesh], material_index: Callable[[Any], int]) -> TriangleSink:
    """addMesh over every mesh (src/compile.ts:212-306), vectorised per group."""
    parts: Dict[str, List[np.ndarray]] = {k: [] for k in ("p", "n", "uv", "c", "hc", "m", "f", "s")}
    for mesh in meshes:
        g = mesh.geometry
        if g is None or g.position is None:
            continue
        position = np.asarray(g.position, np.float32).reshape(-1, 3).astype(np.float64)
        normal = None if g.normal is None else np.asarray(g.normal, np.float32).reshape(-1, 3).astype(np.float64)
        uv = None if g.uv is None else np.asarray(g.uv, np.float32).reshape(-1, 2).astype(np.float64)
        color = None
        if g.color is not None:
            ca = np.asarray(g.color, np.float32)
            item = 4 if ca.ndim == 2 and ca.shape[1] == 4 else 3
            ca = ca.reshape(-1, item).astype(np.float64)
            color = ca if item == 4 else np.concatenate([ca, np.ones((ca.shape[0], 1))], axis=1)
        index = None if g.index is None else np.asarray(g.index, np.int64)
        materials = list(mesh.material) if isinstance(mesh.material, (list, tuple)) else [mesh.material]
        total = index.size if index is not None else position.shape[0]
        start = max(0, g.draw_start)
        end = int(min(total, start + g.draw_count))
        groups = g.groups if (g.groups and isinstance(mesh.material, (list, tuple))) else [(0, math.inf, 0)]
        instances = [mesh.matrix_world]
        if isinstance(mesh, S.InstancedMesh):
            instances = [S.matmul4(mesh.matrix_world, mesh.instance_matrix[i]) for i in range(mesh.count)]
        flags_base = (TRI_CAST_SHADOW if mesh.cast_shadow else 0) | (TRI_RECEIVE_SHADOW if mesh.receive_shadow else 0)
        for world in instances:
            nm, det = _normal_matrix(world)
            w = np.asarray(world, np.float64)
            for gstart, gcount, gmat in groups:
                material = materials[gmat] if gmat < len(materials) else None
                if material is None or material.visible is False:
                    continue
                if material.wireframe:
                    warn_once("wireframe materials are left out")
                    continue
                mi = material_index(material)
                opaque = (not material.transparent) and not (material.alpha_test > 0) and \
                    not (getattr(material, "transmission", 0) > 0)
                flags = flags_base | (TRI_OPAQUE if opaque else 0)
                side = material.side
                use_colors = bool(material.vertex_colors) and color is not None
                lo = max(start, gstart)
                hi = int(min(end, gstart + gcount))
                # for (k = from; k + 2 < to; k += 3)
                ks = np.arange(lo, hi - 2, 3, dtype=np.int64) if hi - 2 > lo else np.zeros(0, np.int64)
                if ks.size == 0:
                    continue
                ids = np.stack([ks, ks + 1, ks + 2], axis=1)
                if index is not None:
                    ids = index[ids]
                if det < 0:
                    ids = ids[:, [0, 2, 1]]
                flat = ids.reshape(-1)
                x, y, z = position[flat, 0], position[flat, 1], position[flat, 2]
                px = w[0] * x + w[4] * y + w[8] * z + w[12]
                py = w[1] * x + w[5] * y + w[9] * z + w[13]
                pz = w[2] * x + w[6] * y + w[10] * z + w[14]
                p = np.stack([px, py, pz], axis=1).reshape(-1, 9)
                if normal is not None and not material.flat_shading:
                    nx0, ny0, nz0 = normal[flat, 0], normal[flat, 1], normal[flat, 2]
                    nn = np.stack([nm[0] * nx0 + nm[3] * ny0 + nm[6] * nz0,
                                   nm[1] * nx0 + nm[4] * ny0 + nm[7] * nz0,
                                   nm[2] * nx0 + nm[5] * ny0 + nm[8] * nz0], axis=1)
                    n = _normalise_rows(nn).reshape(-1, 9)
                else:
                    e = p[:, 3:6] - p[:, 0:3]
                    f = p[:, 6:9] - p[:, 0:3]
                    # normalize(), src/compile.ts:52-55, of the cross product written out as
                    # compile.ts:287-289 does.
                    face = np.stack([e[:, 1] * f[:, 2] - e[:, 2] * f[:, 1], e[:, 2] * f[:, 0] - e[:, 0] * f[:, 2],
                                     e[:, 0] * f[:, 1] - e[:, 1] * f[:, 0]], axis=1)
                    length = js_hypot_rows(face)
                    face = np.where(length[:, None] > 0, face / np.where(length > 0, length, 1)[:, None],
                                    np.array([0.0, 0.0, 1.0]))
                    n = np.tile(face, (1, 3))
                t = uv[flat].reshape(-1, 6) if uv is not None else np.zeros((ks.size, 6))
                if use_colors:
                    c = color[flat].reshape(-1, 12)
                    hc = np.ones(ks.size, np.uint8)
                else:
                    c = np.ones((ks.size, 12))
                    hc = np.zeros(ks.size, np.uint8)
                parts["p"].append(p)
                parts["n"].append(n)
                parts["uv"].append(t)
                parts["c"].append(c)
                parts["hc"].append(hc)
                parts["m"].append(np.full(ks.size, mi, np.uint32))
                parts["f"].append(np.full(ks.size, flags, np.uint8))
                parts["s"].append(np.full(ks.size, side, np.uint8))
    if not parts["p"]:
        return TriangleSink(np.zeros((0, 9)), np.zeros((0, 9)), np.zeros((0, 6)), np.zeros((0, 12)),
                            np.zeros(0, np.uint8), np.zeros(0, np.uint32), np.zeros(0, np.uint8),
                            np.zeros(0, np.uint8))
    cat = lambda k: np.ascontiguousarray(np.concatenate(parts[k]))  # noqa: E731
    return TriangleSink(cat("p"), cat("n"), cat("uv"), cat("c"), cat("hc"), cat("m"), cat("f"), cat("s"))


GeometryBuilder = Callable[[TriangleSink], CompiledGeometry]


def default_builder() -> GeometryBuilder:
    """The product's geometry builder: BVH build, reorder, tangents and epsilon on the
    GPU, through the default executor's `compile_sink`."""
    from .executors import default_executor

    return lambda sink: default_executor().compile_sink(sink)


def compile_geometry(meshes: Sequence[S.Mesh], material_index: Callable[[Any], int],
                     builder: Optional[GeometryBuilder] = None) -> CompiledGeometry:
    """compileGeometry, src/compile.ts:327-403."""
    sink = flatten_meshes(meshes, material_index)
    return (builder or default_builder())(sink)


def compile_scene(scene: S.Scene, filter: Optional[Callable[[Any], bool]] = None,
                  builder: Optional[GeometryBuilder] = None) -> CompiledScene:
    """compileScene, src/compile.ts:513-527."""
    shading, meshes = compile_shading(scene, filter)
    ids = {id(m): i for i, m in enumerate(shading.material_objects)}
    geometry = compile_geometry(meshes, lambda m: ids.get(id(m), 0), builder)
    return CompiledScene(geometry, shading.materials, shading.textures, shading.environments, shading.lights,
                         shading.background, shading.environment, shading.fog)


def compile_camera(camera: S.Camera, aspect: Optional[float] = None) -> CompiledCamera:
    """compileCamera, src/compile.ts:536-557."""
    if camera.parent is None:
        camera.update_matrix_world()
    world = [float(v) for v in camera.matrix_world]
    projection_inverse = [float(v) for v in camera.projection_matrix_inverse()]
    if aspect is not None and aspect > 0:
        p = camera.projection_matrix()
        camera_aspect = p[5] / p[0] if p[0] != 0 else 0
        if camera_aspect > 0:
            k = aspect / camera_aspect
            for i in range(4):
                projection_inverse[i] *= k
    return CompiledCamera(tuple(projection_inverse), tuple(world), bool(camera.orthographic),
                          _normalize((-world[8], -world[9], -world[10])), (world[12], world[13], world[14]))
