"""A small scene description in the shape of the three.js objects the reference reads.

The reference compiles three.js scene graphs (src/compile.ts). three.js is a
JavaScript library, so this module provides the subset of its object model the
compile step duck-types: Object3D transforms, meshes with buffer geometries,
the mesh materials, lights, cameras, data textures and fog. The numbers follow
three.js's published definitions (matrix composition, projection matrices,
geometry vertex layouts, sRGB colour decoding), restated from the mathematics.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence, Tuple, Union

import numpy as np

# ------------------------------------------------------------------ constants
FrontSide, BackSide, DoubleSide = 0, 1, 2
MultiplyOperation, MixOperation, AddOperation = 0, 1, 2
NoToneMapping, LinearToneMapping, ReinhardToneMapping, CineonToneMapping = 0, 1, 2, 3
ACESFilmicToneMapping, CustomToneMapping, AgXToneMapping, NeutralToneMapping = 4, 5, 6, 7
UVMapping = 300
CubeReflectionMapping, CubeRefractionMapping = 301, 302
EquirectangularReflectionMapping, EquirectangularRefractionMapping = 303, 304
RepeatWrapping, ClampToEdgeWrapping, MirroredRepeatWrapping = 1000, 1001, 1002
UnsignedByteType, FloatType, HalfFloatType = 1009, 1015, 1016
RGBAFormat = 1023
SRGBColorSpace, LinearSRGBColorSpace, NoColorSpace = "srgb", "srgb-linear", ""


def srgb_to_linear(c: float) -> float:
    """The sRGB decode three.js applies to hex colours (same formula as src/color.ts:11-13)."""
    return c * 0.0773993808 if c < 0.04045 else math.pow(c * 0.9478672986 + 0.0521327014, 2.4)


# ----------------------------------------------------------------------- math
def compose(position: Sequence[float], quaternion: Sequence[float], scale: Sequence[float]) -> np.ndarray:
    """Column-major 4x4 from translation, rotation quaternion (x, y, z, w) and scale."""
    x, y, z, w = quaternion
    x2, y2, z2 = x + x, y + y, z + z
    xx, xy, xz = x * x2, x * y2, x * z2
    yy, yz, zz = y * y2, y * z2, z * z2
    wx, wy, wz = w * x2, w * y2, w * z2
    sx, sy, sz = scale
    return np.array([
        (1 - (yy + zz)) * sx, (xy + wz) * sx, (xz - wy) * sx, 0,
        (xy - wz) * sy, (1 - (xx + zz)) * sy, (yz + wx) * sy, 0,
        (xz + wy) * sz, (yz - wx) * sz, (1 - (xx + yy)) * sz, 0,
        position[0], position[1], position[2], 1,
    ], dtype=np.float64)


def euler_to_quaternion(x: float, y: float, z: float, order: str = "XYZ") -> Tuple[float, float, float, float]:
    """Quaternion of an intrinsic Euler rotation (three.js Quaternion.setFromEuler)."""
    c1, c2, c3 = math.cos(x / 2), math.cos(y / 2), math.cos(z / 2)
    s1, s2, s3 = math.sin(x / 2), math.sin(y / 2), math.sin(z / 2)
    if order == "XYZ":
        return (s1 * c2 * c3 + c1 * s2 * s3, c1 * s2 * c3 - s1 * c2 * s3,
                c1 * c2 * s3 + s1 * s2 * c3, c1 * c2 * c3 - s1 * s2 * s3)
    raise ValueError(f"Euler order {order} is not supported")


def matmul4(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Column-major a * b."""
    return (a.reshape(4, 4).T @ b.reshape(4, 4).T).T.reshape(16)


def invert4(m: np.ndarray) -> np.ndarray:
    """Column-major inverse (zero matrix when singular, as three.js returns)."""
    mm = m.reshape(4, 4).T
    try:
        return np.linalg.inv(mm).T.reshape(16)
    except np.linalg.LinAlgError:
        return np.zeros(16)


def look_at_rotation(eye: Sequence[float], target: Sequence[float], up: Sequence[float], camera: bool) -> np.ndarray:
    """Column-major rotation that turns an object at `eye` toward `target`.

    Cameras and lights look down their -z axis, other objects down +z
    (three.js Object3D.lookAt).
    """
    e, t, u = np.asarray(eye, float), np.asarray(target, float), np.asarray(up, float)
    z = (e - t) if camera else (t - e)
    if np.dot(z, z) == 0:
        z = np.array([0.0, 0.0, 1.0])
    z = z / np.linalg.norm(z)
    x = np.cross(u, z)
    if np.dot(x, x) == 0:
        z = z + np.array([1e-4, 0, 0]) if abs(u[2]) == 1 else z + np.array([0, 0, 1e-4])
        z = z / np.linalg.norm(z)
        x = np.cross(u, z)
    x = x / np.linalg.norm(x)
    y = np.cross(z, x)
    return np.array([x[0], x[1], x[2], 0, y[0], y[1], y[2], 0, z[0], z[1], z[2], 0, 0, 0, 0, 1], float)


def quaternion_from_rotation(m: np.ndarray) -> Tuple[float, float, float, float]:
    """Quaternion of the rotation in a column-major 4x4 (three.js setFromRotationMatrix)."""
    m11, m12, m13 = m[0], m[4], m[8]
    m21, m22, m23 = m[1], m[5], m[9]
    m31, m32, m33 = m[2], m[6], m[10]
    trace = m11 + m22 + m33
    if trace > 0:
        s = 0.5 / math.sqrt(trace + 1.0)
        return ((m32 - m23) * s, (m13 - m31) * s, (m21 - m12) * s, 0.25 / s)
    if m11 > m22 and m11 > m33:
        s = 2.0 * math.sqrt(1.0 + m11 - m22 - m33)
        return (0.25 * s, (m12 + m21) / s, (m13 + m31) / s, (m32 - m23) / s)
    if m22 > m33:
        s = 2.0 * math.sqrt(1.0 + m22 - m11 - m33)
        return ((m12 + m21) / s, 0.25 * s, (m23 + m32) / s, (m13 - m31) / s)
    s = 2.0 * math.sqrt(1.0 + m33 - m11 - m22)
    return ((m13 + m31) / s, (m23 + m32) / s, 0.25 * s, (m21 - m12) / s)


# ---------------------------------------------------------------------- color
class Color:
    """Linear RGB. Color(0xff8800) decodes an sRGB hex, as three.js's colour management does."""

    def __init__(self, r: Union[float, int, "Color", None] = None, g: Optional[float] = None,
                 b: Optional[float] = None):
        if r is None:
            self.r = self.g = self.b = 1.0
        elif isinstance(r, Color):
            self.r, self.g, self.b = r.r, r.g, r.b
        elif g is None:
            self.set_hex(int(r))
        else:
            self.r, self.g, self.b = float(r), float(g), float(b)

    def set_hex(self, hex_value: int) -> "Color":
        self.r = srgb_to_linear(((hex_value >> 16) & 255) / 255)
        self.g = srgb_to_linear(((hex_value >> 8) & 255) / 255)
        self.b = srgb_to_linear((hex_value & 255) / 255)
        return self

    def set(self, value: Union[int, "Color"]) -> "Color":
        if isinstance(value, Color):
            self.r, self.g, self.b = value.r, value.g, value.b
            return self
        return self.set_hex(int(value))

    def tuple(self, scale: float = 1.0) -> Tuple[float, float, float]:
        return (self.r * scale, self.g * scale, self.b * scale)


def _color(value: Any, default: int) -> Color:
    if value is None:
        return Color(default)
    return value if isinstance(value, Color) else Color(value)


# --------------------------------------------------------------------- object
class Vector3:
    def __init__(self, x: float = 0.0, y: float = 0.0, z: float = 0.0):
        self.x, self.y, self.z = float(x), float(y), float(z)

    def set(self, x: float, y: float, z: float) -> "Vector3":
        self.x, self.y, self.z = float(x), float(y), float(z)
        return self

    def tuple(self) -> Tuple[float, float, float]:
        return (self.x, self.y, self.z)


class Euler(Vector3):
    order = "XYZ"


class Object3D:
    """Transform node: position, XYZ Euler rotation (or a quaternion from lookAt), scale."""

    def __init__(self) -> None:
        self.position = Vector3()
        self.rotation = Euler()
        self.scale = Vector3(1, 1, 1)
        self._quaternion: Optional[Tuple[float, float, float, float]] = None
        self.children: List[Object3D] = []
        self.parent: Optional[Object3D] = None
        self.visible = True
        self.cast_shadow = False
        self.receive_shadow = False
        self.user_data: Dict[str, Any] = {}
        self.name = ""
        self.type = "Object3D"
        self.matrix_world = np.eye(4).reshape(16)

    def add(self, *objects: "Object3D") -> "Object3D":
        for o in objects:
            if o.parent is not None:
                o.parent.children.remove(o)
            o.parent = self
            self.children.append(o)
        return self

    def quaternion(self) -> Tuple[float, float, float, float]:
        if self._quaternion is not None:
            return self._quaternion
        return euler_to_quaternion(self.rotation.x, self.rotation.y, self.rotation.z)

    def local_matrix(self) -> np.ndarray:
        return compose(self.position.tuple(), self.quaternion(), self.scale.tuple())

    def update_matrix_world(self, parent: Optional[np.ndarray] = None) -> None:
        local = self.local_matrix()
        self.matrix_world = local if parent is None else matmul4(parent, local)
        for c in self.children:
            c.update_matrix_world(self.matrix_world)

    def look_at(self, x: float, y: float, z: float) -> None:
        self.update_matrix_world(None if self.parent is None else self.parent.matrix_world)
        eye = self.matrix_world[12:15]
        camera_like = isinstance(self, (Camera, Light))
        m = look_at_rotation(eye, (x, y, z), (0, 1, 0), camera_like)
        self._quaternion = quaternion_from_rotation(m)

    def traverse(self):
        yield self
        for c in self.children:
            yield from c.traverse()


class Scene(Object3D):
    def __init__(self) -> None:
        super().__init__()
        self.type = "Scene"
        self.background: Any = None
        self.background_intensity = 1.0
        self.background_rotation: Optional[Euler] = None
        self.environment: Any = None
        self.environment_intensity = 1.0
        self.environment_rotation: Optional[Euler] = None
        self.fog: Any = None


class Group(Object3D):
    pass


# ------------------------------------------------------------------- textures
class DataTexture:
    """Raw RGBA pixels, rows bottom to top as three.js DataTextures are (flipY false)."""

    _next_id = 1

    def __init__(self, data: np.ndarray, width: int, height: int, format: int = RGBAFormat,
                 type: Optional[int] = None):
        self.data = np.asarray(data)
        self.width, self.height, self.format = int(width), int(height), format
        if type is None:
            type = FloatType if self.data.dtype == np.float32 else UnsignedByteType
        self.type = type
        self.wrap_s = self.wrap_t = ClampToEdgeWrapping
        self.repeat = [1.0, 1.0]
        self.offset = [0.0, 0.0]
        self.center = [0.0, 0.0]
        self.rotation = 0.0
        self.flip_y = False
        self.color_space = NoColorSpace
        self.mapping = UVMapping
        self.version = 0  # bump after editing the pixels in place (three.js texture.needsUpdate)
        self.id = DataTexture._next_id
        DataTexture._next_id += 1

    def matrix(self) -> Tuple[float, ...]:
        """Column-major uv transform (three.js Matrix3.setUvTransform)."""
        tx, ty = self.offset
        sx, sy = self.repeat
        c, s = math.cos(self.rotation), math.sin(self.rotation)
        cx, cy = self.center
        return (sx * c, -sy * s, 0.0, sx * s, sy * c, 0.0,
                -sx * (c * cx + s * cy) + cx + tx, -sy * (-s * cx + c * cy) + cy + ty, 1.0)


class CubeTexture:
    """Six RGBA face images (+x, -x, +y, -y, +z, -z), each first row first, as a
    three.js CubeTexture holds them; mapping CubeReflectionMapping unless set."""

    _next_id = 1

    def __init__(self, images: Sequence[np.ndarray], width: int, height: int, format: int = RGBAFormat,
                 type: Optional[int] = None):
        if len(images) != 6:
            raise ValueError("a cube texture has six face images")
        self.images = [np.asarray(i) for i in images]
        self.width, self.height, self.format = int(width), int(height), format
        if type is None:
            type = FloatType if self.images[0].dtype == np.float32 else UnsignedByteType
        self.type = type
        self.wrap_s = self.wrap_t = ClampToEdgeWrapping
        self.flip_y = False
        self.color_space = NoColorSpace
        self.mapping = CubeReflectionMapping
        self.is_render_target_texture = False
        self.version = 0
        self.id = CubeTexture._next_id
        CubeTexture._next_id += 1


# ------------------------------------------------------------------- geometry
@dataclass
class BufferGeometry:
    """Vertex attributes (float arrays of n x itemSize), optional index and groups."""

    position: np.ndarray
    normal: Optional[np.ndarray] = None
    uv: Optional[np.ndarray] = None
    color: Optional[np.ndarray] = None
    index: Optional[np.ndarray] = None
    groups: List[Tuple[int, int, int]] = field(default_factory=list)  # (start, count, materialIndex)
    draw_start: int = 0
    draw_count: float = math.inf
    version: int = 0  # bump after editing the arrays in place (three.js attribute.needsUpdate)

    def add_group(self, start: int, count: int, material_index: int) -> None:
        self.groups.append((start, count, material_index))


def plane_geometry(width: float = 1, height: float = 1, ws: int = 1, hs: int = 1) -> BufferGeometry:
    """three.js PlaneGeometry: a grid in z = 0 facing +z."""
    gx, gy = int(ws), int(hs)
    sw, sh = width / gx, height / gy
    pos, nrm, uv, idx = [], [], [], []
    for iy in range(gy + 1):
        y = iy * sh - height / 2
        for ix in range(gx + 1):
            x = ix * sw - width / 2
            pos.append((x, -y, 0.0))
            nrm.append((0.0, 0.0, 1.0))
            uv.append((ix / gx, 1 - iy / gy))
    for iy in range(gy):
        for ix in range(gx):
            a = ix + (gx + 1) * iy
            b = ix + (gx + 1) * (iy + 1)
            c = ix + 1 + (gx + 1) * (iy + 1)
            d = ix + 1 + (gx + 1) * iy
            idx += [a, b, d, b, c, d]
    return BufferGeometry(np.array(pos, np.float32), np.array(nrm, np.float32), np.array(uv, np.float32),
                          index=np.array(idx, np.uint32))


def box_geometry(width: float = 1, height: float = 1, depth: float = 1) -> BufferGeometry:
    """three.js BoxGeometry: six planes, one group per face (+x, -x, +y, -y, +z, -z)."""
    pos: List[Tuple[float, ...]] = []
    nrm: List[Tuple[float, ...]] = []
    uv: List[Tuple[float, ...]] = []
    idx: List[int] = []
    geo = BufferGeometry(np.zeros((0, 3), np.float32))
    axes = {"x": 0, "y": 1, "z": 2}

    def plane(u: str, v: str, w: str, udir: float, vdir: float, pw: float, ph: float, pd: float, mat: int) -> None:
        start_vertex = len(pos)
        start_index = len(idx)
        for iy in range(2):
            y = iy * ph - ph / 2
            for ix in range(2):
                x = ix * pw - pw / 2
                vec = [0.0, 0.0, 0.0]
                vec[axes[u]] = x * udir
                vec[axes[v]] = y * vdir
                vec[axes[w]] = pd / 2
                pos.append(tuple(vec))
                n = [0.0, 0.0, 0.0]
                n[axes[w]] = 1.0 if pd > 0 else -1.0
                nrm.append(tuple(n))
                uv.append((ix, 1 - iy))
        a, b, c, d = start_vertex, start_vertex + 2, start_vertex + 3, start_vertex + 1
        idx.extend([a, b, d, b, c, d])
        geo.add_group(start_index, 6, mat)

    plane("z", "y", "x", -1, -1, depth, height, width, 0)
    plane("z", "y", "x", 1, -1, depth, height, -width, 1)
    plane("x", "z", "y", 1, 1, width, depth, height, 2)
    plane("x", "z", "y", 1, -1, width, depth, -height, 3)
    plane("x", "y", "z", 1, -1, width, height, depth, 4)
    plane("x", "y", "z", -1, -1, width, height, -depth, 5)
    geo.position = np.array(pos, np.float32)
    geo.normal = np.array(nrm, np.float32)
    geo.uv = np.array(uv, np.float32)
    geo.index = np.array(idx, np.uint32)
    return geo


def sphere_geometry(radius: float = 1, ws: int = 32, hs: int = 16) -> BufferGeometry:
    """three.js SphereGeometry: latitude rows from +y down, poles as single triangles."""
    ws, hs = max(3, int(ws)), max(2, int(hs))
    pos, nrm, uv = [], [], []
    grid = []
    for iy in range(hs + 1):
        row = []
        v = iy / hs
        u_off = 0.5 / ws if iy == 0 else (-0.5 / ws if iy == hs else 0.0)
        for ix in range(ws + 1):
            u = ix / ws
            x = -radius * math.cos(u * 2 * math.pi) * math.sin(v * math.pi)
            y = radius * math.cos(v * math.pi)
            z = radius * math.sin(u * 2 * math.pi) * math.sin(v * math.pi)
            pos.append((x, y, z))
            length = math.sqrt(x * x + y * y + z * z) or 1.0
            nrm.append((x / length, y / length, z / length))
            uv.append((u + u_off, 1 - v))
            row.append(len(pos) - 1)
        grid.append(row)
    idx = []
    for iy in range(hs):
        for ix in range(ws):
            a, b = grid[iy][ix + 1], grid[iy][ix]
            c, d = grid[iy + 1][ix], grid[iy + 1][ix + 1]
            if iy != 0:
                idx += [a, b, d]
            if iy != hs - 1:
                idx += [b, c, d]
    return BufferGeometry(np.array(pos, np.float32), np.array(nrm, np.float32), np.array(uv, np.float32),
                          index=np.array(idx, np.uint32))


# ------------------------------------------------------------------ materials
class Material:
    """Common material properties (three.js Material) read by compileMaterial."""

    kind = "Material"

    def __init__(self, **kw: Any) -> None:
        self.side = FrontSide
        self.opacity = 1.0
        self.transparent = False
        self.alpha_test = 0.0
        self.vertex_colors = False
        self.flat_shading = False
        self.tone_mapped = True
        self.visible = True
        self.wireframe = False
        self.color: Optional[Color] = Color(0xffffff)
        self.map = self.alpha_map = self.emissive_map = self.normal_map = None
        self.ao_map = self.roughness_map = self.metalness_map = self.env_map = None
        self.emissive: Optional[Color] = None
        self.emissive_intensity = 1.0
        self.normal_scale = (1.0, 1.0)
        self.ao_map_intensity = 1.0
        self.env_map_intensity: Optional[float] = None
        self.env_map_rotation: Optional[Euler] = None
        self.reflectivity: Optional[float] = None
        self.combine: Optional[int] = None
        self._apply(kw)

    def _apply(self, kw: Dict[str, Any]) -> None:
        for key, value in kw.items():
            if not hasattr(self, key):
                raise TypeError(f"{type(self).__name__} has no property {key}")
            if key in ("color", "emissive", "specular", "specular_color", "attenuation_color") and value is not None:
                value = _color(value, 0xffffff)
            setattr(self, key, value)


class MeshBasicMaterial(Material):
    kind = "basic"

    def __init__(self, **kw: Any) -> None:
        super().__init__()
        self.reflectivity = 1.0
        self.combine = MultiplyOperation
        self._apply(kw)


class MeshLambertMaterial(Material):
    kind = "lambert"

    def __init__(self, **kw: Any) -> None:
        super().__init__()
        self.emissive = Color(0x000000)
        self.reflectivity = 1.0
        self.combine = MultiplyOperation
        self._apply(kw)


class MeshToonMaterial(Material):
    kind = "toon"

    def __init__(self, **kw: Any) -> None:
        super().__init__()
        self.emissive = Color(0x000000)
        self._apply(kw)


class MeshPhongMaterial(Material):
    kind = "phong"

    def __init__(self, **kw: Any) -> None:
        super().__init__()
        self.emissive = Color(0x000000)
        self.specular = Color(0x111111)
        self.shininess = 30.0
        self.reflectivity = 1.0
        self.combine = MultiplyOperation
        self._apply(kw)


class MeshStandardMaterial(Material):
    kind = "standard"

    def __init__(self, **kw: Any) -> None:
        super().__init__()
        self.emissive = Color(0x000000)
        self.roughness = 1.0
        self.metalness = 0.0
        self.env_map_intensity = 1.0
        self._apply(kw)


class MeshPhysicalMaterial(MeshStandardMaterial):
    kind = "physical"

    def __init__(self, **kw: Any) -> None:
        super().__init__()
        self.ior = 1.5
        self.specular_intensity = 1.0
        self.specular_color = Color(1.0, 1.0, 1.0)
        self.transmission = 0.0
        self.thickness = 0.0
        self.attenuation_distance = math.inf
        self.attenuation_color = Color(1.0, 1.0, 1.0)
        self._apply(kw)


# ----------------------------------------------------------------------- mesh
class Mesh(Object3D):
    def __init__(self, geometry: BufferGeometry, material: Union[Material, Sequence[Material]]):
        super().__init__()
        self.type = "Mesh"
        self.geometry = geometry
        self.material = material


class InstancedMesh(Mesh):
    def __init__(self, geometry: BufferGeometry, material: Material, count: int):
        super().__init__(geometry, material)
        self.count = int(count)
        self.instance_matrix = np.tile(np.eye(4).reshape(16), (self.count, 1))

    def set_matrix_at(self, i: int, m: np.ndarray) -> None:
        self.instance_matrix[i] = np.asarray(m, float).reshape(16)


# --------------------------------------------------------------------- lights
class Light(Object3D):
    def __init__(self, color: Any = 0xffffff, intensity: float = 1.0):
        super().__init__()
        self.type = "Light"
        self.color = _color(color, 0xffffff)
        self.intensity = float(intensity)


class AmbientLight(Light):
    pass


class HemisphereLight(Light):
    def __init__(self, sky: Any = 0xffffff, ground: Any = 0xffffff, intensity: float = 1.0):
        super().__init__(sky, intensity)
        self.ground_color = _color(ground, 0xffffff)
        self.position.set(0, 1, 0)


class DirectionalLight(Light):
    def __init__(self, color: Any = 0xffffff, intensity: float = 1.0):
        super().__init__(color, intensity)
        self.position.set(0, 1, 0)
        self.target = Object3D()


class PointLight(Light):
    def __init__(self, color: Any = 0xffffff, intensity: float = 1.0, distance: float = 0.0, decay: float = 2.0):
        super().__init__(color, intensity)
        self.distance, self.decay = float(distance), float(decay)


class SpotLight(Light):
    def __init__(self, color: Any = 0xffffff, intensity: float = 1.0, distance: float = 0.0,
                 angle: float = math.pi / 3, penumbra: float = 0.0, decay: float = 2.0):
        super().__init__(color, intensity)
        self.distance, self.angle, self.penumbra, self.decay = float(distance), float(angle), float(penumbra), float(decay)
        self.position.set(0, 1, 0)
        self.target = Object3D()


# -------------------------------------------------------------------- cameras
class Camera(Object3D):
    orthographic = False

    def projection_matrix(self) -> np.ndarray:
        raise NotImplementedError

    def projection_matrix_inverse(self) -> np.ndarray:
        return invert4(self.projection_matrix())


class PerspectiveCamera(Camera):
    def __init__(self, fov: float = 50, aspect: float = 1, near: float = 0.1, far: float = 2000):
        super().__init__()
        self.fov, self.aspect, self.near, self.far = float(fov), float(aspect), float(near), float(far)
        self.zoom = 1.0

    def projection_matrix(self) -> np.ndarray:
        near, far = self.near, self.far
        top = near * math.tan(math.radians(0.5 * self.fov)) / self.zoom
        height = 2 * top
        width = self.aspect * height
        left = -0.5 * width
        right, bottom = left + width, top - height
        x = 2 * near / (right - left)
        y = 2 * near / (top - bottom)
        a = (right + left) / (right - left)
        b = (top + bottom) / (top - bottom)
        c = -(far + near) / (far - near)
        d = -2 * far * near / (far - near)
        return np.array([x, 0, 0, 0, 0, y, 0, 0, a, b, c, -1, 0, 0, d, 0], float)


class OrthographicCamera(Camera):
    orthographic = True

    def __init__(self, left: float = -1, right: float = 1, top: float = 1, bottom: float = -1,
                 near: float = 0.1, far: float = 2000):
        super().__init__()
        self.left, self.right, self.top, self.bottom = float(left), float(right), float(top), float(bottom)
        self.near, self.far = float(near), float(far)
        self.zoom = 1.0

    def projection_matrix(self) -> np.ndarray:
        dx = (self.right - self.left) / (2 * self.zoom)
        dy = (self.top - self.bottom) / (2 * self.zoom)
        cx, cy = (self.right + self.left) / 2, (self.top + self.bottom) / 2
        left, right, top, bottom = cx - dx, cx + dx, cy + dy, cy - dy
        w, h, p = 1 / (right - left), 1 / (top - bottom), 1 / (self.far - self.near)
        x, y, z = (right + left) * w, (top + bottom) * h, (self.far + self.near) * p
        return np.array([2 * w, 0, 0, 0, 0, 2 * h, 0, 0, 0, 0, -2 * p, 0, -x, -y, -z, 1], float)


# ------------------------------------------------------------------------ fog
class Fog:
    def __init__(self, color: Any = 0xffffff, near: float = 1, far: float = 1000):
        self.color = _color(color, 0xffffff)
        self.near, self.far = float(near), float(far)


class FogExp2:
    def __init__(self, color: Any = 0xffffff, density: float = 0.00025):
        self.color = _color(color, 0xffffff)
        self.density = float(density)
