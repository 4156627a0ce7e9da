"""Seeded synthetic scenes of the benchmark configurations.

No public dataset is involved: every scene is generated from a fixed seed
(0x5EED0000 + configuration index) with the shapes, sizes and value
distributions the configurations name. Placements the configurations leave
open (light positions, camera of the mid scene, ground material) are fixed
here, in the functions below.

  small_scene()  22,530 triangles: a 40 x 40 ground plane and 64 UV spheres
                 (16 x 12 segments), 320 x 240, 16 spp, GI off, ACES, sRGB.
  mid_scene()    1,310,720 triangles: 256 icospheres subdivided 4 times
                 (5,120 triangles each) displaced by value noise on a 16 x 16
                 grid, mixed Standard / Physical / Phong materials, half with
                 256 x 256 noise albedo maps; 1920 x 1080, 64 spp, GI on,
                 4 bounces, ACES, sRGB.
  mid_scene(grid=32)  the serving loop's large version: 1,024 icospheres,
                 5,242,880 triangles.
  soup_scene()   2,000,000 random triangles, edge lengths U(0.01, 0.2), in a
                 20^3 box, Lambert albedo U(0, 1)^3 per triangle (vertex colours).
  orbit_camera() the serving loop's clients: a camera on a circle around a
                 scene, aimed at its centre.
"""
from __future__ import annotations

import functools
import math
from dataclasses import dataclass, field
from typing import Any, Dict, List, Tuple

import numpy as np

from . import scene as S

SEED_BASE = 0x5EED0000


@dataclass
class BenchScene:
    """A scene description, its camera, image size and raytrace options."""

    name: str
    scene: S.Scene
    camera: S.Camera
    width: int
    height: int
    options: Dict[str, Any] = field(default_factory=dict)
    triangles: int = 0


def _srgb_color(rgb: np.ndarray) -> S.Color:
    """An sRGB-encoded colour decoded to linear, as three.js's setRGB(..., SRGBColorSpace) does."""
    return S.Color(S.srgb_to_linear(float(rgb[0])), S.srgb_to_linear(float(rgb[1])), S.srgb_to_linear(float(rgb[2])))


def small_scene(seed: int = SEED_BASE + 0) -> BenchScene:
    """The small plain-method scene (a few thousand lines of three.js in the reference's terms)."""
    rng = np.random.default_rng(seed)
    scene = S.Scene()
    ground = S.Mesh(S.plane_geometry(40, 40), S.MeshStandardMaterial(color=S.Color(0.5, 0.5, 0.5), roughness=0.9))
    ground.rotation.x = -math.pi / 2
    scene.add(ground)
    count = 0
    for _ in range(64):
        r = float(rng.uniform(0.3, 1.2))
        x, z = float(rng.uniform(-8, 8)), float(rng.uniform(-8, 8))
        colour = rng.uniform(0, 1, 3)
        material = S.MeshStandardMaterial(color=_srgb_color(colour), roughness=float(rng.uniform(0.05, 1)),
                                          metalness=float(rng.integers(0, 2)))
        sphere = S.Mesh(S.sphere_geometry(r, 16, 12), material)
        sphere.position.set(x, r, z)
        scene.add(sphere)
        count += 352
    sun = S.DirectionalLight(0xffffff, 3)
    sun.position.set(5, 10, 7)
    sun.cast_shadow = True
    lamp = S.PointLight(0xffffff, 50, 0)
    lamp.position.set(-4, 6, 4)
    scene.add(sun, lamp)
    camera = S.PerspectiveCamera(50, 320 / 240, 0.1, 2000)
    camera.position.set(0, 6, 16)
    camera.look_at(0, 0, 0)
    camera.update_matrix_world()
    return BenchScene("small: 64 UV spheres + ground, 22,530 tris, 320x240, 16 spp, GI off", scene, camera, 320, 240,
                      {"samples": 16, "global_illumination": False, "tone_mapping": S.ACESFilmicToneMapping,
                       "output_color_space": "srgb", "max_bounces": 4}, count + 2)


# ------------------------------------------------------------- icospheres
@functools.lru_cache(maxsize=8)
def _icosphere(subdivisions: int) -> Tuple[np.ndarray, np.ndarray]:
    v, f = _make_icosphere(subdivisions)
    v.setflags(write=False)
    f.setflags(write=False)
    return v, f


def icosphere(subdivisions: int) -> Tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: an icosahedron whose faces are split in four `subdivisions`
    times, new vertices pushed to the sphere. Returns (vertices [v, 3], faces [f, 3])."""
    v, f = _icosphere(subdivisions)
    return v.copy(), f.copy()


def _make_icosphere(subdivisions: int) -> Tuple[np.ndarray, np.ndarray]:
    t = (1 + math.sqrt(5)) / 2
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.array(verts, np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(faces, np.int64)
    for _ in range(subdivisions):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inverse = np.unique(key, axis=0, return_inverse=True)
        mids = v[uniq[:, 0]] + v[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mids])
        m = inverse.reshape(3, -1).T + base  # midpoints of edges 01, 12, 20
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    return v, f


def _lattice_hash(ix: np.ndarray, iy: np.ndarray, iz: np.ndarray, seed: int) -> np.ndarray:
    """A value in [0, 1) per integer lattice point (lowbias32-style integer mix)."""
    h = (ix.astype(np.int64) * 73856093) ^ (iy.astype(np.int64) * 19349663) ^ (iz.astype(np.int64) * 83492791)
    h = (h ^ seed) & 0xFFFFFFFF
    h ^= h >> 16
    h = (h * 0x7FEB352D) & 0xFFFFFFFF
    h ^= h >> 15
    h = (h * 0x846CA68B) & 0xFFFFFFFF
    h ^= h >> 16
    return h.astype(np.float64) / 4294967296.0


def value_noise3(p: np.ndarray, seed: int) -> np.ndarray:
    """Smoothly interpolated lattice value noise in [0, 1) at points p [n, 3]."""
    f = np.floor(p)
    i = f.astype(np.int64)
    t = p - f
    w = t * t * (3 - 2 * t)
    out = np.zeros(p.shape[0])
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                h = _lattice_hash(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += h * wx * wy * wz
    return out


def noise_texture(size: int, seed: int) -> np.ndarray:
    """size x size RGBA8 value-noise image: two octaves of smoothly interpolated
    seeded lattice values per colour channel, opaque."""
    rng = np.random.default_rng(seed)
    img = np.zeros((size, size, 3))
    coords = np.arange(size) / 32.0
    for freq, amp in ((1.0, 0.65), (2.7, 0.35)):
        c = coords * freq
        i = np.floor(c).astype(np.int64)
        t = c - i
        w = t * t * (3 - 2 * t)
        n = int(i.max()) + 2
        for ch in range(3):
            g = rng.uniform(0, 1, (n, n))
            v = (g[np.ix_(i, i)] * np.outer(1 - w, 1 - w) + g[np.ix_(i, i + 1)] * np.outer(1 - w, w) +
                 g[np.ix_(i + 1, i)] * np.outer(w, 1 - w) + g[np.ix_(i + 1, i + 1)] * np.outer(w, w))
            img[:, :, ch] += amp * v
    out = np.empty((size, size, 4), np.uint8)
    out[:, :, :3] = np.clip(img * 255 + 0.5, 0, 255).astype(np.uint8)
    out[:, :, 3] = 255
    return out.reshape(-1)


def displaced_icosphere(subdivisions: int, amplitude: float, seed: int) -> S.BufferGeometry:
    """An icosphere whose radius is 1 + amplitude * (noise - 0.5), with smooth
    normals from the displaced faces and spherical uvs."""
    v, f = icosphere(subdivisions)
    r = 1 + amplitude * (value_noise3(v * 3.0 + 11.0, seed) - 0.5)
    p = v * r[:, None]
    e1 = p[f[:, 1]] - p[f[:, 0]]
    e2 = p[f[:, 2]] - p[f[:, 0]]
    fn = np.cross(e1, e2)
    n = np.zeros_like(p)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    uv = np.stack([np.arctan2(v[:, 2], v[:, 0]) / (2 * math.pi) + 0.5, np.arcsin(np.clip(v[:, 1], -1, 1)) / math.pi + 0.5],
                  axis=1)
    return S.BufferGeometry(p.astype(np.float32), n.astype(np.float32), uv.astype(np.float32),
                            index=f.reshape(-1).astype(np.uint32))


def mid_scene(seed: int = SEED_BASE + 1, grid: int = 16, subdivisions: int = 4, width: int = 1920,
              height: int = 1080, samples: int = 64) -> BenchScene:
    """The path-traced mid scene: grid x grid displaced icospheres."""
    rng = np.random.default_rng(seed)
    scene = S.Scene()
    spacing = 5.0
    textures: List[S.DataTexture] = []
    count = 0
    for gz in range(grid):
        for gx in range(grid):
            k = gz * grid + gx
            geometry = displaced_icosphere(subdivisions, 0.1, seed + k)
            kind = rng.uniform()
            if kind < 0.4:
                material: S.Material = S.MeshStandardMaterial(roughness=float(rng.uniform(0, 1)),
                                                              metalness=float(rng.uniform(0, 1)))
            elif kind < 0.7:
                material = S.MeshPhysicalMaterial(transmission=1.0, ior=1.5, roughness=float(rng.uniform(0, 0.2)))
            else:
                material = S.MeshPhongMaterial(shininess=float(rng.uniform(1, 200)))
            material.color = _srgb_color(rng.uniform(0.2, 1.0, 3))
            if rng.uniform() < 0.5:
                tex = S.DataTexture(noise_texture(256, seed + 1000 + k), 256, 256)
                tex.color_space = S.SRGBColorSpace
                tex.wrap_s = tex.wrap_t = S.RepeatWrapping
                material.map = tex
                textures.append(tex)
            mesh = S.Mesh(geometry, material)
            s = float(rng.uniform(0.5, 2.0))
            mesh.scale.set(s, s, s)
            mesh.position.set((gx - (grid - 1) / 2) * spacing, s, (gz - (grid - 1) / 2) * spacing)
            scene.add(mesh)
            count += f_count(subdivisions)
    half = grid * spacing / 2
    for sx, sz in ((-1, -1), (-1, 1), (1, -1), (1, 1)):
        light = S.PointLight(0xffffff, 2500.0, 0, 2)
        light.position.set(sx * half * 0.5, 40.0, sz * half * 0.5)
        scene.add(light)
    scene.add(S.HemisphereLight(0xddeeff, 0x202020, 0.5))
    camera = S.PerspectiveCamera(50, width / height, 0.1, 2000)
    camera.position.set(0, 32, 62)
    camera.look_at(0, 0, 0)
    camera.update_matrix_world()
    return BenchScene(f"mid: {grid * grid} displaced icospheres, {count:,} tris, {width}x{height}, {samples} spp, GI on",
                      scene, camera, width, height,
                      {"samples": samples, "global_illumination": True, "max_bounces": 4,
                       "tone_mapping": S.ACESFilmicToneMapping, "output_color_space": "srgb"}, count)


def f_count(subdivisions: int) -> int:
    return 20 * 4 ** subdivisions


def soup_scene(seed: int = SEED_BASE + 3, count: int = 2_000_000, box: float = 20.0, width: int = 1280,
               height: int = 720, samples: int = 64) -> BenchScene:
    """A random triangle soup: `count` triangles with a random first vertex in the box and
    edges of length U(0.01, 0.2) in random directions, one Lambert material with a
    U(0, 1)^3 albedo per triangle as vertex colours; a sun with shadows and a hemisphere light."""
    rng = np.random.default_rng(seed)
    v0 = rng.uniform(-box / 2, box / 2, (count, 3))

    def edge() -> np.ndarray:
        d = rng.normal(size=(count, 3))
        d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-12)
        return d * rng.uniform(0.01, 0.2, (count, 1))

    v1, v2 = v0 + edge(), v0 + edge()
    p = np.stack([v0, v1, v2], axis=1).astype(np.float32)  # [n, 3, 3]
    fn = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]).astype(np.float64)
    fn /= np.maximum(np.linalg.norm(fn, axis=1, keepdims=True), 1e-30)
    n = np.repeat(fn[:, None, :], 3, axis=1).astype(np.float32)
    albedo = rng.uniform(0, 1, (count, 3))
    colors = np.repeat(albedo[:, None, :], 3, axis=1).astype(np.float32)
    geometry = S.BufferGeometry(p.reshape(-1, 3), n.reshape(-1, 3), None, color=colors.reshape(-1, 3))
    material = S.MeshLambertMaterial(vertex_colors=True, side=S.DoubleSide)
    scene = S.Scene()
    scene.add(S.Mesh(geometry, material))
    sun = S.DirectionalLight(0xffffff, 3)
    sun.position.set(10, 20, 5)
    sun.cast_shadow = True
    scene.add(sun, S.HemisphereLight(0xddeeff, 0x202020, 0.5))
    camera = S.PerspectiveCamera(50, width / height, 0.1, 2000)
    camera.position.set(0, 12, 34)
    camera.look_at(0, 0, 0)
    camera.update_matrix_world()
    return BenchScene(f"soup: {count:,} random triangles in a {box:g}^3 box, {width}x{height}, {samples} spp, GI on",
                      scene, camera, width, height,
                      {"samples": samples, "global_illumination": True, "max_bounces": 4,
                       "tone_mapping": S.ACESFilmicToneMapping, "output_color_space": "srgb"}, count)


def orbit_camera(radius: float, height: float, angle_deg: float, target: Tuple[float, float, float] = (0, 0, 0),
                 aspect: float = 16 / 9, fov: float = 50) -> S.PerspectiveCamera:
    """A perspective camera on a circle of `radius` at `height` above the target, at
    `angle_deg` around the y axis, looking at the target."""
    a = math.radians(angle_deg)
    camera = S.PerspectiveCamera(fov, aspect, 0.1, 4000)
    camera.position.set(target[0] + radius * math.sin(a), target[1] + height, target[2] + radius * math.cos(a))
    camera.look_at(*target)
    camera.update_matrix_world()
    return camera


# ------------------------------------------------------ large instanced scene
@dataclass
class InstancedScene:
    """Instances of one mesh for the per-frame rebuild workload: the mesh, the
    shading (materials, textures, lights as a CompiledScene without geometry),
    one material per instance and the camera."""

    name: str
    mesh: S.BufferGeometry
    shading: Any  # CompiledScene with geometry None
    materials: np.ndarray  # material index of each instance
    camera: S.Camera
    width: int
    height: int
    options: Dict[str, Any]
    count: int
    box: float
    seed: int

    @property
    def triangles(self) -> int:
        return self.count * (len(self.mesh.index) // 3 if self.mesh.index is not None else 0)

    def frame(self, k: int) -> List[Tuple[np.ndarray, int, int, int, int, bool]]:
        """Frame k's instances: rotations uniform on SO(3) (unit quaternions from normal
        deviates), translations uniform in the box, all re-drawn per frame."""
        rng = np.random.default_rng(self.seed * 1000003 + k)
        q = rng.normal(size=(self.count, 4))
        q /= np.linalg.norm(q, axis=1, keepdims=True)
        w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
        r = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y + z * w), 2 * (x * z - y * w),
                      2 * (x * y - z * w), 1 - 2 * (x * x + z * z), 2 * (y * z + x * w),
                      2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y)], axis=1)
        t = rng.uniform(-self.box / 2, self.box / 2, (self.count, 3))
        out = []
        for i in range(self.count):
            m = np.zeros(16)
            m[0:3], m[4:7], m[8:11] = r[i, 0:3], r[i, 3:6], r[i, 6:9]  # columns
            m[12:15] = t[i]
            m[15] = 1.0
            out.append((m, 0, int(self.materials[i]), 7, 0, False))
        return out


def large_scene(seed: int = SEED_BASE + 4, count: int = 4096, subdivisions: int = 5, radius: float = 3.0,
                box: float = 200.0, width: int = 2048, height: int = 2048, samples: int = 16) -> InstancedScene:
    """The per-frame rebuild workload: `count` icospheres subdivided `subdivisions` times
    (20,480 triangles each at 5) under random rigid transforms in a box^3 region, with the
    mid scene's mix of Standard / transmissive Physical / Phong materials (half with noise
    albedo maps); 2048 x 2048, 16 spp, GI on, 8 bounces, ACES, sRGB."""
    from .compile import compile_shading

    rng = np.random.default_rng(seed)
    v, f = icosphere(subdivisions)
    p = (v * radius).astype(np.float32)
    uv = np.stack([np.arctan2(v[:, 2], v[:, 0]) / (2 * math.pi) + 0.5,
                   np.arcsin(np.clip(v[:, 1], -1, 1)) / math.pi + 0.5], axis=1).astype(np.float32)
    mesh = S.BufferGeometry(p, v.astype(np.float32), uv, index=f.reshape(-1).astype(np.uint32))
    # 16 materials drawn like the mid scene's; each instance takes one.
    shade_scene = S.Scene()
    for k in range(16):
        kind = rng.uniform()
        if kind < 0.4:
            material: S.Material = S.MeshStandardMaterial(roughness=float(rng.uniform(0, 1)),
                                                          metalness=float(rng.uniform(0, 1)))
        elif kind < 0.7:
            material = S.MeshPhysicalMaterial(transmission=1.0, ior=1.5, roughness=float(rng.uniform(0, 0.2)))
        else:
            material = S.MeshPhongMaterial(shininess=float(rng.uniform(1, 200)))
        material.color = _srgb_color(rng.uniform(0.2, 1.0, 3))
        if rng.uniform() < 0.5:
            tex = S.DataTexture(noise_texture(256, seed + 1000 + k), 256, 256)
            tex.color_space = S.SRGBColorSpace
            tex.wrap_s = tex.wrap_t = S.RepeatWrapping
            material.map = tex
        holder = S.Mesh(S.BufferGeometry(np.zeros((3, 3), np.float32)), material)
        shade_scene.add(holder)
    half = box / 2
    for sx, sz in ((-1, -1), (-1, 1), (1, -1), (1, 1)):
        light = S.PointLight(0xffffff, 2500.0 * (box / 80.0) ** 2, 0, 2)
        light.position.set(sx * half * 0.5, half * 1.2, sz * half * 0.5)
        shade_scene.add(light)
    shade_scene.add(S.HemisphereLight(0xddeeff, 0x202020, 0.5))
    shading, _ = compile_shading(shade_scene)
    from .types import CompiledScene

    compiled = CompiledScene(None, shading.materials, shading.textures, shading.environments,  # type: ignore[arg-type]
                             shading.lights, shading.background, shading.environment, shading.fog)
    materials = rng.integers(0, len(shading.materials), count)
    camera = S.PerspectiveCamera(50, width / height, 0.1, 4000)
    camera.position.set(0, box * 0.35, box * 1.6)
    camera.look_at(0, 0, 0)
    camera.update_matrix_world()
    tris = count * f.shape[0]
    return InstancedScene(f"large: {count} icospheres x {f.shape[0]:,} tris = {tris:,} tris, rigid transforms "
                          f"re-drawn per frame in a {box:g}^3 box, {width}x{height}, {samples} spp, GI on, 8 bounces",
                          mesh, compiled, materials, camera, width, height,
                          {"samples": samples, "global_illumination": True, "max_bounces": 8,
                           "tone_mapping": S.ACESFilmicToneMapping, "output_color_space": "srgb"}, count, box, seed)
