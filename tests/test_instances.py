"""Instanced geometry compiled on the GPU (mcrt_upload_meshes, mcrt_compile_instances).

The device flatten must give exactly the arrays the host flatten (addMesh,
src/compile.ts:212-306, restated in compile.flatten_meshes) and the oracle's
compile give: float32 triangles, normals (normal matrix, Math.hypot),
uvs, tangents, materials, flags, sides and the epsilon, bit for bit, with
mirrored instances (winding swapped), flat shading and unindexed meshes
among them; its BVH must be the one the GPU builder makes from the host
flatten, and renders from it must equal renders from the uploaded geometry.
A wide build (nodes split by several blocks) must give the tree a single
block per node gives.
"""
import math

import numpy as np
import pytest

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200 import scenes
from meercadraytracer_b200.compile import compile_camera, flatten_meshes
from meercadraytracer_b200.raytrace import trace_settings
from meercadraytracer_b200.types import CompiledScene
from oracle import cpu

pytestmark = pytest.mark.gpu

TRI_OPAQUE, TRI_CAST, TRI_RECEIVE = 1, 2, 4


def canonical(bvh, order, node=0):
    """A node as a comparable value: leaves by their set of original triangle ids."""
    nodes = bvh.nodes.reshape(-1, 3)
    first, count, axis = (int(x) for x in nodes[node])
    if count > 0:
        return frozenset(int(order[k]) for k in range(first, first + count))
    return (axis, canonical(bvh, order, first), canonical(bvh, order, first + 1))


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _world(rng, mirror=False):
    m = np.eye(4)
    m[:3, :3] = _rotation(rng) * rng.uniform(0.5, 2.0)
    if mirror:
        m[:3, 0] *= -1
    m[:3, 3] = rng.uniform(-10, 10, 3)
    return m.T.reshape(16)  # column-major


def _setup(count=40, seed=3):
    rng = np.random.default_rng(seed)
    v, f = scenes.icosphere(2)
    sphere = S.BufferGeometry(v.astype(np.float32), v.astype(np.float32),
                              rng.uniform(0, 1, (v.shape[0], 2)).astype(np.float32),
                              index=f.reshape(-1).astype(np.uint32))
    box = S.box_geometry(1, 2, 0.5)
    # An unindexed copy of the box without normals: face normals.
    bi = np.asarray(box.index, np.int64)
    soup = S.BufferGeometry(np.asarray(box.position, np.float32).reshape(-1, 3)[bi], None,
                            np.asarray(box.uv, np.float32).reshape(-1, 2)[bi])
    geoms = [sphere, soup]
    instances, meshes = [], []
    mats = [S.MeshStandardMaterial(), S.MeshPhongMaterial(), S.MeshStandardMaterial(flat_shading=True)]
    for i in range(count):
        mesh_id = i % 2
        world = _world(rng, mirror=(i % 5 == 0))
        mat = i % 3
        flags = (TRI_OPAQUE | TRI_CAST | TRI_RECEIVE) if i % 4 else TRI_OPAQUE
        side = i % 3
        flat = mats[mat].flat_shading
        instances.append((world, mesh_id, mat, flags, side, flat))
        m = S.Mesh(geoms[mesh_id], mats[mat])
        m.cast_shadow = bool(flags & TRI_CAST)
        m.receive_shadow = bool(flags & TRI_RECEIVE)
        m.material.side = side
        m.matrix_world = np.asarray(world, np.float64)
        meshes.append((m, mat, side))
    return geoms, instances, meshes


def _host_sink(meshes):
    # The host flatten, one mesh at a time with the material index and side of its instance.
    parts = []
    for m, mat, side in meshes:
        material = S.MeshStandardMaterial(flat_shading=m.material.flat_shading)
        material.side = side
        mm = S.Mesh(m.geometry, material)
        mm.cast_shadow, mm.receive_shadow = m.cast_shadow, m.receive_shadow
        mm.matrix_world = m.matrix_world
        parts.append(flatten_meshes([mm], lambda _m, k=mat: k))
    cat = lambda name: np.concatenate([getattr(p, name) for p in parts])  # noqa: E731
    from meercadraytracer_b200.compile import TriangleSink

    return TriangleSink(cat("p"), cat("n"), cat("uv"), cat("colors"), cat("has_color"), cat("materials"),
                        cat("flags"), cat("sides"))


def test_device_flatten_equals_host_flatten_and_oracle():
    from meercadraytracer_b200.executors import GpuExecutor

    geoms, instances, meshes = _setup()
    sink = _host_sink(meshes)
    expect = cpu.compile_sink(sink)
    ex = GpuExecutor(0)
    try:
        gpu_host = ex.compile_sink(sink)
        ex.upload_meshes(geoms)
        info, got = ex.compile_instances(instances, bins=16, download=True)
        assert info["triangle_count"] == sink.count == got.triangle_count
        # Bit for bit the geometry the GPU compiles from the host flatten, tree and order included.
        for name in ("triangles", "normals", "uvs", "tangents", "materials", "flags", "sides", "order"):
            a, b = getattr(got, name), getattr(gpu_host, name)
            assert a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
        assert np.array_equal(got.bvh.bounds, gpu_host.bvh.bounds)
        assert np.array_equal(got.bvh.nodes, gpu_host.bvh.nodes)
        # And the oracle's per-triangle data, once both are mapped back to input order.
        inv_g, inv_o = np.argsort(got.order), np.argsort(expect.order)
        for name, w in (("triangles", 9), ("normals", 9), ("uvs", 6), ("tangents", 4), ("materials", 1),
                        ("flags", 1), ("sides", 1)):
            a = getattr(got, name).reshape(-1, w)[inv_g]
            b = getattr(expect, name).reshape(-1, w)[inv_o]
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), name
        assert got.epsilon == expect.epsilon
        assert info["levels"] > 1 and info["geometry_bytes"] > 0
    finally:
        ex.dispose()


def test_instanced_geometry_renders_like_uploaded_geometry():
    from meercadraytracer_b200.executors import GpuExecutor

    geoms, instances, meshes = _setup(count=30, seed=5)
    sink = _host_sink(meshes)
    compiled_geometry = cpu.compile_sink(sink)
    mats = [cpu_material for cpu_material in _materials()]
    light = S.DirectionalLight(0xffffff, 3)
    light.position.set(5, 10, 7)
    scene = S.Scene()
    scene.add(light, S.HemisphereLight(0xddeeff, 0x202020, 0.5))
    from meercadraytracer_b200.compile import compile_shading

    shading, _ = compile_shading(scene)
    compiled = CompiledScene(compiled_geometry, mats, [], [], shading.lights, shading.background, -1, None)
    cam_obj = S.PerspectiveCamera(50, 4 / 3, 0.1, 500)
    cam_obj.position.set(0, 8, 30)
    cam_obj.look_at(0, 0, 0)
    cam = compile_camera(cam_obj)
    st = trace_settings({"global_illumination": True, "max_bounces": 3})
    a = GpuExecutor(0)
    b = GpuExecutor(0)
    try:
        ref = a.raytrace(compiled, cam, 80, 60, st, 2, True)
        b.upload_meshes(geoms)
        info, _ = b.compile_instances(instances)
        sv = b.send_shading_only(compiled)
        img = b.raytrace_resident((info["version"], sv), cam, 80, 60, st, 2, True)
        assert np.array_equal(img, ref)
    finally:
        a.dispose()
        b.dispose()


def _materials():
    from meercadraytracer_b200.compile import TextureTable, compile_material

    t = TextureTable()
    return [compile_material(m, t) for m in (S.MeshStandardMaterial(color=S.Color(0.8, 0.3, 0.2), roughness=0.4),
                                             S.MeshPhongMaterial(color=S.Color(0.2, 0.6, 0.9), shininess=40),
                                             S.MeshStandardMaterial(color=S.Color(0.9, 0.9, 0.9), metalness=1,
                                                                    roughness=0.2))]


def test_wide_build_equals_the_single_block_build():
    # 80 icospheres subdivided 3 times: 102,400 triangles, so the top nodes (>= 32,768
    # triangles) are binned and partitioned by several blocks; the host-flatten path builds
    # the same triangles. With 16 bins (bvh.ts:3) and with the per-frame rebuild's 32, the
    # device tree is the oracle's tree for that bin count.
    from meercadraytracer_b200.executors import GpuExecutor

    rng = np.random.default_rng(11)
    v, f = scenes.icosphere(3)
    geo = S.BufferGeometry(v.astype(np.float32), v.astype(np.float32), None, index=f.reshape(-1).astype(np.uint32))
    instances, meshes = [], []
    for i in range(80):
        world = _world(rng)
        instances.append((world, 0, 0, TRI_OPAQUE, 0, False))
        m = S.Mesh(geo, S.MeshStandardMaterial())
        m.matrix_world = np.asarray(world, np.float64)
        meshes.append((m, 0, 0))
    sink = _host_sink(meshes)
    ex = GpuExecutor(0)
    try:
        ex.upload_meshes([geo])
        _, wide = ex.compile_instances(instances, bins=16, download=True)
        expect = cpu.compile_sink(sink)
        assert wide.bvh.node_count == expect.bvh.node_count
        assert canonical(wide.bvh, wide.order) == canonical(expect.bvh, expect.order)
        info32, g32 = ex.compile_instances(instances, bins=32, download=True)
        expect32 = cpu.compile_sink(sink, bins=32)
        assert info32["bins"] == 32 and g32.bvh.node_count == expect32.bvh.node_count
        assert canonical(g32.bvh, g32.order) == canonical(expect32.bvh, expect32.order)
        assert canonical(g32.bvh, g32.order) != canonical(wide.bvh, wide.order)  # the bin count matters
    finally:
        ex.dispose()
