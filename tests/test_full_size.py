"""Checks at the configurations' full sizes, through properties that do not need the oracle
to render a whole frame.

  * The mid scene (1,310,720 triangles): the GPU compile equals the oracle's compile
    triangle for triangle (mapped back to input order) with the same tree, and the camera
    rays' closest hits over a 1920x1080 frame agree with the oracle's on a random 16,384-pixel
    sample (disagreements must be shared-edge ties).
  * The full mid workload (1920x1080, 64 spp, GI on) renders byte for byte the same twice,
    and the batch engine's image of it is within one level of the plain path's.
  * Instanced geometry at 4,096,000 triangles (200 icospheres subdivided 5 times): the device
    flatten + compile equals the GPU compile of the host flatten, arrays and tree.
  * The per-frame rebuild workload's build (32 bins, leaves of 4) on a 4,096,000-triangle frame:
    the device tree equals the oracle's 32-bin tree of the same triangles, and camera rays of the
    2048 x 2048 frame hit what the oracle's hit on a 16,384-pixel sample.
"""
import numpy as np
import pytest

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200 import scenes
from meercadraytracer_b200.compile import compile_camera, compile_shading, flatten_meshes
from meercadraytracer_b200.raytrace import as_options, output_srgb, sample_count, trace_settings
from meercadraytracer_b200.types import CompiledScene
from oracle import cpu

pytestmark = pytest.mark.gpu


def canonical(bvh, order):
    """Every node as (axis, leaf set or child keys), bottom up: two trees are equal when
    their root keys are, whatever order their nodes are stored in."""
    nodes = bvh.nodes.reshape(-1, 3).astype(np.int64)
    key = [None] * nodes.shape[0]
    stack = [(0, False)]
    while stack:
        n, done = stack.pop()
        first, count, axis = nodes[n]
        if count > 0:
            key[n] = frozenset(order[first:first + count].tolist())
        elif done:
            key[n] = (int(axis), key[first], key[first + 1])
        else:
            stack += [(n, True), (first, False), (first + 1, False)]
    return key[0]


@pytest.fixture(scope="module")
def mid():
    from meercadraytracer_b200.executors import GpuExecutor

    b = scenes.mid_scene()
    shading, meshes = compile_shading(b.scene)
    ids = {id(m): i for i, m in enumerate(shading.material_objects)}
    sink = flatten_meshes(meshes, lambda m: ids.get(id(m), 0))
    ex = GpuExecutor(0)
    g = ex.compile_sink(sink)
    compiled = CompiledScene(g, shading.materials, shading.textures, shading.environments, shading.lights,
                             shading.background, shading.environment, shading.fog)
    yield b, sink, compiled, ex
    ex.dispose()


def test_mid_scene_compile_equals_oracle(mid):
    b, sink, compiled, ex = mid
    o = cpu.compile_sink(sink)
    g = compiled.geometry
    assert g.triangle_count == o.triangle_count == 1310720
    assert g.bvh.node_count == o.bvh.node_count
    inv_o, inv_g = np.argsort(o.order), np.argsort(g.order)
    for name, w in (("triangles", 9), ("normals", 9), ("uvs", 6), ("tangents", 4)):
        assert np.array_equal(getattr(o, name).reshape(-1, w)[inv_o], getattr(g, name).reshape(-1, w)[inv_g]), name
    assert g.epsilon == o.epsilon
    assert canonical(g.bvh, g.order) == canonical(o.bvh, o.order)


def test_mid_frame_primary_hits_match_oracle_on_a_sample(mid):
    b, sink, compiled, ex = mid
    cam = compile_camera(b.camera)
    rng = np.random.default_rng(5)
    idx = rng.choice(b.width * b.height, 16384, replace=False)
    px, py = (idx % b.width).astype(np.int32), (idx // b.width).astype(np.int32)
    o = cpu.trace_primary(compiled, cam, b.width, b.height, 3, 0, px, py, threads=8)
    g = ex.trace_primary(compiled, cam, b.width, b.height, 3, 0, px, py)
    same = g["tri"] == o["tri"]
    hit = o["tri"] >= 0
    diff = ~same
    ties = diff & (g["tri"] >= 0) & hit & (np.abs(g["t"] - o["t"]) <= 1e-5 * np.abs(o["t"]))
    assert same.mean() >= 0.9999 or (diff == ties).all(), (same.mean(), int(diff.sum()), int(ties.sum()))
    rel = np.abs(g["t"][hit & same] - o["t"][hit & same]) / o["t"][hit & same]
    assert hit.sum() > 2000 and rel.max() <= 1e-5  # about a quarter of the frame shows geometry


def test_mid_frame_is_deterministic_and_batched_within_one_level(mid):
    from meercadraytracer_b200.batch import BatchRenderer, RenderRequest

    b, sink, compiled, ex = mid
    o = as_options(b.options)
    st, spp, srgb = trace_settings(o), sample_count(o), output_srgb(o)
    cam = compile_camera(b.camera)
    first = ex.raytrace(compiled, cam, b.width, b.height, st, spp, srgb)
    again = ex.raytrace(compiled, cam, b.width, b.height, st, spp, srgb)
    assert np.array_equal(first, again)
    r = BatchRenderer(0, 1 << 22, 4 << 30)
    try:
        r.adopt(compiled, ex)
        img = r.render([RenderRequest(compiled, cam, b.width, b.height, st, spp, srgb=srgb)])[0]
        d = np.abs(img.astype(np.int16) - first.astype(np.int16))
        assert d.max() <= 1 and (d.reshape(-1, 4).max(axis=1) > 0).mean() < 1e-4
    finally:
        r.dispose()


def _large_frame_sink(big, instances):
    from meercadraytracer_b200.compile import TriangleSink

    parts = []
    for world, mesh, material, flags, side, flat in instances:
        m = S.Mesh(big.mesh, S.MeshStandardMaterial())
        m.cast_shadow = m.receive_shadow = True
        m.matrix_world = np.asarray(world, np.float64)
        parts.append(flatten_meshes([m], lambda _m, k=material: k))
    cat = lambda name: np.concatenate([getattr(p, name) for p in parts])  # noqa: E731
    return TriangleSink(cat("p"), cat("n"), cat("uv"), cat("colors"), cat("has_color"), cat("materials"),
                        cat("flags"), cat("sides"))


def test_rebuild_frame_with_32_bins_equals_oracle_tree_and_hits():
    from meercadraytracer_b200.executors import GpuExecutor

    big = scenes.large_scene(count=200)
    instances = big.frame(1)
    sink = _large_frame_sink(big, instances)
    assert sink.count == 200 * 20480
    o = cpu.compile_sink(sink, bins=32)
    ex = GpuExecutor(0)
    try:
        ex.upload_meshes([big.mesh])
        info, dev = ex.compile_instances(instances, bins=32, download=True)
        assert info["bins"] == 32 and dev.bvh.node_count == o.bvh.node_count
        assert canonical(dev.bvh, dev.order) == canonical(o.bvh, o.order)
        inv_o, inv_d = np.argsort(o.order), np.argsort(dev.order)
        assert np.array_equal(o.triangles.reshape(-1, 9)[inv_o], dev.triangles.reshape(-1, 9)[inv_d])
        cam = compile_camera(big.camera)
        rng = np.random.default_rng(9)
        idx = rng.choice(big.width * big.height, 16384, replace=False)
        px, py = (idx % big.width).astype(np.int32), (idx // big.width).astype(np.int32)
        scene_d = CompiledScene(dev, big.shading.materials, big.shading.textures, [], big.shading.lights,
                                big.shading.background, -1, None)
        scene_o = CompiledScene(o, big.shading.materials, big.shading.textures, [], big.shading.lights,
                                big.shading.background, -1, None)
        g = ex.trace_primary(scene_d, cam, big.width, big.height, 2, 0, px, py)
        r = cpu.trace_primary(scene_o, cam, big.width, big.height, 2, 0, px, py, threads=8)
        # Input-order triangle of each hit, -1 for a miss (int64: `order` is uint32).
        g_in = np.where(g["tri"] >= 0, dev.order.astype(np.int64)[np.maximum(g["tri"], 0)], -1)
        r_in = np.where(r["tri"] >= 0, o.order.astype(np.int64)[np.maximum(r["tri"], 0)], -1)
        same = g_in == r_in
        hit = r_in >= 0
        ties = ~same & (g_in >= 0) & hit & (np.abs(g["t"] - r["t"]) <= 1e-5 * np.abs(r["t"]))
        assert same.mean() >= 0.9999 or (~same == ties).all(), (same.mean(), int((~same).sum()), int(ties.sum()))
        rel = np.abs(g["t"][hit & same] - r["t"][hit & same]) / r["t"][hit & same]
        assert hit.sum() > 1000 and rel.max() <= 1e-5
    finally:
        ex.dispose()


def test_instanced_compile_at_four_million_triangles_equals_host_flatten():
    from meercadraytracer_b200.executors import GpuExecutor

    big = scenes.large_scene(count=200, width=64, height=64)
    instances = big.frame(0)
    meshes = []
    for world, mesh, material, flags, side, flat in instances:
        m = S.Mesh(big.mesh, S.MeshStandardMaterial())
        m.cast_shadow = m.receive_shadow = True
        m.matrix_world = np.asarray(world, np.float64)
        meshes.append((m, material))
    parts = [flatten_meshes([m], lambda _m, k=k: k) for m, k in meshes]
    from meercadraytracer_b200.compile import TriangleSink

    cat = lambda name: np.concatenate([getattr(p, name) for p in parts])  # noqa: E731
    sink = TriangleSink(cat("p"), cat("n"), cat("uv"), cat("colors"), cat("has_color"), cat("materials"),
                        cat("flags"), cat("sides"))
    assert sink.count == 200 * 20480
    ex = GpuExecutor(0)
    try:
        host = ex.compile_sink(sink)
        ex.upload_meshes([big.mesh])
        info, dev = ex.compile_instances(instances, bins=16, download=True)
        for name in ("triangles", "normals", "uvs", "tangents", "materials", "flags", "sides", "order"):
            assert np.array_equal(getattr(dev, name).view(np.uint8), getattr(host, name).view(np.uint8)), name
        assert np.array_equal(dev.bvh.nodes, host.bvh.nodes) and np.array_equal(dev.bvh.bounds, host.bvh.bounds)
        assert dev.epsilon == host.epsilon
    finally:
        ex.dispose()
