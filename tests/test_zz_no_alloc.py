"""mcrt_intersect_closest_noalloc against mcrt_intersect_closest, both called
through the C ABI.

The no-alloc entry point runs the same closest-hit kernel with its working
memory in the library's fixed per-device array, so results must be equal to
the allocating entry point's: tolerance zero (triangle, t, u and front
compared exactly). Two calls in a row with different ray lists check that the
shared array's leftover contents from the previous call never reach the next
one. This file is collected last and builds its own scene, so it passes alone
in a fresh process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from meercadraytracer_b200 import abi
from meercadraytracer_b200._lib import MCRT_ERR_LIMIT, NOALLOC_MAX_RAYS, McrtError, call
from meercadraytracer_b200.executors import GpuExecutor
from meercadraytracer_b200.types import CompiledGeometry
from oracle import cpu

from test_oracle_bvh_color import lcg_triangles, lissajous_ray, reorder

pytestmark = pytest.mark.gpu

VERSION = 1


@pytest.fixture(scope="module")
def ex():
    ex = GpuExecutor(0)
    count = 3000
    raw = lcg_triangles(count, 7)
    bvh, order = cpu.build_bvh(raw, count)
    data = reorder(raw, order)
    g = CompiledGeometry(count, data, np.zeros(count * 9, np.float32), np.zeros(count * 6, np.float32),
                         np.zeros(count * 4, np.float32), np.zeros(0, np.float32), np.zeros(count, np.uint32),
                         np.ones(count, np.uint8), np.full(count, 2, np.uint8), bvh, 1e-4, order)
    ex.send({"type": "geometry", "version": VERSION, "geometry": g})
    yield ex
    ex.dispose()


def seeded_rays(n: int, seed: int) -> np.ndarray:
    """Rays from a sphere of radius 30 towards points in the triangles' cube, as 8 floats each."""
    rng = np.random.default_rng(seed)
    o = rng.normal(size=(n, 3))
    o *= 30.0 / np.linalg.norm(o, axis=1, keepdims=True)
    d = rng.uniform(-8.0, 8.0, size=(n, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    return rays


def lissajous_rays() -> np.ndarray:
    rays = np.zeros((400, 8), np.float32)
    for i in range(400):
        o, d = lissajous_ray(i)
        rays[i, 0:3] = o
        rays[i, 4:7] = d
    return rays


def closest(ex: GpuExecutor, name: str, rays: np.ndarray, cull: int):
    """One call of `name` (mcrt_intersect_closest or its no-alloc variant) through the C ABI."""
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    tri = np.full(n, -7, np.int32)
    t = np.full(n, np.nan, np.float32)
    u = np.full(n, np.nan, np.float32)
    front = np.full(n, -7, np.int32)
    call(name, ex._h, VERSION, n, abi.ptr(rays, C.c_float), cull, abi.ptr(tri, C.c_int32),
         abi.ptr(t, C.c_float), abi.ptr(u, C.c_float), abi.ptr(front, C.c_int32))
    return tri, t, u, front


def assert_same(a, b):
    for field, x, y in zip(("triangle", "t", "u", "front"), a, b):
        assert np.array_equal(x, y, equal_nan=True), (field, np.nonzero(x != y)[0][:10])


@pytest.mark.parametrize("cull", [1, 0])
def test_noalloc_matches_closest_on_two_calls_in_a_row(ex, cull):
    first = seeded_rays(20000, 5)
    second = np.concatenate([lissajous_rays(), seeded_rays(1000, 6)])  # shorter: leftovers must not leak
    a1 = closest(ex, "mcrt_intersect_closest_noalloc", first, cull)
    a2 = closest(ex, "mcrt_intersect_closest_noalloc", second, cull)
    b1 = closest(ex, "mcrt_intersect_closest", first, cull)
    b2 = closest(ex, "mcrt_intersect_closest", second, cull)
    assert_same(a1, b1)
    assert_same(a2, b2)
    assert (a1[0] >= 0).sum() > 1000 and (a2[0] >= 0).sum() > 100  # the rays do hit the scene
    assert ex.stats()["status"] == 0


def test_noalloc_at_its_limit(ex):
    rays = seeded_rays(NOALLOC_MAX_RAYS, 8)
    assert_same(closest(ex, "mcrt_intersect_closest_noalloc", rays, 1),
                closest(ex, "mcrt_intersect_closest", rays, 1))


def test_noalloc_rejects_more_rays_than_its_limit(ex):
    rays = seeded_rays(NOALLOC_MAX_RAYS + 1, 9)
    with pytest.raises(McrtError) as err:
        closest(ex, "mcrt_intersect_closest_noalloc", rays, 1)
    assert err.value.code == MCRT_ERR_LIMIT
    assert str(NOALLOC_MAX_RAYS) in str(err.value)


def test_noalloc_empty_call_and_executor_method(ex):
    empty = np.zeros((0, 8), np.float32)
    assert all(x.size == 0 for x in closest(ex, "mcrt_intersect_closest_noalloc", empty, 1))
    rays = lissajous_rays()
    got = ex.intersect_closest_noalloc(VERSION, rays)
    want = ex.intersect_closest(VERSION, rays)
    for key in ("tri", "t", "u", "front"):
        assert np.array_equal(got[key], want[key]), key
