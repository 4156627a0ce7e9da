"""Bounds of the BVH walks reach the caller as errors.

The reference's walks have no bounds (src/bvh.ts:202-332 keeps an explicit
stack of 256 entries, and attenuateShadow, src/tracer.ts:557-594, keeps every
see-through hit in a growing list). The device walks keep a traversal stack
of bounded depth, a list of 64 distinct see-through hits per shadow ray, and
a step budget per query; reaching any of them ends the query without a fault
and sets a status bit, and the call then fails with MCRT_ERR_WALK
(WalkLimitError) instead of returning an image that may differ from the
reference's, as the reference's worker turns any failure into
{type: 'error'} (src/protocol.ts:101-104).

Each case makes one bound run out on a well-formed input (nothing faults or
waits), checks the error, then renders or traces a normal input on the same
executor to show the context is still usable.
"""
import math

import numpy as np
import pytest

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200._lib import MCRT_ERR_WALK, WalkLimitError
from meercadraytracer_b200.compile import compile_camera
from meercadraytracer_b200.raytrace import trace_settings
from meercadraytracer_b200.types import TRI_CAST_SHADOW, TRI_OPAQUE, TRI_RECEIVE_SHADOW, CompiledBvh, CompiledGeometry

from helpers import compile_with_oracle, floor, top_camera

pytestmark = pytest.mark.gpu


@pytest.fixture
def ex():
    from meercadraytracer_b200.executors import GpuExecutor

    e = GpuExecutor(0)
    yield e
    e.dispose()


def _plain_scene():
    """A grey Lambert floor of 4 x 4 quads (32 triangles, so the BVH root is an inner
    node) under a white sun straight above (tests/render.test.ts:10-18)."""
    scene = S.Scene()
    light = S.DirectionalLight(0xffffff, math.pi)
    light.position.set(0, 0, 10)
    scene.add(S.Mesh(S.plane_geometry(4, 4, 4, 4), S.MeshLambertMaterial(color=S.Color(0.5, 0.5, 0.5))), light)
    return compile_with_oracle(scene)


def _still_usable(ex):
    compiled = _plain_scene()
    img = ex.raytrace(compiled, compile_camera(top_camera()), 16, 16, trace_settings({}), 1, False)
    assert img.reshape(-1, 4)[8 * 16 + 8, 0] == 128  # 0.5 of a white light: tests/render.test.ts:10-18


def test_shadow_ray_through_more_than_64_see_through_layers_fails(ex):
    """70 fully open (opacity 0) transparent panels stacked along the sun's direction
    above the floor, out of the camera's view: each central floor pixel's shadow ray
    crosses all of them at distinct distances."""
    scene = S.Scene()
    sun = S.DirectionalLight(0xffffff, math.pi)
    sun.position.set(5, 0, 10)  # direction (1, 0, 2) / sqrt(5): x = z / 2 along a shadow ray from the centre
    scene.add(floor(S.MeshLambertMaterial(color=0xffffff)), sun)
    veil = S.MeshLambertMaterial(transparent=True, opacity=0.0)
    for k in range(70):
        z = 4 + 0.07 * k
        panel = S.Mesh(S.plane_geometry(1.2, 1.2), veil)
        panel.position.set(z / 2, 0, z)
        scene.add(panel)
    compiled = compile_with_oracle(scene)
    with pytest.raises(WalkLimitError) as err:
        ex.raytrace(compiled, compile_camera(top_camera()), 16, 16, trace_settings({}), 1, False)
    assert err.value.code == MCRT_ERR_WALK and "see-through" in str(err.value)
    assert ex.stats()["status"] & 2
    _still_usable(ex)


def _chain_geometry(depth: int) -> CompiledGeometry:
    """A valid BVH that is a chain `depth` inner nodes deep: inner node k has leaf k
    (one triangle in the plane z = k + 0.25) as left child and inner node k + 1 as
    right child, children adjacent as the reference lays them out (src/types.ts:158-167).
    A ray coming down the z axis enters each right child (whose box reaches the top)
    before its left leaf, so a walk pushes one leaf per level."""
    n = depth + 1
    z = np.arange(n, dtype=np.float64) + 0.25
    tris = np.zeros((n, 9), np.float32)
    tris[:, 0:3] = np.stack([-1 + 0 * z, -1 + 0 * z, z], axis=1)
    tris[:, 3:6] = (3, 0, 0)
    tris[:, 6:9] = (0, 3, 0)
    m = 2 * depth + 1
    nodes = np.zeros((m, 3), np.int32)
    bounds = np.zeros((m, 6), np.float32)

    def box(lo, hi):
        return [-1, -1, z[lo], 2, 2, z[hi]]

    for k in range(depth):
        inner = 0 if k == 0 else 2 * k
        nodes[inner] = (2 * k + 1, 0, 2)
        bounds[inner] = box(k, n - 1)
        nodes[2 * k + 1] = (k, 1, 0)  # leaf k
        bounds[2 * k + 1] = box(k, k)
    nodes[2 * depth] = (depth, 1, 0)  # the last inner node's right child is leaf `depth`
    bounds[2 * depth] = box(depth, depth)
    flags = np.full(n, TRI_OPAQUE | TRI_CAST_SHADOW | TRI_RECEIVE_SHADOW, np.uint8)
    return CompiledGeometry(
        triangle_count=n, triangles=tris.reshape(-1), normals=np.tile([0, 0, 1], 3 * n).astype(np.float32),
        uvs=np.zeros(6 * n, np.float32), tangents=np.tile([1, 0, 0, 1], n).astype(np.float32),
        colors=np.zeros(0, np.float32), materials=np.zeros(n, np.uint32), flags=flags,
        sides=np.full(n, 2, np.uint8), bvh=CompiledBvh(bounds.reshape(-1), nodes.reshape(-1), m),
        epsilon=1e-4, order=np.arange(n, dtype=np.uint32))


def test_bvh_deeper_than_the_traversal_stack_fails(ex):
    # The walk pushes one entry per level of this chain: a thousand levels need
    # more than its 104 entries (the builder's trees are at most 100 deep).
    ex.send({"type": "geometry", "version": 1, "geometry": _chain_geometry(1000)})
    ray = np.array([[0.1, 0.1, 500, 0, 0, 0, -1, 0]], np.float32)
    with pytest.raises(WalkLimitError) as err:
        ex.intersect_closest(1, ray)
    assert "stack" in str(err.value)
    # A chain within the stack's reach is walked to its closest triangle (z = 100.25).
    ex.send({"type": "geometry", "version": 2, "geometry": _chain_geometry(100)})
    hit = ex.intersect_closest(2, ray)
    assert hit["tri"][0] == 100 and abs(hit["t"][0] - (500 - 100.25)) < 1e-3
    _still_usable(ex)


def test_step_budget_fails_the_call_and_resets(ex):
    compiled = _plain_scene()
    cam, st = compile_camera(top_camera()), trace_settings({})
    expect = ex.raytrace(compiled, cam, 16, 16, st, 1, False)
    ex.set_step_limit(1)  # the root is an inner node: every query needs at least two steps
    with pytest.raises(WalkLimitError) as err:
        ex.raytrace(compiled, cam, 16, 16, st, 1, False)
    assert "step budget" in str(err.value)
    ex.set_step_limit(0)
    assert np.array_equal(ex.raytrace(compiled, cam, 16, 16, st, 1, False), expect)
