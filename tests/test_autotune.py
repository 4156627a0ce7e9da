"""The autotuner and the traversal variants it chooses between.

Every variant (threads per block, short-stack depth) must give byte-identical
images: the choice may change time, never results. CPU: the library lists its
variants without touching a GPU. GPU: renders with every variant, plain and
batched, and a tuning round trip through the cache.
"""
import numpy as np
import pytest

from meercadraytracer_b200 import _lib, autotune, scenes
from meercadraytracer_b200.compile import compile_camera, compile_scene
from meercadraytracer_b200.raytrace import as_options, trace_settings
from oracle import cpu


def test_variants_are_listed_without_a_gpu():
    v = _lib.traversal_variants()
    assert v[0] == (128, 4)  # the default: fastest on the mid scene
    assert len(set(v)) == len(v) and len(v) >= 4
    assert all(b % 32 == 0 and 0 < s < 104 for b, s in v)


@pytest.fixture(scope="module")
def small():
    b = scenes.small_scene()
    b.camera.aspect = 64 / 48
    gi = trace_settings(as_options({"global_illumination": True, "max_bounces": 4,
                                    "tone_mapping": b.options["tone_mapping"]}))
    return compile_scene(b.scene, builder=cpu.compile_sink), compile_camera(b.camera), gi


@pytest.mark.gpu
def test_every_variant_renders_the_same_bytes(small):
    from meercadraytracer_b200.executors import GpuExecutor

    scene, cam, st = small
    ex = GpuExecutor(0)
    try:
        ex.set_capacity(4096)  # several chunks and bounces per render
        ref = ex.raytrace(scene, cam, 64, 48, st, 3, True)
        for b, s in _lib.traversal_variants():
            ex.set_traversal(b, s)
            assert np.array_equal(ex.raytrace(scene, cam, 64, 48, st, 3, True), ref), (b, s)
        with pytest.raises(_lib.McrtError):
            ex.set_traversal(96, 5)
    finally:
        ex.dispose()


@pytest.mark.gpu
def test_every_variant_batches_the_same_bytes(small):
    from meercadraytracer_b200.batch import BatchRenderer, RenderRequest

    scene, cam, st = small
    reqs = [RenderRequest(scene, cam, 64, 48, st, 3), RenderRequest(scene, cam, 40, 30, st, 2)]
    r = BatchRenderer(capacity=5000, memory_budget=16 << 20)
    try:
        ref = r.render(reqs)
        for b, s in _lib.traversal_variants():
            r.set_traversal(b, s)
            out = r.render(reqs)
            assert all(np.array_equal(x, y) for x, y in zip(out, ref)), (b, s)
    finally:
        r.dispose()


@pytest.mark.gpu
def test_tune_plain_picks_a_variant_and_caches_it(small, tmp_path):
    from meercadraytracer_b200.executors import GpuExecutor

    scene, cam, st = small
    ex = GpuExecutor(0)
    path = str(tmp_path / "tune.json")
    try:
        c = autotune.tune_plain(ex, scene, cam, st, 64, 48, 2, capacities=(4096, 1 << 14), key="t", cache_path=path)
        assert (c.block, c.stack) in _lib.traversal_variants() and c.capacity in (4096, 1 << 14)
        assert len(c.timings) == len(_lib.traversal_variants()) + 2
        autotune._memory.clear()
        again = autotune.tune_plain(ex, scene, cam, st, 64, 48, 2, key="t", cache_path=path)
        assert again == c
    finally:
        ex.dispose()
