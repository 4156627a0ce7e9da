"""Path order and pool size do not change images.

A frame's paths run pixel-major, in chunks of every pass of as many pixels as
the path pool holds; a pool smaller than a pixel's passes splits those passes
over chunks. Each pixel's passes still reach its Float32 running sum in pass
order (writeTile, src/progressive.ts:288-313), so the image must be the same
bytes whatever the pool: checked with pools that hold a few pixels' passes,
and one smaller than a single pixel's passes.

Camera rays take the warp-coherent walk where a warp's rays (passes of one
pixel) span at most 1/360 of the image height; its closest hits are the
per-lane walk's but for the order among equal-distance hits. A tall, narrow
image at 32 passes takes it and is compared with the oracle pixel by pixel
(deterministic: GI off), at the parity bar for deterministic renders.
"""
import numpy as np
import pytest

from meercadraytracer_b200 import scenes
from meercadraytracer_b200.compile import compile_camera, compile_scene
from meercadraytracer_b200.raytrace import as_options, output_srgb, trace_settings
from oracle import cpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    b = scenes.small_scene()
    return compile_scene(b.scene, builder=cpu.compile_sink), b.camera, as_options(b.options)


def _render(ex, compiled, camera, width, height, options, samples):
    cam = compile_camera(camera, aspect=width / height)
    return ex.raytrace(compiled, cam, width, height, trace_settings(options), samples, output_srgb(options))


@pytest.mark.parametrize("capacity,samples", [(4096, 300), (1024, 2500)])
def test_small_pools_give_the_same_bytes(small, capacity, samples):
    # 4096 paths hold 13 pixels' 300 passes per chunk; 1024 paths hold fewer
    # passes than one pixel has, so each pixel's 2500 passes take three chunks.
    from meercadraytracer_b200.executors import GpuExecutor

    compiled, camera, o = small
    width, height = (12, 9) if samples < 1000 else (3, 2)
    ex = GpuExecutor(0)
    try:
        ref = _render(ex, compiled, camera, width, height, o, samples)
        ex.set_capacity(capacity)
        got = _render(ex, compiled, camera, width, height, o, samples)
        assert np.array_equal(got, ref)
    finally:
        ex.dispose()


def test_coherent_camera_walk_matches_the_oracle(small):
    # 4 x 720 at 32 passes: a warp's rays are one pixel's passes and span 1/720
    # of the height, so the camera rays take the warp-coherent walk.
    from meercadraytracer_b200.executors import GpuExecutor

    compiled, camera, o = small
    width, height, samples = 4, 720, 32
    ex = GpuExecutor(0)
    try:
        got = _render(ex, compiled, camera, width, height, o, samples)
        cam = compile_camera(camera, aspect=width / height)
        ref = cpu.raytrace_compiled(compiled, cam, width, height, trace_settings(o), samples, output_srgb(o),
                                    threads=8)
        d = np.abs(got.astype(np.int32) - ref.astype(np.int32)).reshape(-1, 4)
        assert (d <= 1).all(axis=1).mean() >= 0.999
    finally:
        ex.dispose()
