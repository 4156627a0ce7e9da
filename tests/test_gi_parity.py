"""Statistical parity of path-traced (GI on) renders with the oracle.

Criterion: a GPU render at S samples per pixel lies within 1.05x the
oracle's own RMSE at the same S, both measured against a 4096-spp mean from
the oracle (a different seed, so the reference mean is independent of the
S-spp samples). Renders are compared as float means of the per-sample
tone-mapped premultiplied RGBA (the accumulation sums of encodeTile,
src/progressive.ts:288-313) on a seeded subset of pixels; the S-spp renders
use the same seed on both sides, as the reference's own determinism tests
do (tests/render.test.ts:321-327).

Scenes: the small scene with GI turned on (ground bounce, metal and rough
spheres, directional + point light), a reduced mid scene (6 x 6 displaced
icospheres, Standard / transmissive Physical / Phong materials, noise albedo
maps, 4 point lights + hemisphere light), camera moved in, and the mid scene
itself at its benchmarked size (1,310,720 triangles, 1920 x 1080, GI on,
4 bounces, ACES, sRGB) on 1024 seeded pixels whose camera ray hits geometry.
"""
import os

import numpy as np
import pytest

from meercadraytracer_b200 import scenes
from meercadraytracer_b200.compile import compile_camera, compile_scene
from meercadraytracer_b200.executors import GpuExecutor
from meercadraytracer_b200.raytrace import as_options, trace_settings
from oracle import cpu

pytestmark = pytest.mark.gpu

REFERENCE_SPP = 4096
REFERENCE_SEED = 7919
SEED = 3
PIXELS = 1024
THREADS = os.cpu_count() or 8


@pytest.fixture(scope="module")
def gpu():
    ex = GpuExecutor(0)
    yield ex
    ex.dispose()


def _small():
    b = scenes.small_scene()
    b.options = dict(b.options, global_illumination=True, max_bounces=4)
    return b


def _mid_reduced():
    b = scenes.mid_scene(grid=6, subdivisions=2, width=160, height=90)
    b.camera.position.set(0, 10, 12)
    b.camera.look_at(0, 0, 0)
    b.camera.update_matrix_world()
    return b


@pytest.fixture(scope="module", params=["small_gi", "mid_reduced", "mid_full"])
def case(request):
    b = {"small_gi": _small, "mid_reduced": _mid_reduced, "mid_full": scenes.mid_scene}[request.param]()
    compiled = compile_scene(b.scene, builder=cpu.compile_sink)
    cam = compile_camera(b.camera)
    rng = np.random.default_rng(11)
    if request.param == "mid_full":
        # Three quarters of the 1080p frame is background: keep pixels whose
        # pass-0 camera ray hits a triangle.
        idx = rng.choice(b.width * b.height, 16 * PIXELS, replace=False)
        px, py = (idx % b.width).astype(np.int32), (idx // b.width).astype(np.int32)
        hit = cpu.trace_primary(compiled, cam, b.width, b.height, 0, 0, px, py, threads=THREADS)["tri"] >= 0
        keep = np.nonzero(hit)[0][:PIXELS]
        assert keep.size == PIXELS
        px, py = px[keep], py[keep]
    else:
        idx = rng.choice(b.width * b.height, PIXELS, replace=False)
        px, py = (idx % b.width).astype(np.int32), (idx // b.width).astype(np.int32)
    st_ref = trace_settings(as_options(b.options, seed=REFERENCE_SEED))
    _, sums = cpu.render_pixels(compiled, cam, st_ref, b.width, b.height, REFERENCE_SPP, True, px, py,
                                threads=THREADS)
    return b, compiled, cam, px, py, sums.astype(np.float64) / REFERENCE_SPP


def _rmse(a, b):
    return float(np.sqrt(np.mean((a[:, :3] - b[:, :3]) ** 2)))


@pytest.mark.parametrize("spp", [16, 64])
def test_gi_render_rmse_within_oracle_rmse(gpu, case, spp):
    b, compiled, cam, px, py, mean = case
    st = trace_settings(as_options(b.options, seed=SEED))
    _, g = gpu.render_pixels(compiled, cam, b.width, b.height, st, spp, True, px, py)
    _, o = cpu.render_pixels(compiled, cam, st, b.width, b.height, spp, True, px, py, threads=THREADS)
    g = g.astype(np.float64) / spp
    o = o.astype(np.float64) / spp
    rmse_gpu, rmse_oracle = _rmse(g, mean), _rmse(o, mean)
    assert rmse_oracle > 0 and np.isfinite(g).all()
    assert mean[:, :3].max() > 0.05  # the pixels do see lit geometry
    assert rmse_gpu <= 1.05 * rmse_oracle, (rmse_gpu, rmse_oracle)
