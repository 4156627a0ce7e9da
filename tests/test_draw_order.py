"""The order of the path loop's random draws, pinned site by site.

Each sample takes its random numbers from one xorshift32 generator seeded from
(pixel, pass, seed) (src/random.ts:2-31, Tracer.renderTile src/tracer.ts:69-78)
in a fixed order: the transparency test (tracer.ts:170), the GI-off
environment estimate's cosine direction (tracer.ts:343-344, 601), the
continuation pick (tracer.ts:420), the diffuse cosine direction (tracer.ts:455)
or the GGX half vector (tracer.ts:610-612), and Russian roulette from the
third bounce (tracer.ts:465-467).

With the same seed on both sides, a 1-sample render of a path-traced scene
gives the GPU the same sample as the oracle for every path on which no
floating-point comparison flips (the GPU computes in FP32, the oracle in FP64).
So the GPU's per-pixel samples must agree with the oracle's on at least
AGREE of the pixels, within a float tolerance.

The CPU half shows that this comparison catches a wrong order: each mistake
planted in the oracle (one per draw site: a swapped pair, an extra draw, or
roulette a bounce early) drops the agreement between the mistaken and the
correct oracle below CAUGHT on at least one of the two renders (GI on and
GI off).
"""
import math

import numpy as np
import pytest

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200.compile import compile_camera
from meercadraytracer_b200.raytrace import as_options, trace_settings
from oracle import cpu

from helpers import compile_with_oracle

AGREE = 0.99
CAUGHT = 0.9
TOL = 2e-3  # absolute + relative, per channel of the tone-mapped sample
WIDTH, HEIGHT = 64, 48
SEEDS = (0, 12345, 777)


def draw_scene(gi: bool):
    """A corner of a room (a rough dielectric floor and two matte walls, so paths
    take several bounces and roulette plays), a rough metal sphere (GGX draws), a
    plastic sphere (GGX or diffuse pick), a large see-through sphere near the
    camera (transparency draws), a bright, graded equirectangular environment
    through the open sides, so every direction drawn shows in the sample, and a
    shadowing sun; GI on with 6 bounces, or GI off (environment estimate)."""
    scene = S.Scene()
    floor = S.Mesh(S.plane_geometry(12, 12), S.MeshStandardMaterial(color=S.Color(0.75, 0.7, 0.6), roughness=0.6,
                                                                    metalness=0))
    floor.rotation.x = -math.pi / 2
    back = S.Mesh(S.plane_geometry(12, 8), S.MeshLambertMaterial(color=S.Color(0.8, 0.8, 0.8)))
    back.position.set(0, 4, -4)
    side = S.Mesh(S.plane_geometry(12, 8), S.MeshLambertMaterial(color=S.Color(0.8, 0.5, 0.4)))
    side.rotation.y = math.pi / 2
    side.position.set(-4, 4, 0)
    metal = S.Mesh(S.sphere_geometry(1.2, 32, 16), S.MeshStandardMaterial(color=0xddccaa, metalness=1,
                                                                          roughness=0.45))
    metal.position.set(-1.8, 1.2, -1.5)
    plastic = S.Mesh(S.sphere_geometry(1, 32, 16), S.MeshStandardMaterial(color=0x3366cc, metalness=0,
                                                                          roughness=0.3))
    plastic.position.set(1.2, 1, -1.8)
    veil = S.Mesh(S.sphere_geometry(1.3, 32, 16), S.MeshLambertMaterial(color=0x44cc66, transparent=True,
                                                                        opacity=0.5))
    veil.position.set(0.6, 1.3, 1.6)
    sun = S.DirectionalLight(0xffffff, 2.5)
    sun.position.set(4, 8, 3)
    sun.cast_shadow = True
    for m in (floor, back, side, metal, plastic, veil):
        m.cast_shadow = m.receive_shadow = True
    scene.add(floor, back, side, metal, plastic, veil, sun)
    # Graded and grainy (seeded noise per texel), so a different direction drawn
    # almost always reads a different radiance.
    h, w = 32, 64
    y = np.linspace(1, 0, h)[:, None, None]
    x = np.linspace(0, 1, w)[None, :, None]
    grain = np.random.default_rng(41).uniform(0.6, 1.4, (h, w, 3))
    sky = np.concatenate([(0.2 + 2.5 * y * np.ones_like(x)) * grain[..., :1],
                          (0.3 + 2.0 * x * np.ones_like(y)) * grain[..., 1:2],
                          (0.8 + 1.5 * y * x) * grain[..., 2:], np.ones((h, w, 1))], axis=2)
    env = S.DataTexture(sky.astype(np.float32).reshape(-1), w, h)
    env.mapping = S.EquirectangularReflectionMapping
    scene.environment = env
    camera = S.PerspectiveCamera(60, WIDTH / HEIGHT, 0.1, 100)
    camera.position.set(2.5, 3.0, 6.5)
    camera.look_at(-0.5, 1.2, -1)
    camera.update_matrix_world()
    options = {"global_illumination": gi, "max_bounces": 6, "tone_mapping": S.ACESFilmicToneMapping}
    return scene, camera, options


def _prepared(gi):
    scene, camera, options = draw_scene(gi)
    return compile_with_oracle(scene), compile_camera(camera), options


def _pixels():
    idx = np.arange(WIDTH * HEIGHT)
    return (idx % WIDTH).astype(np.int32), (idx // WIDTH).astype(np.int32)


def oracle_samples(compiled, cam, options, seed, mistake=0):
    px, py = _pixels()
    st = trace_settings(as_options(options, seed=seed))
    cpu.plant_draw_mistake(mistake)
    try:
        return cpu.render_pixels(compiled, cam, st, WIDTH, HEIGHT, 1, False, px, py, threads=8)[1]
    finally:
        cpu.plant_draw_mistake(0)


def agreement(a, b):
    a, b = a.astype(np.float64), b.astype(np.float64)
    return float((np.abs(a - b) <= TOL * (1 + np.abs(b))).all(axis=1).mean())


@pytest.fixture(scope="module", params=[True, False], ids=["gi_on", "gi_off"])
def prepared(request):
    return request.param, _prepared(request.param)


def test_planted_draw_mistakes_are_caught():
    seed = SEEDS[1]
    renders = [_prepared(gi) for gi in (True, False)]
    right = [oracle_samples(c, cam, o, seed) for c, cam, o in renders]
    for (c, cam, o), r in zip(renders, right):
        assert agreement(oracle_samples(c, cam, o, seed), r) == 1.0  # deterministic
    for mistake in range(1, 7):
        scores = [agreement(oracle_samples(c, cam, o, seed, mistake), r) for (c, cam, o), r in zip(renders, right)]
        assert min(scores) < CAUGHT, (mistake, scores)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", SEEDS)
def test_gpu_samples_follow_the_oracle_draw_for_draw(prepared, seed):
    from meercadraytracer_b200.executors import GpuExecutor

    gi, (compiled, cam, options) = prepared
    right = oracle_samples(compiled, cam, options, seed)
    px, py = _pixels()
    st = trace_settings(as_options(options, seed=seed))
    ex = GpuExecutor(0)
    try:
        _, g = ex.render_pixels(compiled, cam, WIDTH, HEIGHT, st, 1, False, px, py)
    finally:
        ex.dispose()
    assert np.abs(right[:, :3]).max() > 0.1
    assert agreement(g, right) >= AGREE, agreement(g, right)
