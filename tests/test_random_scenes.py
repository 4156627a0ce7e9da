"""Seeded random scenes, rendered on the GPU and by the oracle, compared pixel for pixel.

Each scene draws meshes (spheres, boxes, subdivided planes) under random
transforms, some mirrored (negative scale, so the flatten flips their winding,
src/compile.ts:256-262); materials of every model (Basic, Lambert, Toon, Phong,
Standard, Physical with transmission and volume attenuation) with random
parameters and random maps (base colour, alpha, emissive, normal, ambient
occlusion, roughness, metalness) over 8-bit, sRGB and float texels with repeat,
clamp or mirrored wrapping and uv transforms; vertex colours, flat shading,
alpha test, stochastic transparency, front / back / double sides; lights of
every type (ambient, hemisphere, directional, point with a distance cutoff and
decay, spot with penumbra), some casting shadows, with every shadows mode;
linear or exp2 fog, a clear or background colour, an environment map, any
tone map and exposure, sRGB or linear output.

GI is off, so each render is deterministic on both sides (same seed, same
random draws): the RGBA8 images agree within one level on at least 99.9 % of
pixels (the parity bar for deterministic renders), and the float samples (tone-mapped,
premultiplied) within 2e-4 on at least 99 %.
"""
import math

import numpy as np
import pytest

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200.compile import compile_camera
from meercadraytracer_b200.raytrace import as_options, output_srgb, sample_count, trace_settings
from oracle import cpu

from helpers import compile_with_oracle

W, H = 64, 48
SEEDS = list(range(40))
TONE_MAPS = [S.NoToneMapping, S.LinearToneMapping, S.ReinhardToneMapping, S.CineonToneMapping,
             S.ACESFilmicToneMapping, S.AgXToneMapping, S.NeutralToneMapping]
WRAPS = [S.RepeatWrapping, S.ClampToEdgeWrapping, S.MirroredRepeatWrapping]


def _texture(rng, kind):
    n = int(rng.choice([2, 4, 8]))
    if kind == "float":
        t = S.DataTexture(rng.uniform(0, 1.5, n * n * 4).astype(np.float32), n, n)
    else:
        t = S.DataTexture(rng.integers(0, 256, n * n * 4).astype(np.uint8), n, n)
        if kind == "srgb":
            t.color_space = S.SRGBColorSpace
    t.wrap_s, t.wrap_t = WRAPS[int(rng.integers(3))], WRAPS[int(rng.integers(3))]
    t.repeat = [float(rng.uniform(0.5, 3)), float(rng.uniform(0.5, 3))]
    t.offset = [float(rng.uniform(-0.5, 0.5)), float(rng.uniform(-0.5, 0.5))]
    t.rotation = float(rng.uniform(-1, 1))
    t.flip_y = bool(rng.integers(2))
    return t


def _maybe(rng, p, kind=None):
    return _texture(rng, kind or str(rng.choice(["u8", "srgb", "float"]))) if rng.uniform() < p else None


def _material(rng):
    model = str(rng.choice(["basic", "lambert", "toon", "phong", "standard", "physical"]))
    color = S.Color(*rng.uniform(0.05, 1, 3))
    common = dict(color=color, map=_maybe(rng, 0.4), side=int(rng.choice([S.FrontSide, S.BackSide, S.DoubleSide])),
                  flat_shading=bool(rng.uniform() < 0.25))
    if rng.uniform() < 0.15:
        common.update(transparent=True, opacity=float(rng.uniform(0.2, 0.9)))
    if rng.uniform() < 0.15:
        common.update(alpha_map=_maybe(rng, 1.0, "u8"), alpha_test=float(rng.uniform(0.1, 0.6)))
    if model == "basic":
        return S.MeshBasicMaterial(**common)
    lit = dict(common, emissive=S.Color(*rng.uniform(0, 0.3, 3)), emissive_map=_maybe(rng, 0.2),
               ao_map=_maybe(rng, 0.2, "u8"), ao_map_intensity=float(rng.uniform(0, 1)))
    if model == "lambert":
        return S.MeshLambertMaterial(**lit)
    if model == "toon":
        return S.MeshToonMaterial(**lit)
    lit.update(normal_map=_maybe(rng, 0.3, "u8"), normal_scale=(float(rng.uniform(0.2, 1.5)),) * 2)
    if model == "phong":
        return S.MeshPhongMaterial(shininess=float(rng.uniform(1, 200)), specular=S.Color(*rng.uniform(0, 0.5, 3)),
                                   **lit)
    pbr = dict(lit, roughness=float(rng.uniform(0, 1)), metalness=float(rng.uniform(0, 1)),
               roughness_map=_maybe(rng, 0.2, "u8"), metalness_map=_maybe(rng, 0.2, "u8"))
    if model == "standard":
        return S.MeshStandardMaterial(**pbr)
    phys = dict(pbr, ior=float(rng.uniform(1.1, 2.0)), specular_intensity=float(rng.uniform(0.3, 1)))
    if rng.uniform() < 0.5:
        phys.update(transmission=1.0, metalness=0.0, roughness=float(rng.uniform(0, 0.3)),
                    thickness=float(rng.choice([0.0, 1.0])))
        if phys["thickness"] > 0:
            phys.update(attenuation_color=S.Color(*rng.uniform(0.3, 1, 3)),
                        attenuation_distance=float(rng.uniform(0.5, 3)))
    return S.MeshPhysicalMaterial(**phys)


def _geometry(rng):
    kind = int(rng.integers(3))
    if kind == 0:
        g = S.sphere_geometry(float(rng.uniform(0.4, 1.2)), int(rng.integers(8, 24)), int(rng.integers(6, 16)))
    elif kind == 1:
        g = S.box_geometry(*rng.uniform(0.4, 1.6, 3))
    else:
        g = S.plane_geometry(float(rng.uniform(1, 4)), float(rng.uniform(1, 4)), int(rng.integers(1, 4)),
                             int(rng.integers(1, 4)))
    if rng.uniform() < 0.25:
        count = np.asarray(g.position).reshape(-1, 3).shape[0]
        g.color = rng.uniform(0.2, 1, (count, 3)).astype(np.float32)
    return g


def random_scene(seed):
    rng = np.random.default_rng(0xC0FFEE + seed)
    scene = S.Scene()
    floor = S.Mesh(S.plane_geometry(12, 12), S.MeshLambertMaterial(color=S.Color(0.6, 0.6, 0.6)))
    floor.rotation.x = -math.pi / 2
    floor.position.y = -1.2
    floor.receive_shadow = True
    scene.add(floor)
    for _ in range(int(rng.integers(3, 7))):
        m = _material(rng)
        if m.vertex_colors is False and rng.uniform() < 0.5:
            m.vertex_colors = True
        mesh = S.Mesh(_geometry(rng), m)
        mesh.position.set(*rng.uniform([-2.5, -0.8, -2.5], [2.5, 1.5, 1.5]))
        mesh.rotation.x, mesh.rotation.y, mesh.rotation.z = rng.uniform(-math.pi, math.pi, 3)
        sc = rng.uniform(0.6, 1.4, 3) * np.where(rng.uniform(size=3) < 0.15, -1, 1)
        mesh.scale.set(*sc)
        mesh.cast_shadow = bool(rng.uniform() < 0.8)
        mesh.receive_shadow = bool(rng.uniform() < 0.8)
        scene.add(mesh)
    lights = []
    if rng.uniform() < 0.5:
        lights.append(S.AmbientLight(S.Color(*rng.uniform(0.3, 1, 3)), float(rng.uniform(0.1, 0.6))))
    if rng.uniform() < 0.5:
        hemi = S.HemisphereLight(S.Color(*rng.uniform(0.3, 1, 3)), S.Color(*rng.uniform(0, 0.4, 3)),
                                 float(rng.uniform(0.2, 1)))
        hemi.position.set(*rng.uniform(-1, 1, 3))
        lights.append(hemi)
    for _ in range(int(rng.integers(1, 4))):
        kind = int(rng.integers(3))
        if kind == 0:
            light = S.DirectionalLight(S.Color(*rng.uniform(0.5, 1, 3)), float(rng.uniform(1, 3)))
        elif kind == 1:
            light = S.PointLight(S.Color(*rng.uniform(0.5, 1, 3)), float(rng.uniform(10, 40)),
                                 float(rng.choice([0.0, rng.uniform(6, 15)])), float(rng.uniform(1, 2)))
        else:
            light = S.SpotLight(S.Color(*rng.uniform(0.5, 1, 3)), float(rng.uniform(20, 60)), 0.0,
                                float(rng.uniform(0.3, 0.9)), float(rng.uniform(0, 0.8)), 2.0)
            light.target.position.set(*rng.uniform(-1, 1, 3))
            scene.add(light.target)
        light.position.set(*rng.uniform([-5, 3, -3], [5, 8, 6]))
        light.cast_shadow = bool(rng.uniform() < 0.7)
        lights.append(light)
    scene.add(*lights)
    fog = rng.uniform()
    if fog < 0.2:
        scene.fog = S.Fog(S.Color(*rng.uniform(0, 1, 3)), float(rng.uniform(2, 6)), float(rng.uniform(8, 20)))
    elif fog < 0.35:
        scene.fog = S.FogExp2(S.Color(*rng.uniform(0, 1, 3)), float(rng.uniform(0.02, 0.12)))
    if rng.uniform() < 0.3:
        scene.background = S.Color(*rng.uniform(0, 1, 3))
    if rng.uniform() < 0.3:
        env = S.DataTexture(rng.uniform(0, 2, 8 * 4 * 4).astype(np.float32), 8, 4)
        env.mapping = S.EquirectangularReflectionMapping
        scene.environment = env
    camera = S.PerspectiveCamera(float(rng.uniform(40, 70)), W / H, 0.1, 100)
    camera.position.set(*rng.uniform([-3, 1.5, 6], [3, 4, 9]))
    camera.look_at(0, 0, 0)
    camera.update_matrix_world()
    options = {"samples": 2, "tone_mapping": TONE_MAPS[int(rng.integers(len(TONE_MAPS)))],
               "tone_mapping_exposure": float(rng.uniform(0.6, 1.8)),
               "output_color_space": str(rng.choice(["srgb", "srgb-linear"])),
               "shadows": str(rng.choice(["all", "castShadow", "none"])), "max_bounces": int(rng.integers(0, 5)),
               "clear_color": tuple(rng.uniform(0, 1, 3)), "clear_alpha": float(rng.choice([0.0, 1.0])),
               "seed": int(rng.integers(1 << 30))}
    return scene, camera, options


def _prepare(seed):
    scene, camera, options = random_scene(seed)
    o = as_options(options)
    compiled = compile_with_oracle(scene, o.filter)
    idx = np.arange(W * H)
    return (compiled, compile_camera(camera), trace_settings(o), sample_count(o), output_srgb(o),
            (idx % W).astype(np.int32), (idx // W).astype(np.int32))


@pytest.mark.parametrize("seed", SEEDS[:2])
def test_random_scene_renders_on_the_oracle_deterministically(seed):
    compiled, cam, st, spp, srgb, px, py = _prepare(seed)
    a = cpu.render_pixels(compiled, cam, st, W, H, spp, srgb, px, py, threads=4)
    b = cpu.render_pixels(compiled, cam, st, W, H, spp, srgb, px, py, threads=2)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert compiled.geometry.triangle_count > 2


@pytest.fixture(scope="module")
def gpu():
    from meercadraytracer_b200.executors import GpuExecutor

    ex = GpuExecutor(0)
    yield ex
    ex.dispose()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", SEEDS)
def test_random_scene_matches_oracle(gpu, seed):
    compiled, cam, st, spp, srgb, px, py = _prepare(seed)
    o_rgba, o_sum = cpu.render_pixels(compiled, cam, st, W, H, spp, srgb, px, py, threads=4)
    g_rgba, g_sum = gpu.render_pixels(compiled, cam, W, H, st, spp, srgb, px, py)
    d8 = np.abs(g_rgba.astype(np.int32) - o_rgba.astype(np.int32)).max(axis=1)
    assert (d8 <= 1).mean() >= 0.999, (float((d8 <= 1).mean()), int(d8.max()))
    df = np.abs(g_sum.astype(np.float64) - o_sum.astype(np.float64))
    ok = (df <= 2e-4 * (1 + np.abs(o_sum))).all(axis=1)
    assert ok.mean() >= 0.99, float(ok.mean())
