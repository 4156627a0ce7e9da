"""Per-pixel parity of shading branches with the oracle, and the reference's exact
texture-sampling answers.

Each case renders one small scene at 1 sample with GI off (deterministic), on
the oracle and through the C ABI on the GPU, and compares every pixel: the
RGBA8 bytes within one level (the parity bar for deterministic
renders), and the Float32 sample sums (tone-mapped, premultiplied RGBA, as
encodeTile accumulates them, src/progressive.ts:288-313) within a float
tolerance on at least 99 % of pixels (the GPU computes in FP32, the oracle in
FP64 as the reference does).

Branches: cube-map backgrounds and reflections (sampleEnvironment's cube face
selection with flipX, src/textures.ts:300-313, compiled as addEnvironment
does, src/textures.ts:171-189), the Toon material (src/tracer.ts:380-389),
every tone mapping at exposure 1.5 (src/color.ts:81-136), and texture
sampling with repeat, clamp and mirrored wrapping, uv transforms, flipY, and
8-bit sRGB, half-float and float texels (src/textures.ts:229-281).

The exact answers are those of tests/compile.test.ts:154-200 (repeat 2 on u
lands on texel centres; a half-float texel reads back exactly), rendered
through a Basic material so that each pixel is one texture sample.
"""
import math

import numpy as np
import pytest

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200.compile import compile_camera
from meercadraytracer_b200.raytrace import as_options, output_srgb, sample_count, trace_settings
from oracle import cpu

from helpers import compile_with_oracle, top_camera

FLOAT_TOL = 2e-4  # absolute + relative, per channel, on the float sums
FLOAT_SHARE = 0.99


@pytest.fixture(scope="module")
def gpu():
    from meercadraytracer_b200.executors import GpuExecutor

    ex = GpuExecutor(0)
    yield ex
    ex.dispose()


def _pixels(width, height):
    idx = np.arange(width * height)
    return (idx % width).astype(np.int32), (idx // width).astype(np.int32)


def _render(impl, scene, camera, width, height, options, gpu=None):
    opts = {"output_color_space": "srgb-linear", "samples": 1}
    opts.update(options or {})
    o = as_options(opts)
    compiled = compile_with_oracle(scene, o.filter)
    cam = compile_camera(camera)
    st, spp, srgb = trace_settings(o), sample_count(o), output_srgb(o)
    px, py = _pixels(width, height)
    if impl == "oracle":
        return cpu.render_pixels(compiled, cam, st, width, height, spp, srgb, px, py, threads=4)
    return gpu.render_pixels(compiled, cam, width, height, st, spp, srgb, px, py)


def assert_same(gpu, scene, camera, width=32, height=32, options=None, min_signal=0.02):
    o_rgba, o_sum = _render("oracle", scene, camera, width, height, options)
    g_rgba, g_sum = _render("gpu", scene, camera, width, height, options, gpu)
    assert np.abs(o_sum[:, :3]).max() > min_signal, "the scene renders (nearly) black: nothing is compared"
    d8 = np.abs(g_rgba.astype(np.int32) - o_rgba.astype(np.int32))
    assert d8.max() <= 1, (int(d8.max()), int((d8.max(axis=1) > 1).sum()))
    df = np.abs(g_sum.astype(np.float64) - o_sum.astype(np.float64))
    ok = (df <= FLOAT_TOL * (1 + np.abs(o_sum))).all(axis=1)
    assert ok.mean() >= FLOAT_SHARE, (float(ok.mean()), float(df.max()))
    return o_sum, g_sum


# ----------------------------------------------------------------- environments
def _cube(kind):
    """Six 4 x 4 faces, each its own colour ramp, so a wrong face or a mirrored
    coordinate changes the pixel."""
    rng = np.random.default_rng(17)
    faces = []
    for f in range(6):
        base = np.array([(f + 1) % 2, (f // 2) % 2, (f // 4) % 2 + 0.2 * f, 1.0])
        ramp = rng.uniform(0.2, 1.0, (4, 4, 1))
        img = np.concatenate([np.clip(base[:3] * ramp + 0.1, 0, 1), np.ones((4, 4, 1))], axis=2)
        if kind == "u8":
            faces.append(np.round(img * 255).astype(np.uint8).reshape(-1))
        else:
            faces.append((img * 1.5).astype(np.float32).reshape(-1))
    cube = S.CubeTexture(faces, 4, 4)
    if kind == "u8":
        cube.color_space = S.SRGBColorSpace
    return cube


def _wide_camera(target):
    camera = S.PerspectiveCamera(110, 1, 0.1, 100)
    camera.position.set(0, 0, 0)
    camera.look_at(*target)
    camera.update_matrix_world()
    return camera


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["u8", "float"])
@pytest.mark.parametrize("target", [(0, 0, -1), (0, 0, 1), (1, 0.2, 0), (-1, 0.1, 0.3), (0.1, 1, 0.2),
                                    (0.2, -1, 0.1)])
def test_cube_background_matches_oracle(gpu, kind, target):
    scene = S.Scene()
    scene.background = _cube(kind)
    scene.background_intensity = 0.8
    scene.background_rotation = S.Euler(0.3, -0.5, 0.2)
    assert_same(gpu, scene, _wide_camera(target), options={"tone_mapping": S.ACESFilmicToneMapping})


@pytest.mark.gpu
def test_cube_reflections_match_oracle(gpu):
    """A mirror sphere and a rough metal sphere lit by a cube scene.environment, and
    a Phong sphere whose own cube envMap mixes in (combine = Mix)."""
    scene = S.Scene()
    cube = _cube("float")
    scene.environment = cube
    scene.environment_rotation = S.Euler(0, 0.7, 0)
    scene.background = cube
    mirror = S.Mesh(S.sphere_geometry(0.9, 24, 16), S.MeshStandardMaterial(metalness=1, roughness=0))
    mirror.position.set(-1.1, 0, 0)
    rough = S.Mesh(S.sphere_geometry(0.9, 24, 16), S.MeshStandardMaterial(color=0xccaa88, metalness=0.5,
                                                                          roughness=0.4))
    rough.position.set(1.1, 0, 0)
    own = _cube("u8")
    phong = S.Mesh(S.sphere_geometry(0.6, 24, 16), S.MeshPhongMaterial(color=0x88ccff, env_map=own, reflectivity=0.6,
                                                                       combine=S.MixOperation))
    phong.material.env_map_rotation = S.Euler(0.4, 0, 0)
    phong.position.set(0, 1.2, -0.5)
    light = S.DirectionalLight(0xffffff, 2)
    light.position.set(1, 3, 2)
    scene.add(mirror, rough, phong, light)
    camera = S.PerspectiveCamera(50, 1, 0.1, 100)
    camera.position.set(0, 1, 6)
    camera.look_at(0, 0.3, 0)
    camera.update_matrix_world()
    assert_same(gpu, scene, camera, 48, 48, {"tone_mapping": S.ACESFilmicToneMapping, "max_bounces": 3})


def test_cube_environment_compiles_as_the_reference():
    """addEnvironment, src/textures.ts:164-197: six face textures, flipX for a cube
    that is not a render target, identity uv matrix, and one entry per (texture,
    version, intensity, rotation) however often it is used."""
    from meercadraytracer_b200.compile import compile_shading

    scene = S.Scene()
    cube = _cube("u8")
    scene.background = cube
    scene.environment = cube
    m = S.MeshStandardMaterial(env_map=cube)
    scene.add(S.Mesh(S.plane_geometry(), m))
    shading, _ = compile_shading(scene)
    assert len(shading.environments) == 1  # background, environment and envMap share it
    env = shading.environments[0]
    assert env.kind == "cube" and env.flip_x and len(shading.textures) == 6
    assert list(env.faces) == list(range(6))
    assert shading.background.kind == "environment" and shading.background.environment == 0
    assert shading.environment == 0 and shading.materials[0].env_map == 0
    assert all(t.srgb and t.matrix == (1, 0, 0, 0, 1, 0, 0, 0, 1) for t in shading.textures)
    scene.background_intensity = 2.0
    shading, _ = compile_shading(scene)
    # Materials, then the background, then scene.environment (compile.ts:484-496).
    assert len(shading.environments) == 2 and shading.background.environment == 1 and shading.environment == 0
    cube.is_render_target_texture = True
    cube.version += 1
    shading, _ = compile_shading(scene)
    assert not shading.environments[0].flip_x


def test_cube_lookup_selects_opengl_faces():
    """The oracle's cube lookup against the face-selection rule written out here:
    each axis direction reads the centre texel of its face (+x, -x, +y, -y, +z, -z)."""
    from meercadraytracer_b200.types import CompiledEnvironment, CompiledTexture

    textures = []
    for f in range(6):
        img = np.zeros((2, 2, 4), np.float32)
        img[..., 0] = f
        img[..., 3] = 1
        textures.append(CompiledTexture(2, 2, img.reshape(-1), False, False, 1001, 1001,
                                        (1, 0, 0, 0, 1, 0, 0, 0, 1)))
    env = CompiledEnvironment("cube", faces=tuple(range(6)), flip_x=False)
    for face, d in enumerate([(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]):
        assert cpu.sample_environment(env, textures, d)[0] == face
    flipped = CompiledEnvironment("cube", faces=tuple(range(6)), flip_x=True)
    assert cpu.sample_environment(flipped, textures, (1, 0, 0))[0] == 1


# ----------------------------------------------------------------------- toon
@pytest.mark.gpu
def test_toon_matches_oracle(gpu):
    """MeshToonMaterial: irradiance 0.7 below cosine 0.4 (half-Lambert 0.7), 1 above,
    including the unlit side, on a sphere lit from the side."""
    scene = S.Scene()
    ball = S.Mesh(S.sphere_geometry(1, 32, 16), S.MeshToonMaterial(color=0xff8040))
    light = S.DirectionalLight(0xffffff, 2)
    light.position.set(3, 1, 1)
    point = S.PointLight(0x4080ff, 8, 0, 2)
    point.position.set(-2, 2, 2)
    scene.add(ball, light, point, S.AmbientLight(0xffffff, 0.3))
    camera = S.PerspectiveCamera(40, 1, 0.1, 100)
    camera.position.set(0, 0, 4)
    camera.update_matrix_world()
    o, _ = assert_same(gpu, scene, camera, 40, 40)
    # Both irradiance steps show up: the sphere is not one flat colour.
    lit = o[o[:, 3] > 0, 0]
    assert len(np.unique(np.round(lit, 3))) > 3


# ---------------------------------------------------------------- tone mapping
TONE_MAPS = [S.LinearToneMapping, S.ReinhardToneMapping, S.CineonToneMapping, S.ACESFilmicToneMapping,
             S.AgXToneMapping, S.NeutralToneMapping]


@pytest.mark.gpu
@pytest.mark.parametrize("mapping", TONE_MAPS)
def test_tone_mapping_at_exposure_matches_oracle(gpu, mapping):
    """A Standard sphere under a strong light, so radiance spans dark to well above 1,
    tone mapped at exposure 1.5 and encoded to sRGB."""
    scene = S.Scene()
    ball = S.Mesh(S.sphere_geometry(1, 32, 16), S.MeshStandardMaterial(color=0xffeedd, roughness=0.35,
                                                                       metalness=0.2))
    light = S.PointLight(0xffffff, 60, 0, 2)
    light.position.set(2, 2, 3)
    scene.add(ball, light, S.HemisphereLight(0x8899ff, 0x332211, 0.6))
    camera = S.PerspectiveCamera(40, 1, 0.1, 100)
    camera.position.set(0, 0, 4)
    camera.update_matrix_world()
    opts = {"tone_mapping": mapping, "tone_mapping_exposure": 1.5, "output_color_space": "srgb"}
    assert_same(gpu, scene, camera, 40, 40, opts)


# -------------------------------------------------------------------- textures
def _rgba_grid():
    """A 4 x 4 RGBA8 texture of distinct colours and alphas."""
    rng = np.random.default_rng(23)
    return rng.integers(0, 256, (4, 4, 4)).astype(np.uint8).reshape(-1)


def _textured_plane(texture, alpha_map=None):
    scene = S.Scene()
    scene.add(S.Mesh(S.plane_geometry(2, 2), S.MeshBasicMaterial(map=texture, alpha_map=alpha_map,
                                                                 transparent=False)))
    return scene


def _texture(kind):
    if kind == "u8":
        return S.DataTexture(_rgba_grid(), 4, 4)
    if kind == "srgb":
        t = S.DataTexture(_rgba_grid(), 4, 4)
        t.color_space = S.SRGBColorSpace
        return t
    if kind == "float":
        rng = np.random.default_rng(29)
        return S.DataTexture(rng.uniform(0, 2, 4 * 4 * 4).astype(np.float32), 4, 4)
    rng = np.random.default_rng(31)
    halves = rng.uniform(0, 3, 4 * 4 * 4).astype(np.float16).view(np.uint16)
    return S.DataTexture(halves, 4, 4, S.RGBAFormat, S.HalfFloatType)


WRAPS = {"repeat": S.RepeatWrapping, "clamp": S.ClampToEdgeWrapping, "mirror": S.MirroredRepeatWrapping}


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["u8", "srgb", "float", "half"])
@pytest.mark.parametrize("wrap", ["repeat", "clamp", "mirror"])
def test_texture_sampling_matches_oracle(gpu, kind, wrap):
    """Bilinear filtering, each wrap mode on both axes, a uv transform (repeat, offset,
    rotation about a centre) and flipY; every pixel of the plane is one sample."""
    t = _texture(kind)
    t.wrap_s = t.wrap_t = WRAPS[wrap]
    t.repeat = [2.5, 1.75]
    t.offset = [0.3, -0.2]
    t.rotation = 0.4
    t.center = [0.5, 0.5]
    scene = _textured_plane(t)
    assert_same(gpu, scene, top_camera(), 37, 29, min_signal=0.01)
    t.flip_y = True
    assert_same(gpu, scene, top_camera(), 37, 29, min_signal=0.01)


@pytest.mark.gpu
def test_alpha_map_and_texture_alpha_match_oracle(gpu):
    """An alpha map (its green channel) times the map's alpha on a transparent Basic
    material: the coverage of the stochastic pass-through, at 16 samples."""
    t = _texture("u8")
    a = _texture("srgb")
    a.wrap_s = a.wrap_t = S.MirroredRepeatWrapping
    a.repeat = [3, 2]
    scene = S.Scene()
    scene.add(S.Mesh(S.plane_geometry(2, 2), S.MeshBasicMaterial(map=t, alpha_map=a, transparent=True)))
    assert_same(gpu, scene, top_camera(), 24, 24, {"samples": 16, "clear_color": (0.2, 0.4, 0.9),
                                                   "clear_alpha": 1})


# compile.test.ts:154-174, as pixels: a 2 x 2 plane seen by the top camera at 4 x 2
# pixels puts pixel (x, y) at uv ((x + 0.5) / 4, 1 - (y + 0.5) / 2).
IMPLS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


def _exact_render(impl, gpu_fixture, scene, width, height):
    if impl == "gpu":
        return _render("gpu", scene, top_camera(), width, height, None, gpu_fixture())[1]
    return _render("oracle", scene, top_camera(), width, height, None)[1]


@pytest.fixture
def lazy_gpu(request):
    return lambda: request.getfixturevalue("gpu")


@pytest.mark.parametrize("impl", IMPLS)
def test_repeat_transform_lands_on_texel_centres(impl, lazy_gpu):  # compile.test.ts:154-174
    data = np.array([255, 0, 0, 255, 0, 255, 0, 255, 0, 0, 255, 255, 255, 255, 255, 255], np.uint8)
    texture = S.DataTexture(data, 2, 2)
    texture.wrap_s = texture.wrap_t = S.RepeatWrapping
    texture.repeat = [2, 1]
    sums = _exact_render(impl, lazy_gpu, _textured_plane(texture), 4, 2)
    at = lambda x, y: sums[y * 4 + x, :3]  # noqa: E731
    assert np.allclose(at(0, 1), [1, 0, 0], atol=1e-5)  # uv (0.125, 0.25)
    assert np.allclose(at(2, 1), [1, 0, 0], atol=1e-5)  # uv (0.625, 0.25)
    assert np.allclose(at(1, 0), [1, 1, 1], atol=1e-5)  # uv (0.375, 0.75)


@pytest.mark.parametrize("impl", IMPLS)
def test_half_float_texel_reads_back_exactly(impl, lazy_gpu):  # compile.test.ts:190-199
    halves = np.array([0.25, 2, 4, 1], np.float16).view(np.uint16)
    texture = S.DataTexture(halves, 1, 1, S.RGBAFormat, S.HalfFloatType)
    sums = _exact_render(impl, lazy_gpu, _textured_plane(texture), 2, 2)
    assert np.allclose(sums, np.tile([0.25, 2, 4, 1], (4, 1)), rtol=0, atol=1e-6)
