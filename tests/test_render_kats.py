"""Known-answer render tests restated from the reference's tests/render.test.ts.

Each scene and expected value follows the reference test it cites (closed-form
three.js shading, 1 sample, linear output, tolerance ONE_LEVEL). Every test
runs twice: on the oracle (pins the oracle to the reference's own expected
values) and on the CUDA path through the C-ABI (marked gpu).
"""
import math

import pytest

from meercadraytracer_b200 import scene as S
from oracle import cpu

from helpers import ONE_LEVEL, centre, floor, overhead_light, render, top_camera

IMPLS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


@pytest.fixture(params=IMPLS)
def impl(request):
    return request.param


def near(v, e, tol=ONE_LEVEL):
    return abs(v - e) <= tol


# ---- "raytrace shading matches three.js formulas", tests/render.test.ts:9-131

def test_lambert(impl):  # render.test.ts:10-18
    scene = S.Scene()
    scene.add(floor(S.MeshLambertMaterial(color=S.Color(0.5, 0.25, 1))), overhead_light(math.pi))
    r, g, b, a = centre(render(scene, top_camera(), impl=impl))
    assert abs(r - 0.5) < 0.005 and abs(g - 0.25) < 0.005 and abs(b - 1) < 0.005
    assert a == 1


def test_ambient(impl):  # render.test.ts:20-24
    scene = S.Scene()
    scene.add(floor(S.MeshLambertMaterial(color=S.Color(0.5, 0.5, 0.5))), S.AmbientLight(0xffffff, math.pi))
    assert near(centre(render(scene, top_camera(), impl=impl))[0], 0.5)


def test_hemisphere(impl):  # render.test.ts:26-31
    scene = S.Scene()
    hemi = S.HemisphereLight(0xffffff, 0x000000, math.pi)
    hemi.position.set(0, 0, 1)
    scene.add(floor(S.MeshLambertMaterial(color=S.Color(0.5, 0.5, 0.5))), hemi)
    assert near(centre(render(scene, top_camera(), impl=impl))[0], 0.5)


def test_standard_ggx(impl):  # render.test.ts:34-49
    scene = S.Scene()
    c = 0.5
    scene.add(floor(S.MeshStandardMaterial(color=S.Color(c, c, c), roughness=1, metalness=0)),
              overhead_light(math.pi))
    fw = cpu.fresnel_weight(1)
    F = 0.04 * (1 - fw) + fw
    fa, fb = cpu.dfg(1, 1)
    compensation = 1 + 0.04 * (1 / (fa + fb) - 1)
    specular = F * 0.25 * (1 / math.pi) * compensation
    diffuse = (c / math.pi) * (1 - F)
    expected = math.pi * (specular + diffuse)
    assert near(centre(render(scene, top_camera(), impl=impl))[0], expected)


def test_phong(impl):  # render.test.ts:51-58
    scene = S.Scene()
    scene.add(floor(S.MeshPhongMaterial(color=S.Color(0.2, 0.2, 0.2), specular=S.Color(0.1, 0.1, 0.1),
                                        shininess=10)), overhead_light(math.pi))
    fw = cpu.fresnel_weight(1)
    specular = (0.1 * (1 - fw) + fw) * 0.25 * (1 / math.pi) * (10 * 0.5 + 1)
    expected = math.pi * (0.2 / math.pi + specular)
    assert near(centre(render(scene, top_camera(), impl=impl))[0], expected)


def test_point_light(impl):  # render.test.ts:60-67
    scene = S.Scene()
    light = S.PointLight(0xffffff, 4, 0, 2)
    light.position.set(0, 0, 2)
    scene.add(floor(S.MeshLambertMaterial(color=0xffffff)), light)
    assert near(centre(render(scene, top_camera(), impl=impl))[0], 1 / math.pi)


def test_spot_light(impl):  # render.test.ts:69-77
    scene = S.Scene()
    spot = S.SpotLight(0xffffff, 20, 0, math.pi / 12, 0, 0)
    spot.position.set(0, 0, 2)
    scene.add(floor(S.MeshLambertMaterial(color=0xffffff)), spot, spot.target)
    image = render(scene, top_camera(), impl=impl)
    assert centre(image)[0] > 0.5
    assert image.at(0, 0)[0] == 0


def test_emission(impl):  # render.test.ts:79-85
    scene = S.Scene()
    scene.add(floor(S.MeshStandardMaterial(color=0x000000, emissive=0xff0000, emissive_intensity=0.5)))
    r, g, _, _ = centre(render(scene, top_camera(), impl=impl))
    assert near(r, 0.5)
    assert g == 0


def test_vertex_colours(impl):  # render.test.ts:87-93
    import numpy as np

    scene = S.Scene()
    geometry = S.plane_geometry(4, 4)
    geometry.color = np.array([[0, 1, 0]] * 4, np.float32)
    scene.add(S.Mesh(geometry, S.MeshBasicMaterial(vertex_colors=True)))
    assert centre(render(scene, top_camera(), impl=impl))[:3] == (0, 1, 0)


def test_textures(impl):  # render.test.ts:95-108
    import numpy as np

    data = np.array([255, 0, 0, 255, 0, 255, 0, 255, 0, 0, 255, 255, 255, 255, 255, 255], np.uint8)
    texture = S.DataTexture(data, 2, 2)
    scene = S.Scene()
    scene.add(S.Mesh(S.plane_geometry(2, 2), S.MeshBasicMaterial(map=texture)))
    image = render(scene, top_camera(), impl=impl)

    def close(p, q):
        return all(abs(p[i] - q[i]) < 0.2 for i in range(3))

    assert close(image.at(3, 12), (1, 0, 0))  # bottom left
    assert close(image.at(12, 12), (0, 1, 0))  # bottom right
    assert close(image.at(3, 3), (0, 0, 1))  # top left
    assert close(image.at(12, 3), (1, 1, 1))  # top right


def test_reinhard(impl):  # render.test.ts:110-115
    scene = S.Scene()
    scene.add(floor(S.MeshLambertMaterial(color=0xffffff)), overhead_light(math.pi))
    value = centre(render(scene, top_camera(), {"tone_mapping": S.ReinhardToneMapping}, impl=impl))[0]
    assert near(value, 0.5)


def test_srgb_output(impl):  # render.test.ts:117-122
    scene = S.Scene()
    scene.add(floor(S.MeshBasicMaterial(color=S.Color(0.5, 0.5, 0.5))))
    image = render(scene, top_camera(), {"output_color_space": "srgb"}, impl=impl)
    assert abs(centre(image)[0] - 0.7354) <= ONE_LEVEL * 1.5


def test_linear_fog(impl):  # render.test.ts:124-130
    scene = S.Scene()
    scene.fog = S.Fog(0xffffff, 0, 20)
    scene.add(floor(S.MeshBasicMaterial(color=0x000000)))
    assert near(centre(render(scene, top_camera(), impl=impl))[0], 0.5)


# ---- "raytrace visibility", tests/render.test.ts:133-328

def test_clear_colour(impl):  # render.test.ts:134-140
    scene = S.Scene()
    assert centre(render(scene, top_camera(), impl=impl)) == (0, 0, 0, 0)
    assert centre(render(scene, top_camera(), {"clear_color": (0, 0, 1), "clear_alpha": 1}, impl=impl)) == (0, 0, 1, 1)
    scene.background = S.Color(1, 0, 0)
    assert centre(render(scene, top_camera(), impl=impl)) == (1, 0, 0, 1)


def test_culling(impl):  # render.test.ts:142-154
    scene = S.Scene()
    material = S.MeshLambertMaterial(color=0xffffff)
    plane = floor(material)
    plane.rotation.x = math.pi
    scene.add(plane, overhead_light(math.pi))
    assert centre(render(scene, top_camera(), impl=impl))[3] == 0
    material.side = S.DoubleSide
    r, _, _, a = centre(render(scene, top_camera(), impl=impl))
    assert a == 1
    assert abs(r - 1) < 0.005


def test_shadows(impl):  # render.test.ts:156-174
    scene = S.Scene()
    ground = floor(S.MeshLambertMaterial(color=S.Color(0.5, 0.5, 0.5)))
    blocker = S.Mesh(S.plane_geometry(1, 1), S.MeshLambertMaterial())
    blocker.rotation.x = math.pi
    blocker.position.z = 2
    sun = overhead_light(math.pi)
    scene.add(ground, blocker, sun, S.AmbientLight(0xffffff, math.pi * 0.2))
    camera = top_camera()
    lit, shadowed = 0.5 * 1.2, 0.5 * 0.2
    assert near(centre(render(scene, camera, impl=impl))[0], shadowed)
    assert near(render(scene, camera, impl=impl).at(0, 0)[0], lit)
    assert near(centre(render(scene, camera, {"shadows": "none"}, impl=impl))[0], lit)
    assert near(centre(render(scene, camera, {"shadows": "castShadow"}, impl=impl))[0], lit)
    sun.cast_shadow = blocker.cast_shadow = ground.receive_shadow = True
    assert near(centre(render(scene, camera, {"shadows": "castShadow"}, impl=impl))[0], shadowed)


def test_transparent_blocker(impl):  # render.test.ts:176-184
    scene = S.Scene()
    ground = floor(S.MeshLambertMaterial(color=0xffffff))
    blocker = S.Mesh(S.plane_geometry(1, 1), S.MeshLambertMaterial(transparent=True, opacity=0.25))
    blocker.rotation.x = math.pi
    blocker.position.z = 2
    scene.add(ground, blocker, overhead_light(math.pi))
    assert abs(centre(render(scene, top_camera(), impl=impl))[0] - 0.75) < 0.005


def test_mirror(impl):  # render.test.ts:186-200
    scene = S.Scene()
    scene.add(floor(S.MeshStandardMaterial(color=0xffffff, metalness=1, roughness=0)))
    panel = S.Mesh(S.plane_geometry(10, 10), S.MeshBasicMaterial(color=0xff0000))
    panel.rotation.x = math.pi
    panel.position.z = 20
    scene.add(panel)
    r, g, b, _ = centre(render(scene, top_camera(), impl=impl))
    assert r > 0.85 and g == 0 and b == 0
    assert centre(render(scene, top_camera(), {"max_bounces": 0}, impl=impl))[0] == 0


def test_environment_reflection(impl):  # render.test.ts:202-216
    import numpy as np

    scene = S.Scene()
    env = S.DataTexture(np.array([0.5, 0.25, 0, 1, 0.5, 0.25, 0, 1], np.float32), 2, 1, S.RGBAFormat, S.FloatType)
    env.mapping = S.EquirectangularReflectionMapping
    scene.environment = env
    scene.add(floor(S.MeshStandardMaterial(color=0xffffff, metalness=1, roughness=0)))
    r, g, _, _ = centre(render(scene, top_camera(), impl=impl))
    assert r > 0.4
    assert abs(g / r - 0.5) < 0.05
    scene.background = env
    br, bg, _, _ = render(scene, top_camera(), impl=impl).at(8, 8)
    assert br > 0 and bg > 0


def test_stochastic_transparency(impl):  # render.test.ts:218-225
    scene = S.Scene()
    scene.add(floor(S.MeshBasicMaterial(color=0xff0000, transparent=True, opacity=0.5)))
    r, _, b, a = centre(render(scene, top_camera(), {"samples": 200, "clear_color": (0, 0, 1), "clear_alpha": 1},
                               impl=impl))
    assert abs(r - 0.5) < 0.05 and abs(b - 0.5) < 0.05
    assert a == 1


def test_alpha_test(impl):  # render.test.ts:227-231
    scene = S.Scene()
    scene.add(floor(S.MeshBasicMaterial(color=0xff0000, opacity=0.2, alpha_test=0.5)))
    assert centre(render(scene, top_camera(), impl=impl))[3] == 0


def test_perspective(impl):  # render.test.ts:233-242
    scene = S.Scene()
    scene.add(S.Mesh(S.box_geometry(1, 1, 1), S.MeshBasicMaterial(color=0xffffff)))
    camera = S.PerspectiveCamera(60, 1, 0.1, 100)
    camera.position.set(0, 0, 5)
    camera.update_matrix_world()
    image = render(scene, camera, impl=impl)
    assert centre(image) == (1, 1, 1, 1)
    assert image.at(0, 0)[3] == 0


def test_global_illumination(impl):  # render.test.ts:244-257
    scene = S.Scene()
    scene.add(floor(S.MeshLambertMaterial(color=0xffffff), 40))
    lamp = S.Mesh(S.plane_geometry(40, 40), S.MeshBasicMaterial(color=0xff0000))
    lamp.rotation.x = math.pi
    lamp.position.z = 20
    scene.add(lamp)
    off = centre(render(scene, top_camera(), {"samples": 8}, impl=impl))
    on = centre(render(scene, top_camera(), {"samples": 64, "global_illumination": True}, impl=impl))
    assert off[0] == 0
    assert on[0] > 0.3
    assert on[1] == 0


def test_refraction(impl):  # render.test.ts:259-269
    scene = S.Scene()
    scene.add(floor(S.MeshBasicMaterial(color=0x00ff00)))
    glass = S.Mesh(S.box_geometry(1, 1, 1), S.MeshPhysicalMaterial(transmission=1, roughness=0, thickness=1,
                                                                    color=0xffffff))
    glass.position.z = 1
    scene.add(glass)
    r, g, _, a = centre(render(scene, top_camera(), {"samples": 32}, impl=impl))
    assert a == 1 and g > 0.6 and r < 0.1


def _glass(attenuated):
    kw = dict(color=0xffffff, transmission=1, roughness=0, thickness=1)
    if attenuated:
        kw.update(attenuation_color=S.Color(0.5, 1, 1), attenuation_distance=1)
    return S.MeshPhysicalMaterial(**kw)


def test_volume_absorption(impl):  # render.test.ts:271-296
    scene = S.Scene()
    scene.add(floor(S.MeshBasicMaterial(color=0xffffff)))
    slab = S.Mesh(S.box_geometry(3, 3, 1), _glass(True))
    slab.position.z = 1
    scene.add(slab)
    r, g, b, _ = centre(render(scene, top_camera(), {"samples": 16}, impl=impl))
    assert abs(r / g - 0.5) < 0.05
    assert abs(b - g) < 0.005
    assert g > 0.7
    slab.scale.z = 2
    slab.position.z = 1.5
    r2, g2, _, _ = centre(render(scene, top_camera(), {"samples": 16}, impl=impl))
    assert abs(r2 / g2 - 0.25) < 0.05
    slab.material = _glass(False)
    r3, g3, _, _ = centre(render(scene, top_camera(), {"samples": 16}, impl=impl))
    assert abs(r3 / g3 - 1) < 0.005


def test_tinted_shadows(impl):  # render.test.ts:298-319
    scene = S.Scene()
    light = S.DirectionalLight(0xffffff, math.pi)
    light.position.set(1, 0.5, 10)
    scene.add(floor(S.MeshLambertMaterial(color=0xffffff)), light)
    slab = S.Mesh(S.box_geometry(3, 3, 1), _glass(True))
    slab.position.z = 1
    scene.add(slab)

    def ratio(shadows):
        r, g, _, _ = centre(render(scene, top_camera(), {"samples": 32, "shadows": shadows}, impl=impl))
        return r / g

    assert abs(ratio("none") - 0.5) < 0.05
    assert abs(ratio("all") - 0.25) < 0.05


def test_same_seed_same_bytes(impl):  # render.test.ts:321-327
    scene = S.Scene()
    scene.add(floor(S.MeshStandardMaterial(roughness=0.5, metalness=0.5)), overhead_light(2),
              S.AmbientLight(0xffffff, 1))
    a = render(scene, top_camera(), {"samples": 4, "output_color_space": "srgb"}, 8, 8, impl=impl).data
    b = render(scene, top_camera(), {"samples": 4, "output_color_space": "srgb"}, 8, 8, impl=impl).data
    assert (a == b).all()
