"""The oracle pinned to the reference's tests/bvh.test.ts and tests/color.test.ts.

These run the oracle alone (CPU): the same brute-force, culling, flat-box,
coincident and empty-scene cases as the reference, and its colour / BRDF
known answers.
"""
import math

import numpy as np
import pytest

from oracle import cpu

from meercadraytracer_b200.types import CompiledTexture


def lcg_triangles(count: int, seed: int) -> np.ndarray:
    """randomTriangles, tests/bvh.test.ts:4-19 (LCG s = s * 1664525 + 1013904223)."""
    s = seed

    def rand():
        nonlocal s
        s = (s * 1664525 + 1013904223) % (1 << 32)
        return s / 4294967296

    data = np.zeros(count * 9, np.float32)
    for i in range(count):
        cx, cy, cz = rand() * 20 - 10, rand() * 20 - 10, rand() * 20 - 10
        v = [[cx + rand() * 2 - 1, cy + rand() * 2 - 1, cz + rand() * 2 - 1] for _ in range(3)]
        data[i * 9:i * 9 + 3] = v[0]
        data[i * 9 + 3:i * 9 + 6] = [v[1][a] - v[0][a] for a in range(3)]
        data[i * 9 + 6:i * 9 + 9] = [v[2][a] - v[0][a] for a in range(3)]
    return data


def reorder(data: np.ndarray, order: np.ndarray) -> np.ndarray:
    return data.reshape(-1, 9)[order].reshape(-1).copy()


def brute_force(data: np.ndarray, o, d):
    """bruteForce, tests/bvh.test.ts:27-51 (double-precision Moller-Trumbore)."""
    best, tri, allhits = math.inf, -1, 0
    t9 = data.reshape(-1, 9).astype(np.float64)
    for k in range(t9.shape[0]):
        b = t9[k]
        e1, e2 = b[3:6], b[6:9]
        p = [d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]]
        det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2]
        if det == 0:
            continue
        s = [o[0] - b[0], o[1] - b[1], o[2] - b[2]]
        u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) / det
        if u < 0 or u > 1:
            continue
        q = [s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]]
        v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) / det
        if v < 0 or u + v > 1:
            continue
        t = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) / det
        if t > 0:
            allhits += 1
            if t < best:
                best, tri = t, k
    return best, tri, allhits


def lissajous_ray(i: int):
    """The 400 deterministic rays of tests/bvh.test.ts:84-89."""
    o = [math.sin(i) * 30, math.cos(i * 1.3) * 30, math.sin(i * 0.7) * 30]
    target = [math.sin(i * 2.1) * 8, math.cos(i * 0.4) * 8, math.sin(i * 1.7) * 8]
    d = [target[a] - o[a] for a in range(3)]
    length = math.hypot(*d)
    return o, [x / length for x in d]


@pytest.fixture(scope="module")
def bvh3000():
    raw = lcg_triangles(3000, 7)
    bvh, order = cpu.build_bvh(raw, 3000)
    return raw, bvh, order, reorder(raw, order)


def test_every_triangle_once_in_bounded_leaves(bvh3000):  # bvh.test.ts:62-80
    raw, bvh, order, data = bvh3000
    assert sorted(order.tolist()) == list(range(3000))
    covered = 0
    nodes = bvh.nodes.reshape(-1, 3)
    bounds = bvh.bounds.reshape(-1, 6)
    t9 = data.reshape(-1, 9).astype(np.float64)
    for n in range(bvh.node_count):
        first, c = nodes[n, 0], nodes[n, 1]
        if c == 0:
            continue
        covered += c
        for k in range(first, first + c):
            for v in range(3):
                x = t9[k, 0:3] + (t9[k, v * 3:v * 3 + 3] if v > 0 else 0)
                assert (x >= bounds[n, 0:3] - 1e-4).all() and (x <= bounds[n, 3:6] + 1e-4).all()
    assert covered == 3000


def test_closest_and_all_hits_match_brute_force(bvh3000):  # bvh.test.ts:82-107
    raw, bvh, order, data = bvh3000
    sides = np.full(3000, 2, np.uint8)
    hits = 0
    for i in range(400):
        o, d = lissajous_ray(i)
        best, tri, allhits = brute_force(data, o, d)
        found, hit = cpu.intersect_closest(data, sides, bvh, o, d)
        assert found == (tri >= 0)
        if found:
            hits += 1
            assert abs(hit.t - best) < 0.5e-3
            assert hit.triangle == tri
        assert cpu.intersect_any_count(data, bvh, o, d) == allhits
    assert hits > 100


@pytest.mark.parametrize("bins", [16, 32])
def test_bin_count_parameter(bvh3000, bins):
    """BINS (bvh.ts:3) as a parameter: 16 is the default build, and a 32-bin tree of the
    same triangles is another valid BVH (every triangle once, hits equal brute force)
    whose split decisions differ."""
    raw, bvh16, order16, _ = bvh3000
    bvh, order = cpu.build_bvh(raw, 3000, bins=bins)
    assert sorted(order.tolist()) == list(range(3000))
    if bins == 16:
        assert np.array_equal(bvh.nodes, bvh16.nodes) and np.array_equal(order, order16)
        return
    assert not (bvh.node_count == bvh16.node_count and np.array_equal(order, order16))
    data = reorder(raw, order)
    sides = np.full(3000, 2, np.uint8)
    for i in range(0, 400, 4):
        o, d = lissajous_ray(i)
        best, tri, allhits = brute_force(data, o, d)
        found, hit = cpu.intersect_closest(data, sides, bvh, o, d)
        assert found == (tri >= 0) and (not found or hit.triangle == tri)
        assert cpu.intersect_any_count(data, bvh, o, d) == allhits


def test_culling_front_back_double():  # bvh.test.ts:109-123
    tri = np.array([-1, -1, 0, 2, 0, 0, 0, 2, 0], np.float32)
    bvh, _ = cpu.build_bvh(tri, 1)

    def front(side):
        return cpu.intersect_closest(tri, np.array([side], np.uint8), bvh, (0, 0, 5), (0, 0, -1))

    def back(side):
        return cpu.intersect_closest(tri, np.array([side], np.uint8), bvh, (0, 0, -5), (0, 0, 1))

    found, hit = front(0)
    assert found and hit.front
    assert not back(0)[0]
    assert not front(1)[0]
    found, hit = back(1)
    assert found and not hit.front
    assert front(2)[0] and back(2)[0]


def test_flat_box_along_face():  # bvh.test.ts:125-133
    quad = np.array([-1, -1, 0, 2, 0, 0, 2, 2, 0, -1, -1, 0, 2, 2, 0, 0, 2, 0], np.float32)
    bvh, order = cpu.build_bvh(quad, 2)
    ordered = reorder(quad, order)
    found, hit = cpu.intersect_closest(ordered, np.full(2, 2, np.uint8), bvh, (-1, 0, 3), (0, 0, -1))
    assert found and abs(hit.t - 3) < 1e-6


def test_coincident_triangles():  # bvh.test.ts:135-142
    same = np.tile(np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32), 500)
    bvh, _ = cpu.build_bvh(same, 500)
    assert bvh.node_count > 1
    assert cpu.intersect_closest(same, np.full(500, 2, np.uint8), bvh, (0.2, 0.2, 1), (0, 0, -1))[0]


def test_empty_scene():  # bvh.test.ts:144-148
    bvh, _ = cpu.build_bvh(np.zeros(0, np.float32), 0)
    assert bvh.node_count == 0
    assert not cpu.intersect_closest(np.zeros(0, np.float32), np.zeros(0, np.uint8), bvh, (0, 0, 0), (0, 0, 1))[0]


# ---- tests/color.test.ts

NO, LINEAR, REINHARD, CINEON, ACES, AGX, NEUTRAL = 0, 1, 2, 3, 4, 6, 7


def test_srgb_round_trip():  # color.test.ts:22-25
    for v in [0, 0.001, 0.02, 0.2, 0.5, 0.8, 1]:
        assert abs(cpu.srgb_to_linear(cpu.linear_to_srgb(v)) - v) < 0.5e-4
    assert abs(cpu.linear_to_srgb(0.5) - 0.7354) < 0.5e-3


def test_half_floats():  # color.test.ts:27-32
    assert cpu.half_to_float(0x3c00) == 1
    assert cpu.half_to_float(0xc000) == -2
    assert cpu.half_to_float(0x3800) == 0.5
    assert cpu.half_to_float(0x0000) == 0


def test_tone_mapping_operators():  # color.test.ts:34-57
    assert cpu.tone_map([1, 0.5, 4], NO) == [1, 0.5, 4]
    assert cpu.tone_map([0.5, 2, 0], LINEAR, 1) == [0.5, 1, 0]
    assert abs(cpu.tone_map([1, 3, 0], REINHARD)[0] - 0.5) < 1e-9
    assert abs(cpu.tone_map([1, 3, 0], REINHARD)[1] - 0.75) < 1e-9
    assert abs(cpu.tone_map([1, 0, 0], REINHARD, 3)[0] - 0.75) < 1e-9
    x = 0.18 - 0.004
    expected = math.pow((x * (6.2 * x + 0.5)) / (x * (6.2 * x + 1.7) + 0.06), 2.2)
    assert abs(cpu.tone_map([0.18] * 3, CINEON)[0] - expected) < 0.5e-6
    assert abs(cpu.tone_map([0.5] * 3, NEUTRAL)[0] - 0.46) < 0.5e-6
    for mapping in (ACES, AGX, NEUTRAL):
        bright = cpu.tone_map([20, 20, 20], mapping)
        dark = cpu.tone_map([0.05, 0.05, 0.05], mapping)
        assert bright[0] <= 1.000001 and bright[0] > dark[0] and dark[0] >= 0
    grey = cpu.tone_map([0.3] * 3, ACES)
    assert abs(grey[0] - grey[1]) < 0.005 and abs(grey[1] - grey[2]) < 0.005


def test_dfg_texel_centres():  # color.test.ts:61-70
    import os
    import re

    header = os.path.join(os.path.dirname(__file__), "..", "meercadraytracer_b200", "csrc", "dfg_lut.h")
    lut = [int(v, 16) for v in re.findall(r"0x([0-9a-f]{4})", open(header).read().split("{", 1)[1])]
    a, b = cpu.dfg(3.5 / 16, 5.5 / 16)
    assert abs(a - cpu.half_to_float(int(lut[(5 * 16 + 3) * 2]))) < 0.5e-6
    assert abs(b - cpu.half_to_float(int(lut[(5 * 16 + 3) * 2 + 1]))) < 0.5e-6
    a, b = cpu.dfg(0, 1)
    assert a + b > 0.9


def test_ggx_normalised():  # color.test.ts:72-83
    for alpha in (0.1, 0.5, 1):
        steps = 4000
        total = 0.0
        for i in range(steps):
            theta = ((i + 0.5) / steps) * (math.pi / 2)
            total += cpu.distribution_ggx(alpha, math.cos(theta)) * math.cos(theta) * math.sin(theta) * 2 * math.pi * (
                math.pi / 2 / steps)
        assert abs(total - 1) < 0.005


def test_helpers():  # color.test.ts:85-93
    assert cpu.fresnel_weight(0) == 1
    assert cpu.fresnel_weight(1) < 0.001
    assert cpu.smoothstep(0, 1, 0.5) == 0.5
    assert cpu.smoothstep(0.5, 0.5, 0.6) == 1
    assert abs(cpu.distance_attenuation(2, 0, 2) - 0.25) < 1e-9
    assert cpu.distance_attenuation(0.01, 0, 2) == 100
    assert cpu.distance_attenuation(10, 10, 2) == 0


# ---- compile.test.ts texture sampling known answers (154-174, 191-200)

def test_texture_transform_and_wrapping():
    data = np.array([255, 0, 0, 255, 0, 255, 0, 255, 0, 0, 255, 255, 255, 255, 255, 255], np.uint8)
    # repeat (2, 1), RepeatWrapping: matrix diag(2, 1).
    t = CompiledTexture(2, 2, data, srgb=False, flip_y=False, wrap_s=1000, wrap_t=1000,
                        matrix=(2, 0, 0, 0, 1, 0, 0, 0, 1))
    assert cpu.sample_texture(t, 0.125, 0.25)[:3] == [1, 0, 0]
    assert cpu.sample_texture(t, 0.625, 0.25)[:3] == [1, 0, 0]
    assert cpu.sample_texture(t, 0.375, 0.75)[:3] == [1, 1, 1]


def test_half_float_texture():
    half = np.array([0.25, 2, 4, 1], np.float16).view(np.uint16)
    from meercadraytracer_b200 import scene as S
    from meercadraytracer_b200.compile import TextureTable

    tex = S.DataTexture(half, 1, 1, S.RGBAFormat, S.HalfFloatType)
    table = TextureTable()
    table.add(tex)
    assert cpu.sample_texture(table.textures[0], 0.5, 0.5) == [0.25, 2, 4, 1]


def test_uint8_clamped_rounding():
    # ToUint8Clamp: clamp, NaN -> 0, round half to even.
    assert cpu.uint8_clamp(float("nan")) == 0
    assert cpu.uint8_clamp(-3) == 0
    assert cpu.uint8_clamp(300) == 255
    assert cpu.uint8_clamp(127.5) == 128
    assert cpu.uint8_clamp(126.5) == 126
    assert cpu.uint8_clamp(126.50001) == 127


def test_random_is_lowbias32_xorshift():
    # Random.seed / next, src/random.ts:6-20: a hand-evaluated first step.
    h = cpu.hash32(0)
    assert h == 0
    state = cpu.seed(0, 0, 0, 0)
    assert state == 0x9E3779B9  # a zero hash is replaced by the golden ratio constant
    values, after = cpu.random_sequence(1, 3)
    x = 1
    expect = []
    for _ in range(3):
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        expect.append(x / 4294967296)
    assert values == expect and after == x
