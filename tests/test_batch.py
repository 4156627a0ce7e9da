"""Batched and served rendering (mcrt_batch_*), through the C ABI.

Every request's final image must equal the plain per-request render
(mcrt_raytrace, i.e. raytraceCompiled) byte for byte: the same paths are
traced and each pixel's passes are accumulated in pass order, whatever else
shares the wavefront. The block preview must equal the reference's
ProgressiveRenderer preview: the block tile render (Tracer.renderTile with
block > 1) written with writeTile(..., sum = null, count = 1).
"""
import numpy as np
import pytest

from meercadraytracer_b200 import scenes
from meercadraytracer_b200.batch import EVENT_DONE, EVENT_PREVIEW, EVENT_PROGRESS, BatchRenderer, RenderRequest
from meercadraytracer_b200.compile import compile_camera, compile_scene
from meercadraytracer_b200.raytrace import as_options, trace_settings
from meercadraytracer_b200.types import Tile
from oracle import cpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def two_scenes():
    small = scenes.small_scene()
    mid = scenes.mid_scene(grid=4, subdivisions=2, width=160, height=90)
    mid.camera.position.set(0, 8, 14)
    mid.camera.look_at(0, 0, 0)
    mid.camera.update_matrix_world()
    out = []
    for b in (small, mid):
        out.append((compile_scene(b.scene, builder=cpu.compile_sink), compile_camera(b.camera),
                    trace_settings(as_options(b.options))))
    return out


def _requests(two_scenes):
    (s_scene, s_cam, s_st), (m_scene, m_cam, m_st) = two_scenes
    gi = trace_settings(as_options({"global_illumination": True, "max_bounces": 4,
                                    "tone_mapping": s_st.tone_mapping, "seed": 9}))
    return [
        RenderRequest(s_scene, s_cam, 64, 48, s_st, 4),
        RenderRequest(m_scene, m_cam, 96, 54, m_st, 3),
        RenderRequest(s_scene, s_cam, 33, 17, gi, 1),
        RenderRequest(m_scene, m_cam, 40, 40, m_st, 5),
        RenderRequest(s_scene, s_cam, 70, 50, s_st, 2),
    ]


def _plain(renderer, r):
    ex = renderer.executor(r.scene)
    return ex.raytrace(r.scene, r.camera, r.width, r.height, r.settings, r.samples, r.srgb)


def test_host_loop_matches_plain_renders(two_scenes):
    renderer = BatchRenderer(capacity=1 << 15, memory_budget=64 << 20, use_graph=False)
    try:
        reqs = _requests(two_scenes)
        for r, img in zip(reqs, renderer.render(reqs)):
            assert np.array_equal(img, _plain(renderer, r))
    finally:
        renderer.dispose()


@pytest.mark.parametrize("capacity", [1 << 15, 3000])
def test_batch_matches_plain_renders(two_scenes, capacity):
    # 3000 paths split the larger passes by pixel range over several chunks.
    renderer = BatchRenderer(capacity=capacity, memory_budget=64 << 20)
    try:
        reqs = _requests(two_scenes)
        images = renderer.render(reqs)
        for r, img in zip(reqs, images):
            assert np.array_equal(img, _plain(renderer, r))
        st = renderer.stats()
        assert st["graph_launches"] >= 1 and st["status"] == 0
        assert st["closest_rays"] > 0 and st["arena_used"] == 0
    finally:
        renderer.dispose()


def test_whole_batch_is_one_graph_launch(two_scenes):
    # mcrt_batch_render plans every chunk ahead and runs them all as one graph
    # launch, the two halves of the pool side by side; the images are still the
    # plain renders', and a second batch reuses the graph (one more launch).
    renderer = BatchRenderer(capacity=6000, memory_budget=64 << 20)
    try:
        reqs = _requests(two_scenes)
        images = renderer.render(reqs)
        st = renderer.stats()
        assert st["graph_launches"] == 1 and st["chunks"] > 2 and st["status"] == 0
        assert st["arena_used"] == 0
        for r, img in zip(reqs, images):
            assert np.array_equal(img, _plain(renderer, r))
        again = renderer.render(reqs[1:4])
        assert renderer.stats()["graph_launches"] == 2
        for r, img in zip(reqs[1:4], again):
            assert np.array_equal(img, _plain(renderer, r))
    finally:
        renderer.dispose()


def test_request_alone_equals_request_in_mix(two_scenes):
    reqs = _requests(two_scenes)
    alone = BatchRenderer(capacity=1 << 15, memory_budget=64 << 20)
    mixed = BatchRenderer(capacity=1 << 15, memory_budget=64 << 20)
    try:
        a = alone.render([reqs[1]])[0]
        m = mixed.render(reqs)[1]
        assert np.array_equal(a, m)
    finally:
        alone.dispose()
        mixed.dispose()


def test_memory_budget_admits_requests_in_turn(two_scenes):
    # Buffers take 20 B per pixel (Float32 sum + RGBA8): the 96x54 request needs
    # ~104 kB and two 70x50 ones ~140 kB, so requests wait for each other.
    reqs = _requests(two_scenes)
    renderer = BatchRenderer(capacity=1 << 15, memory_budget=130_000)
    try:
        for r, img in zip(reqs, renderer.render(reqs)):
            assert np.array_equal(img, _plain(renderer, r))
    finally:
        renderer.dispose()


def test_preview_then_done_events(two_scenes):
    s_scene, s_cam, s_st = two_scenes[0]
    w, h, block = 64, 48, 8
    renderer = BatchRenderer(capacity=1 << 15, memory_budget=64 << 20)
    try:
        rid = renderer.submit(RenderRequest(s_scene, s_cam, w, h, s_st, 3, preview_block=block))
        seen = []
        for _ in range(1000):
            events, idle = renderer.step()
            seen += [(e[0], e[1]) for e in events]
            if idle:
                break
        assert seen == [(rid, EVENT_PREVIEW), (rid, EVENT_DONE)]
        # The preview: one block-centre sample per 8x8 block, written with count 1.
        ex = renderer.executor(s_scene)
        gv, sv = ex.load_scene(s_scene)
        tile = Tile(0, 0, w, h)
        fut = ex.render({"type": "tile", "job": 1, "geometry_version": gv, "shading_version": sv, "camera": s_cam,
                         "settings": s_st, "tile": tile, "width": w, "height": h, "pass": 0, "block": block})
        data = fut.result()
        expect = np.zeros(w * h * 4, np.uint8)
        cpu.encode_tile(expect, w, tile, data, None, 1, True)
        assert np.array_equal(renderer.preview(rid), expect)
        assert np.array_equal(renderer.result(rid), _plain(renderer, RenderRequest(s_scene, s_cam, w, h, s_st, 3)))
    finally:
        renderer.dispose()


def test_cancelled_requests_return_their_memory(two_scenes):
    reqs = _requests(two_scenes)
    renderer = BatchRenderer(capacity=4096, memory_budget=64 << 20)
    try:
        ids = [renderer.submit(r) for r in reqs]
        renderer.step()
        for rid in ids[1:]:
            renderer.cancel(rid)
        done = []
        for _ in range(10000):
            events, idle = renderer.step()
            done += [e[0] for e in events if e[1] == EVENT_DONE]
            if idle:
                break
        assert done == [ids[0]]
        assert np.array_equal(renderer.result(ids[0]), _plain(renderer, reqs[0]))
        assert renderer.stats()["arena_used"] == 0
    finally:
        renderer.dispose()


def test_progress_events_report_completed_passes(two_scenes):
    # 64 x 48 = 3072 pixels; a 6144-path chunk (half of the pool) holds two passes, so a
    # 6-sample render reports progress at 2 and 4 passes, then done at 6.
    s_scene, s_cam, s_st = two_scenes[0]
    w, h = 64, 48
    renderer = BatchRenderer(capacity=4 * w * h, memory_budget=64 << 20)
    try:
        rid = renderer.submit(RenderRequest(s_scene, s_cam, w, h, s_st, 6, progress=True))
        seen, frames = [], []
        for _ in range(1000):
            events, idle = renderer.step()
            for e in events:
                seen.append((e[1], e[2]))
                if e[1] == EVENT_PROGRESS:
                    frames.append((e[2], renderer.progress(rid).copy()))
            if idle:
                break
        assert seen == [(EVENT_PROGRESS, 2), (EVENT_PROGRESS, 4), (EVENT_DONE, 6)]
        plain = {n: _plain(renderer, RenderRequest(s_scene, s_cam, w, h, s_st, n)) for n in (2, 4, 6)}
        # The progress image holds at least the passes the event reports (a later chunk's
        # copy may have refreshed it before the host looked).
        for n, img in frames:
            assert any(np.array_equal(img, plain[k]) for k in plain if k >= n)
        assert np.array_equal(renderer.result(rid), plain[6])
    finally:
        renderer.dispose()
