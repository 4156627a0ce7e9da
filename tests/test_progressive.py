"""Progressive rendering, scene sync and the headless RaytracingRenderer, restated
from the reference's tests/progressive.test.ts.

The CPU tests cover the host logic (tiles, what SceneSync sends and when,
renderer sizing and settings) with the oracle's geometry builder and a
recording executor; the GPU tests run ProgressiveRenderer and
RaytracingRenderer on the device and compare their images with raytrace's.
"""
import threading
import time

import numpy as np
import pytest

from meercadraytracer_b200 import scene as S
from meercadraytracer_b200.progressive import ProgressiveOptions, ProgressiveRenderer, SceneSync, make_tiles
from meercadraytracer_b200.raytrace import trace_settings
from meercadraytracer_b200.renderer import RaytracingRenderer
from oracle import cpu

from helpers import floor, overhead_light, top_camera


def scene_for_test() -> S.Scene:
    """testScene, tests/progressive.test.ts:38-47."""
    scene = S.Scene()
    texture = S.DataTexture(np.array([255, 255, 255, 255, 128, 128, 128, 255], np.uint8), 2, 1)
    scene.add(floor(S.MeshStandardMaterial(map=texture, roughness=0.6)), overhead_light(2),
              S.AmbientLight(0xffffff, 1))
    box = S.Mesh(S.box_geometry(0.5, 0.5, 0.5), S.MeshPhongMaterial(color=S.Color(0xff8800)))
    box.position.z = 0.5
    scene.add(box)
    return scene


def options(**kw) -> ProgressiveOptions:
    """options, tests/progressive.test.ts:49-54."""
    base = dict(width=20, height=12, settings=trace_settings({}), output_color_space="srgb", samples=3,
                preview_block=1, tile_size=8, frame_interval=0)
    base.update(kw)
    return ProgressiveOptions(**base)


def test_make_tiles_cover_the_image_centre_first():  # progressive.test.ts:57-63
    tiles = make_tiles(20, 12, 8)
    assert sum(t.width * t.height for t in tiles) == 240
    first = tiles[0]
    assert first.x <= 10 <= first.x + first.width
    covered = np.zeros((12, 20), np.int32)
    for t in tiles:
        covered[t.y:t.y + t.height, t.x:t.x + t.width] += 1
    assert (covered == 1).all()


class RecordingExecutor:
    """A TileExecutor stand-in that records the messages SceneSync sends it."""

    def __init__(self):
        self.received = []
        self.textures = set()

    def send(self, message, transfer=None):
        self.received.append(message)


def test_scene_sync_sends_scene_data_only_when_it_changes():  # progressive.test.ts:78-111
    scene, camera = scene_for_test(), top_camera()
    sync = SceneSync(builder=cpu.compile_sink)
    workers = [RecordingExecutor(), RecordingExecutor()]
    count = lambda kind: sum(1 for w in workers for m in w.received if m["type"] == kind)  # noqa: E731

    def render_once():
        sync.update(scene, camera)
        for w in workers:
            sync.sync(w)

    render_once()
    assert (count("geometry"), count("textures"), count("shading")) == (2, 2, 2)
    # Moving the camera resends nothing.
    camera.position.x = 0.3
    camera.update_matrix_world()
    render_once()
    assert (count("geometry"), count("shading")) == (2, 2)
    # A colour change resends shading, but not geometry or textures.
    scene.children[0].material.color = S.Color(0x00ff00)
    render_once()
    assert (count("geometry"), count("textures"), count("shading")) == (2, 2, 4)
    # Moving a mesh resends geometry.
    scene.children[3].position.x = 0.2
    render_once()
    assert count("geometry") == 4
    assert sync.geometry_version == 2 and sync.shading_version == 2
    # A new executor gets everything once.
    late = RecordingExecutor()
    sync.sync(late)
    assert [m["type"] for m in late.received] == ["geometry", "textures", "shading"]


def test_renderer_sizes_like_webgl_renderer():  # progressive.test.ts:175-187
    renderer = RaytracingRenderer(executors=[])
    renderer.set_pixel_ratio(2)
    renderer.set_size(40, 30)
    assert (renderer.width, renderer.height) == (80, 60)
    assert renderer.image.size == 80 * 60 * 4
    assert renderer.get_size() == (40, 30)
    renderer.set_pixel_ratio(1)
    assert renderer.width == 40
    renderer.dispose()


def test_renderer_copies_output_settings():  # progressive.test.ts:189-204
    class WebGL:
        tone_mapping = S.ReinhardToneMapping
        tone_mapping_exposure = 1.5
        output_color_space = S.LinearSRGBColorSpace

        def get_clear_color(self):
            return (0.25, 0.5, 1.0)

        def get_clear_alpha(self):
            return 0.5

        def get_pixel_ratio(self):
            return 1

    renderer = RaytracingRenderer(executors=[]).copy_settings_from(WebGL())
    assert renderer.tone_mapping == S.ReinhardToneMapping
    assert renderer.tone_mapping_exposure == 1.5
    assert renderer.output_color_space == S.LinearSRGBColorSpace
    assert renderer.get_clear_color() == (0.25, 0.5, 1.0)
    assert renderer.get_clear_alpha() == 0.5
    renderer.set_clear_color(0xffffff, 1)
    assert renderer.get_clear_alpha() == 1
    assert renderer.get_clear_color() == (1.0, 1.0, 1.0)
    renderer.dispose()


def test_renderer_without_executors_does_not_render():
    renderer = RaytracingRenderer(executors=[])
    renderer.set_size(8, 8)
    assert renderer.render_async(scene_for_test(), top_camera()).result(timeout=30) is False
    renderer.dispose()


# ------------------------------------------------------------------ GPU

def _gpu_raytrace(scene, camera, width, height, samples):
    from meercadraytracer_b200.raytrace import raytrace

    return raytrace(scene, camera, width, height, {"samples": samples}).data


@pytest.mark.gpu
def test_progressive_renders_the_same_image_as_raytrace():  # progressive.test.ts:66-76
    from meercadraytracer_b200.executors import GpuExecutor

    scene, camera = scene_for_test(), top_camera()
    frames = []
    renderer = ProgressiveRenderer([GpuExecutor(0)], capacity=1 << 12)
    try:
        done = renderer.render(scene, camera, options(), lambda f: frames.append((f.samples, f.done, f.image.copy())))
        assert done is True
        samples, is_done, image = frames[-1]
        assert is_done and samples == 3
        assert np.array_equal(image, _gpu_raytrace(scene, camera, 20, 12, 3))
    finally:
        renderer.dispose()


@pytest.mark.gpu
def test_progressive_shows_a_block_preview_first_then_each_pass():  # progressive.test.ts:112-118
    from meercadraytracer_b200.executors import GpuExecutor

    scene, camera = scene_for_test(), top_camera()
    frames = []
    # 240 paths per chunk: one pass of the 20 x 12 image per chunk, so every pass is reported.
    renderer = ProgressiveRenderer([GpuExecutor(0)], capacity=240)
    try:
        assert renderer.render(scene, camera, options(preview_block=4), lambda f: frames.append((f.samples, f.image.copy())))
        assert frames[0][0] == 0
        assert frames[-1][0] == 3
        counts = [s for s, _ in frames]
        assert counts == sorted(counts)
        # Every intermediate frame holds at least the passes it reports, and is the image
        # raytrace gives at some sample count from there to the end.
        refs = {n: _gpu_raytrace(scene, camera, 20, 12, n) for n in (1, 2, 3)}
        for s, img in frames[1:]:
            assert any(np.array_equal(img, refs[n]) for n in range(max(1, s), 4))
    finally:
        renderer.dispose()


@pytest.mark.gpu
def test_progressive_stops_when_superseded():  # progressive.test.ts:120-129
    from meercadraytracer_b200.executors import GpuExecutor

    renderer = ProgressiveRenderer([GpuExecutor(0)], capacity=240)
    try:
        results = {}
        started = threading.Event()

        def first():
            results["first"] = renderer.render(scene_for_test(), top_camera(), options(samples=5000),
                                               lambda f: started.set())

        t = threading.Thread(target=first)
        t.start()
        assert started.wait(60)
        results["second"] = renderer.render(scene_for_test(), top_camera(), options(samples=1), lambda f: None)
        t.join(60)
        assert results == {"first": False, "second": True}

        def stop_on_first_frame(f):
            renderer.stop()

        assert renderer.render(scene_for_test(), top_camera(), options(samples=50), stop_on_first_frame) is False
    finally:
        renderer.dispose()


@pytest.mark.gpu
def test_renderer_draws_progressively_and_reports_progress():  # progressive.test.ts:206-220
    renderer = RaytracingRenderer(samples=2, preview_block=4, frame_interval=0)
    renderer.set_size(20, 12)
    progress = []
    drawn = []
    renderer.on_progress(lambda p: (progress.append(p.samples), drawn.append(renderer.image.copy())))
    try:
        assert renderer.render_async(scene_for_test(), top_camera()).result(timeout=120) is True
        assert len(drawn) > 1
        assert np.array_equal(drawn[-1], _gpu_raytrace(scene_for_test(), top_camera(), 20, 12, 2))
        assert progress[0] == 0
        p = renderer.progress
        assert (p.samples, p.max_samples, p.done, p.stopped) == (2, 2, True, False)
        assert p.elapsed >= 0
    finally:
        renderer.dispose()


@pytest.mark.gpu
def test_renderer_reports_a_stopped_render():  # progressive.test.ts:222-236
    # 10^8 samples of 240 pixels: far more than the GPU traces before stop() comes.
    renderer = RaytracingRenderer(samples=10 ** 8, preview_block=1)
    renderer.set_size(20, 12)
    states = []
    renderer.on_progress(lambda p: states.append("stopped" if p.stopped else "done" if p.done else "rendering"))
    try:
        result = renderer.render_async(scene_for_test(), top_camera())
        time.sleep(0.3)
        renderer.stop()
        assert result.result(timeout=120) is False
        assert states[0] == "rendering"
        assert states[-1] == "stopped"
        assert renderer.progress.stopped
    finally:
        renderer.dispose()


@pytest.mark.gpu
def test_renderer_reports_a_failed_render():  # progressive.test.ts:238-248
    def bad(_obj):
        raise ValueError("bad scene")

    renderer = RaytracingRenderer(samples=1, filter=bad)
    renderer.set_size(8, 8)
    try:
        assert renderer.render_async(scene_for_test(), top_camera()).result(timeout=120) is False
        assert renderer.progress.error == "bad scene"
        assert renderer.progress.stopped
    finally:
        renderer.dispose()


@pytest.mark.gpu
def test_renderer_fit_aspect_keeps_camera_proportions():  # progressive.test.ts:264-283
    scene = S.Scene()
    marker = S.Mesh(S.plane_geometry(0.2, 0.2), S.MeshBasicMaterial(color=S.Color(0xffffff)))
    marker.position.x = 1.5
    scene.add(marker)
    renderer = RaytracingRenderer(samples=1, preview_block=1)
    renderer.set_size(40, 20)
    try:
        assert renderer.render_async(scene, top_camera()).result(timeout=120) is True
        assert not (renderer.image.reshape(-1, 4)[:, 3] > 0).any()
        renderer.fit_aspect = True
        assert renderer.render_async(scene, top_camera()).result(timeout=120) is True
        alpha = lambda x, y: renderer.image[(y * 40 + x) * 4 + 3]  # noqa: E731
        assert alpha(35, 10) == 255
        assert alpha(20, 10) == 0
    finally:
        renderer.dispose()


@pytest.mark.gpu
def test_renderer_merges_render_calls():  # progressive.test.ts:285-294
    renderer = RaytracingRenderer(samples=1, preview_block=1)
    renderer.set_size(8, 8)
    scene, camera = scene_for_test(), top_camera()
    try:
        for _ in range(5):
            renderer.render(scene, camera)
        time.sleep(0.2)
        deadline = time.time() + 120
        while renderer.progress.samples < 1 and time.time() < deadline:
            time.sleep(0.05)
        assert renderer.when_done().result(timeout=120) is True
    finally:
        renderer.dispose()
