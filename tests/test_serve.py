"""The serving loop (continuous batching of progressive renders).

CPU: the seeded Poisson schedule of camera moves. GPU: orbiting clients over
two resident scenes, with camera moves restarting requests while others run;
every request that finishes must give the image the plain per-request render
(raytraceCompiled) gives for its camera, byte for byte, and the loop must
return every buffer to its memory budget.
"""
import numpy as np
import pytest

from meercadraytracer_b200 import scenes
from meercadraytracer_b200.compile import compile_camera, compile_scene
from meercadraytracer_b200.raytrace import as_options, trace_settings
from meercadraytracer_b200.serve import Client, RenderServer, arrival_times, simulate_clients
from oracle import cpu


def test_arrival_times_are_seeded_poisson():
    a = arrival_times(8, 20.0, 0.1, seed=5)
    assert a == arrival_times(8, 20.0, 0.1, seed=5)
    assert a == sorted(a)
    assert sorted({c for _, c in a}) == list(range(8))
    assert all(t == 0.0 for t, c in a[:8])  # every client starts at once
    gaps = []
    for c in range(8):
        ts = [t for t, k in a if k == c]
        gaps += list(np.diff(ts))
    assert 0.09 < float(np.mean(gaps)) < 0.11  # mean inter-arrival 100 ms


@pytest.mark.gpu
def test_served_requests_equal_plain_renders():
    small = scenes.small_scene()
    mid = scenes.mid_scene(grid=3, subdivisions=2, width=160, height=90)
    compiled = {name: compile_scene(b.scene, builder=cpu.compile_sink) for name, b in (("small", small), ("mid", mid))}
    gi = trace_settings(as_options({"global_illumination": True, "max_bounces": 4,
                                    "tone_mapping": small.options["tone_mapping"]}))
    settings = {"small": gi, "mid": gi}
    server = RenderServer(capacity=1 << 15, memory_budget=8 << 20, keep_images=True)
    try:
        for name, c in compiled.items():
            server.add_scene(name, c)
        clients = [Client("small", 17.0, 6.0), Client("mid", 14.0, 8.0), Client("small", 20.0, 4.0, phase=90),
                   Client("mid", 12.0, 6.0, phase=180)]
        out = simulate_clients(server, clients, settings, duration=1.0, mean_interval=0.1, width=64, height=36,
                               samples=8, preview_block=8, seed=11)
        assert out["requests"] >= 4 and out["previews"] >= 1
        assert out["time_to_preview_ms"]["p99"] is not None
        assert out["settled_time_to_done_ms"]["count"] == 4
        assert out["mrays_s"] > 0
        done = [r for r in server.requests.values() if r.done is not None]
        assert len(done) >= 4
        for r in done:
            ex, _, scene = server.scenes[r.scene]
            plain = ex.raytrace(scene, r.camera, r.width, r.height, settings[r.scene], r.samples, True)
            assert np.array_equal(r.image, plain)
        st = server.stats()
        assert st["arena_used"] == 0 and st["status"] == 0
    finally:
        server.close()


@pytest.mark.gpu
def test_plain_one_at_a_time_serving_runs_the_same_clients():
    from meercadraytracer_b200.serve import simulate_clients_plain

    small = scenes.small_scene()
    compiled = compile_scene(small.scene, builder=cpu.compile_sink)
    gi = trace_settings(as_options({"global_illumination": True, "max_bounces": 4}))
    server = RenderServer(capacity=1 << 15, memory_budget=8 << 20)
    try:
        server.add_scene("small", compiled)
        clients = [Client("small", 17.0, 6.0), Client("small", 20.0, 4.0, phase=90)]
        out = simulate_clients_plain(server, clients, {"small": gi}, duration=0.5, width=64, height=36, samples=4)
        assert out["requests"] >= 2 and out["previews"] >= 1
        assert out["time_to_preview_ms"]["p50"] is not None and out["rays"] > 0
    finally:
        server.close()
