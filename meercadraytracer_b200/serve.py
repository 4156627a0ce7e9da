"""A serving loop for progressive renders: continuous batching on one GPU.

The reference serves one viewer: a camera move restarts its ProgressiveRenderer
(src/progressive.ts:177-188; RaytracingRenderer.render merges calls per
animation frame, src/RaytracingRenderer.ts:215-228). RenderServer serves many
clients at once over the batch engine (mcrt_batch_* in include/mcrt.h):

  * scenes are compiled and uploaded once and stay resident in HBM (BVH,
    triangles, attributes, textures), whatever the cameras do;
  * each client has at most one live request: a new camera move cancels the
    old request and submits the new one (restart on move);
  * requests are admitted as device memory for their accumulation buffers
    frees up (the engine's arena, sized by `memory_budget`), and requests that
    arrive while others are on the GPU join the next chunk: previews first,
    then passes, so their work overlaps on the device;
  * every request's images are those it would get alone (the engine traces the
    same paths and accumulates each pixel's passes in pass order).

`simulate_clients` drives it with orbiting clients and Poisson camera moves
and reports time-to-preview, time-to-N-spp and Mrays/s.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .batch import EVENT_DONE, EVENT_PREVIEW, EVENT_PROGRESS, BatchRenderer
from .executors import GpuExecutor
from .types import CompiledCamera, CompiledScene, TraceSettings


@dataclass
class ServedRequest:
    """Timeline of one served request (seconds on time.perf_counter's clock)."""

    id: int
    client: int
    scene: str
    arrival: float  # when the camera moved (the request's due time)
    submitted: float
    samples: int
    preview: Optional[float] = None
    progress: Dict[int, float] = field(default_factory=dict)  # passes -> when they were accumulated
    done: Optional[float] = None
    cancelled: Optional[float] = None
    camera: Optional[CompiledCamera] = None
    width: int = 0
    height: int = 0
    image: Optional[np.ndarray] = None  # final RGBA8 (when the server keeps images)


class RenderServer:
    """Continuous batching of progressive renders over resident scenes on one GPU."""

    def __init__(self, device: int = 0, capacity: int = 1 << 22, memory_budget: int = 2 << 30,
                 chunk_paths: int = 0, use_graph: bool = True, progress_images: bool = False,
                 keep_images: bool = False):
        self.device = device
        self.batch = BatchRenderer(device, capacity, memory_budget, use_graph)
        if chunk_paths:
            self.batch.set_chunk(chunk_paths)
        self.progress_images = progress_images
        self.keep_images = keep_images
        self.scenes: Dict[str, Tuple[GpuExecutor, Tuple[int, int], CompiledScene]] = {}
        self.requests: Dict[int, ServedRequest] = {}
        self.live: Dict[int, int] = {}  # client -> its live request id
        # Cancelled requests whose host buffers may still receive a copy from a chunk in
        # flight: kept for two more engine steps (at most two chunks are in flight, and
        # each step finishes the oldest).
        self._retiring: Dict[int, int] = {}
        self.clock: Callable[[], float] = time.perf_counter

    def add_scene(self, name: str, scene: CompiledScene) -> None:
        """Uploads a scene to its own executor; it stays resident until close()."""
        ex = GpuExecutor(self.device)
        versions = ex.load_scene(scene)
        self.scenes[name] = (ex, versions, scene)
        self.batch.adopt(scene, ex)

    def request(self, client: int, scene: str, camera: CompiledCamera, width: int, height: int,
                settings: TraceSettings, samples: int = 64, preview_block: int = 8, srgb: bool = True,
                arrival: Optional[float] = None) -> int:
        """A camera move of `client`: cancels its live request and submits a new one."""
        now = self.clock()
        old = self.live.pop(client, None)
        if old is not None:
            self.batch.cancel(old)
            r = self.requests.get(old)
            if r is not None and r.done is None:
                r.cancelled = now
            self._retiring[old] = 2
        ex, versions, _ = self.scenes[scene]
        rid = self.batch.submit_to(ex, versions, camera, settings, width, height, samples, preview_block, srgb,
                                   progress=self.progress_images)
        self.requests[rid] = ServedRequest(rid, client, scene, now if arrival is None else arrival, now, samples,
                                           camera=camera, width=width, height=height)
        self.live[client] = rid
        return rid

    def poll(self) -> Tuple[List[Tuple[int, int, int]], bool]:
        """One engine step: launches the next chunk, collects finished events, stamps them."""
        events, idle = self.batch.step()
        now = self.clock()
        for rid, kind, n in events:
            r = self.requests.get(rid)
            if r is None:
                continue
            if kind == EVENT_PREVIEW:
                r.preview = now
            elif kind == EVENT_PROGRESS:
                r.progress.setdefault(int(n), now)
            elif kind == EVENT_DONE:
                r.done = now
                r.progress.setdefault(int(n), now)
                if self.live.get(r.client) == rid:
                    del self.live[r.client]
                if self.keep_images:
                    r.image = self.batch.result(rid)
                self.batch.forget(rid)
        for rid in list(self._retiring):
            self._retiring[rid] -= 1
            if self._retiring[rid] <= 0:
                del self._retiring[rid]
                self.batch.forget(rid)
        return events, idle

    def stats(self) -> Dict[str, Any]:
        return self.batch.stats()

    def close(self) -> None:
        self.batch.dispose()
        for ex, _, _ in self.scenes.values():
            ex.dispose()
        self.scenes.clear()


# --------------------------------------------------------------- simulation
@dataclass
class Client:
    """A viewer orbiting a scene: camera on a circle, `speed` degrees per second."""

    scene: str
    radius: float
    height: float
    target: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    speed: float = 30.0
    phase: float = 0.0


def _pct(values: Sequence[float], q: float) -> Optional[float]:
    if not values:
        return None
    return float(np.percentile(np.asarray(values, np.float64), q))


def arrival_times(clients: int, duration: float, mean_interval: float, seed: int) -> List[Tuple[float, int]]:
    """Seeded Poisson camera moves: (time, client), sorted; every client moves at t = 0."""
    rng = np.random.default_rng(seed)
    out: List[Tuple[float, int]] = []
    for c in range(clients):
        t = 0.0
        while t < duration:
            out.append((t, c))
            t += float(rng.exponential(mean_interval))
    out.sort()
    return out


def simulate_clients(server: RenderServer, clients: Sequence[Client], settings: Dict[str, TraceSettings],
                     duration: float = 10.0, mean_interval: float = 0.1, width: int = 1280, height: int = 720,
                     samples: int = 64, preview_block: int = 8, seed: int = 0x5EED0003,
                     camera_at: Optional[Callable[[Client, float], CompiledCamera]] = None,
                     settle: bool = True, thresholds: Sequence[int] = (1, 4, 16, 64)) -> Dict[str, Any]:
    """Runs the clients in real time for `duration` seconds, then (settle) lets the last
    request of each client run to completion with no further moves.

    Returns p50 / p99 time-to-preview over every request that got a preview, time-to-N-spp
    for each threshold over the requests that reached it (the request's due time to the
    host seeing the event), the counts, and the rays traced per second of wall time."""
    if camera_at is None:
        from .compile import compile_camera
        from .scenes import orbit_camera

        def camera_at(c: Client, t: float) -> CompiledCamera:
            return compile_camera(orbit_camera(c.radius, c.height, c.phase + c.speed * t, c.target,
                                               aspect=width / height))

    moves = arrival_times(len(clients), duration, mean_interval, seed)
    st0 = server.stats()
    t0 = server.clock()
    server.requests.clear()
    i = 0
    while True:
        now = server.clock() - t0
        while i < len(moves) and moves[i][0] <= now:
            t, c = moves[i]
            cl = clients[c]
            server.request(c, cl.scene, camera_at(cl, t), width, height, settings[cl.scene], samples,
                           preview_block, arrival=t0 + t)
            i += 1
        if now >= duration:
            break
        _, idle = server.poll()
        if idle and i < len(moves):
            # Nothing to do until the next move: wait for it rather than spin.
            time.sleep(max(0.0, min(0.002, moves[i][0] - (server.clock() - t0))))
    t_moving = server.clock() - t0
    if settle:
        for _ in range(1 << 22):
            _, idle = server.poll()
            if idle:
                break
    else:
        for c in list(server.live):
            rid = server.live.pop(c)
            server.batch.cancel(rid)
            server._retiring[rid] = 2
        for _ in range(1 << 22):
            _, idle = server.poll()
            if idle:
                break
    t_end = server.clock() - t0
    st1 = server.stats()
    reqs = list(server.requests.values())
    rays = (st1["closest_rays"] - st0["closest_rays"]) + (st1["any_rays"] - st0["any_rays"])
    gpu_ms = st1["gpu_ms"] - st0["gpu_ms"]
    ttp = [(r.preview - r.arrival) * 1e3 for r in reqs if r.preview is not None]
    out: Dict[str, Any] = {
        "clients": len(clients), "duration_s": round(t_moving, 3), "wall_s": round(t_end, 3),
        "requests": len(reqs), "previews": len(ttp),
        "completed": sum(1 for r in reqs if r.done is not None),
        "cancelled": sum(1 for r in reqs if r.cancelled is not None),
        "time_to_preview_ms": {"p50": _pct(ttp, 50), "p99": _pct(ttp, 99), "max": max(ttp) if ttp else None},
        "mrays_s": rays / t_end / 1e6 if t_end > 0 else 0.0,
        "rays": int(rays), "gpu_busy": gpu_ms / 1e3 / t_end if t_end > 0 else 0.0,
    }
    for n in thresholds:
        vals = []
        for r in reqs:
            reached = [t for k, t in r.progress.items() if k >= n]
            if reached:
                vals.append((min(reached) - r.arrival) * 1e3)
        out[f"time_to_{n}spp_ms"] = {"p50": _pct(vals, 50), "p99": _pct(vals, 99), "count": len(vals)}
    if settle:
        # Each client's last request: nothing restarts it, so it runs to the full sample count.
        last: Dict[int, ServedRequest] = {}
        for r in reqs:
            if r.client not in last or r.arrival > last[r.client].arrival:
                last[r.client] = r
        settled = [(r.done - r.arrival) * 1e3 for r in last.values() if r.done is not None]
        out["settled_time_to_done_ms"] = {"p50": _pct(settled, 50), "p99": _pct(settled, 99), "count": len(settled)}
    return out


def simulate_clients_plain(server: RenderServer, clients: Sequence[Client], settings: Dict[str, TraceSettings],
                           duration: float = 10.0, mean_interval: float = 0.1, width: int = 1280, height: int = 720,
                           samples: int = 64, preview_block: int = 8, seed: int = 0x5EED0003) -> Dict[str, Any]:
    """The same clients and camera moves served by the plain path, one request at a time:
    each client's latest request, oldest first, gets its block preview (one tile render
    with block `preview_block`, as the reference's ProgressiveRenderer starts) and then,
    unless the client has moved on meanwhile, its full render (one raytraceCompiled call of
    `samples` passes, which cannot be interrupted). Uses the server's resident scenes; no
    batching, no overlap. Returns the same figures as simulate_clients (without settling)."""
    from .compile import compile_camera
    from .scenes import orbit_camera
    from .types import Tile

    moves = arrival_times(len(clients), duration, mean_interval, seed)
    execs = {name: (ex, versions, scene) for name, (ex, versions, scene) in server.scenes.items()}
    for ex, _, _ in execs.values():
        ex.reset_stats()
    clock = server.clock
    t0 = clock()
    latest: Dict[int, Tuple[float, int]] = {}  # client -> (arrival, move index)
    served: List[Dict[str, Any]] = []
    i = 0
    requests = 0
    while True:
        now = clock() - t0
        while i < len(moves) and moves[i][0] <= now:
            latest[moves[i][1]] = (moves[i][0], i)
            requests += 1
            i += 1
        if now >= duration:
            break
        if not latest:
            time.sleep(max(0.0, min(0.002, moves[i][0] - now)) if i < len(moves) else 0.002)
            continue
        c, (t_arr, k) = min(latest.items(), key=lambda kv: kv[1][0])
        del latest[c]
        cl = clients[c]
        ex, (gv, sv), scene = execs[cl.scene]
        cam = compile_camera(orbit_camera(cl.radius, cl.height, cl.phase + cl.speed * t_arr, cl.target,
                                          aspect=width / height))
        rec: Dict[str, Any] = {"arrival": t0 + t_arr, "preview": None, "done": None}
        if preview_block > 1:
            ex.render({"type": "tile", "job": k, "geometry_version": gv, "shading_version": sv, "camera": cam,
                       "settings": settings[cl.scene], "tile": Tile(0, 0, width, height), "width": width,
                       "height": height, "pass": 0, "block": preview_block}).result()
            rec["preview"] = clock()
        # A newer move of this client (arrived while previewing) restarts it: no full render.
        now = clock() - t0
        while i < len(moves) and moves[i][0] <= now:
            latest[moves[i][1]] = (moves[i][0], i)
            requests += 1
            i += 1
        if c not in latest:
            ex.raytrace(scene, cam, width, height, settings[cl.scene], samples, True)
            rec["done"] = clock()
        served.append(rec)
    t_end = clock() - t0
    rays = sum(e.stats()["closest_rays"] + e.stats()["any_rays"] for e, _, _ in execs.values())
    ttp = [(r["preview"] - r["arrival"]) * 1e3 for r in served if r["preview"] is not None]
    ttd = [(r["done"] - r["arrival"]) * 1e3 for r in served if r["done"] is not None]
    return {"clients": len(clients), "wall_s": round(t_end, 3), "requests": requests, "previews": len(ttp),
            "completed": len(ttd),
            "time_to_preview_ms": {"p50": _pct(ttp, 50), "p99": _pct(ttp, 99), "max": max(ttp) if ttp else None},
            "time_to_64spp_ms": {"p50": _pct(ttd, 50), "p99": _pct(ttd, 99), "count": len(ttd)},
            "mrays_s": rays / t_end / 1e6 if t_end > 0 else 0.0, "rays": int(rays)}
