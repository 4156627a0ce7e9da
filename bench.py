"""Benchmark: Mrays/s of the plain GPU path on the mid scene (1920x1080, 64 spp,
GI on, 4 bounces), with the oracle's CPU time of the same workload beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config mid|small]

A step is one full frame: every pass of every pixel, accumulated and encoded
to RGBA8 on the device. Rays are BVH queries: camera and bounce rays
(closest hit) plus shadow rays (any hit). `value` is device time (CUDA events
on the library's stream around each frame) with the scene resident in HBM and
the image left on the device; `e2e` is the public `raytrace_compiled` call
with the image read back to host memory. L2 is flushed between steps.

Multi-GPU: every rank renders its own frame (replicas; the path has no data
exchange), value = all ranks' rays / the slowest rank's time.
`--impl reference` times the reference's algorithm on the host cores: the
reference is TypeScript and no Node.js is installed, so this is the oracle
(a C++ restatement of it) on all host threads, on a bounded sample of pixels.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s (closest-hit + shadow BVH queries per second)"
UNIT = "Mrays/s"
# Algorithmic bytes per BVH query (per node visit: one 32-byte box + reference
# word; per triangle test: 36 bytes of v0, e1, e2), with the visit counts of
# the reference algorithm measured by the oracle on a sample of the same rays.
BOX_BYTES = 32
TRI_BYTES = 36


def dist_env() -> Tuple[int, int, int]:
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks() -> Dict[str, Any]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def load_config(name: str, width: int = 0, height: int = 0, spp: int = 0):
    """The benchmark scene; width / height / spp override its image (for profiling runs)."""
    from meercadraytracer_b200 import scenes

    if name == "small":
        b = scenes.small_scene()
    elif name == "mid":
        b = scenes.mid_scene()
    else:
        raise SystemExit(f"unknown config {name}")
    if width or height or spp:
        b.width = width or b.width
        b.height = height or b.height
        b.options = dict(b.options, samples=spp or b.options["samples"])
        if hasattr(b.camera, "aspect"):
            b.camera.aspect = b.width / b.height
        b.name += f" (resized to {b.width}x{b.height}, {b.options['samples']} spp)"
    return b


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc: Optional[subprocess.Popen] = None
        self.lines: List[str] = []
        self._t: Optional[threading.Thread] = None

    def start(self) -> None:
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()

    def _read(self) -> None:
        assert self.proc and self.proc.stdout
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> Dict[str, Any]:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_sample(compiled, camera, bench, seconds: float, threads: int, seed: int = 1
                  ) -> Dict[str, Any]:
    """Times the oracle on a random pixel subset of the workload (all passes), growing the
    subset until the run takes about `seconds`. Returns rays/s and per-query visit counts."""
    from meercadraytracer_b200.raytrace import as_options, output_srgb, sample_count, trace_settings
    from oracle import cpu

    o = as_options(bench.options)
    st, spp, srgb = trace_settings(o), sample_count(o), output_srgb(o)
    rng = np.random.default_rng(seed)
    total = bench.width * bench.height
    n = 64
    while True:
        idx = rng.choice(total, min(n, total), replace=False)
        px, py = (idx % bench.width).astype(np.int32), (idx // bench.width).astype(np.int32)
        ctr = cpu.oracle_counters()
        t0 = time.perf_counter()
        cpu.render_pixels(compiled, camera, st, bench.width, bench.height, spp, srgb, px, py, threads, ctr)
        dt = time.perf_counter() - t0
        if dt >= seconds * 0.5 or n >= total:
            c = ctr.as_dict()
            rays = c["closest_queries"] + c["any_queries"]
            return {"seconds": dt, "pixels": int(idx.size), "samples": int(idx.size) * spp, "rays": rays,
                    "mrays_s": rays / dt / 1e6, "counters": c, "threads": threads}
        n = int(min(total, n * max(2.0, seconds / max(dt, 1e-3) * 0.8)))


def bytes_per_query(counters: Dict[str, int]) -> Dict[str, float]:
    cq, aq = max(1, counters["closest_queries"]), max(1, counters["any_queries"])
    return {"closest": (BOX_BYTES * counters["closest_boxes"] + TRI_BYTES * counters["closest_tris"]) / cq,
            "any": (BOX_BYTES * counters["any_boxes"] + TRI_BYTES * counters["any_tris"]) / aq}


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    from meercadraytracer_b200.compile import compile_camera, compile_scene
    from oracle import cpu

    bench = load_config(args.config, args.width, args.height, args.spp)
    compiled = compile_scene(bench.scene, builder=cpu.compile_sink)
    cam = compile_camera(bench.camera)
    threads = os.cpu_count() or 1
    vals = []
    for i in range(args.warmup + args.steps):
        r = oracle_sample(compiled, cam, bench, args.ref_seconds, threads, seed=100 + i)
        if i >= args.warmup:
            vals.append(r)
    value = statistics.mean(v["mrays_s"] for v in vals)
    sample = (f"{vals[0]['pixels']} random pixels x all {bench.options['samples']} passes per step "
              f"({vals[0]['rays']} rays, {vals[0]['seconds']:.1f} s), oracle C++ restatement of the reference "
              f"(TypeScript; no Node.js on the box)")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * statistics.mean(v["seconds"] for v in vals), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded scene)", "config": {"workload": bench.name},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def combine_over_ranks(device_ms: float, rays: float, dist: Any, device: str) -> Tuple[float, float]:
    """Whole-job figures of a replicated run: the slowest rank's device time and every
    rank's rays (each rank renders its own frame; there is no data exchange). Without a
    process group, this rank's own figures."""
    if dist is None:
        return float(device_ms), float(rays)
    import torch

    t = torch.tensor([float(device_ms), float(rays)], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tsum[1])


def run_ours(args, rank: int, world: int, local: int) -> None:
    import ctypes as C

    import torch

    from meercadraytracer_b200 import abi
    from meercadraytracer_b200.compile import compile_camera, compile_shading, flatten_meshes
    from meercadraytracer_b200.executors import GpuExecutor
    from meercadraytracer_b200.raytrace import as_options, output_srgb, raytrace_compiled, sample_count, trace_settings
    from meercadraytracer_b200.types import CompiledScene

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod

    bench = load_config(args.config, args.width, args.height, args.spp)
    o = as_options(bench.options)
    st, spp, srgb = trace_settings(o), sample_count(o), output_srgb(o)
    ex = GpuExecutor(local)
    if args.capacity:
        ex.set_capacity(args.capacity)
    t0 = time.perf_counter()
    shading, meshes = compile_shading(bench.scene)
    ids = {id(m): i for i, m in enumerate(shading.material_objects)}
    sink = flatten_meshes(meshes, lambda m: ids.get(id(m), 0))
    t_flat = time.perf_counter() - t0
    t0 = time.perf_counter()
    geometry = ex.compile_sink(sink)
    t_build = time.perf_counter() - t0
    compiled = CompiledScene(geometry, shading.materials, shading.textures, shading.environments, shading.lights,
                             shading.background, shading.environment, shading.fog)
    cam = compile_camera(bench.camera)
    t0 = time.perf_counter()
    ex.load_scene(compiled)
    t_upload = time.perf_counter() - t0
    w, h = bench.width, bench.height
    image = torch.empty(w * h * 4, dtype=torch.uint8, device=f"cuda:{local}")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def frame() -> None:
        ex.raytrace_device(compiled, cam, w, h, st, spp, srgb, image.data_ptr())

    tuned: Dict[str, Any] = {}
    if not args.no_tune:
        # The autotuner picks the traversal variant on the same scene and image at an eighth
        # of the samples, then the path pool at the full sample count (outside the timed region).
        from meercadraytracer_b200 import autotune

        choice = autotune.tune_plain(ex, compiled, cam, st, w, h, max(2, spp // 8),
                                     capacities=(1 << 23, 1 << 24, 1 << 25) if not args.capacity else (args.capacity,),
                                     capacity_samples=spp)
        tuned = {"block": choice.block, "stack": choice.stack, "capacity": choice.capacity,
                 "timings_ms": choice.timings}
    for _ in range(args.warmup):
        frame()
    # Timed region: K frames, device time from the library's CUDA events.
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ex.reset_stats()
    clocks = ClockSampler(local)
    clocks.start()
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        frame()
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    s = ex.stats()
    device_ms = s["ms_total"]
    rays = s["closest_rays"] + s["any_rays"]
    device_ms, all_rays = combine_over_ranks(device_ms, rays, dist, f"cuda:{local}")
    value = all_rays / (device_ms / 1000.0) / 1e6
    launches = int(s["launches"])

    e2e = None
    kernels = None
    top = "extend"
    k: Dict[str, Any] = {}
    if not args.no_e2e:
        # End to end through the public API: host image read back every step.
        ex.reset_stats()
        e2e_times = []
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            res = raytrace_compiled(compiled, cam, w, h, o, executor=ex)
            e2e_times.append(time.perf_counter() - t1)
        e2e_rays = ex.stats()
        e2e_value = (e2e_rays["closest_rays"] + e2e_rays["any_rays"]) / sum(e2e_times) / 1e6 * world
        e2e = {"value": round(e2e_value, 3), "unit": UNIT,
               "h2d_bytes_per_step": C.sizeof(abi.mcrt_camera) + C.sizeof(abi.mcrt_settings),
               "d2h_bytes_per_step": int(res.data.nbytes),
               "note": "scene resident in HBM (uploaded once per geometry/shading version, as the executor "
                       "protocol ships it); per step the camera and settings go down and the RGBA8 image comes back"}
        # Kernel breakdown of one frame (events around every kernel) for the roofline.
        ex.reset_stats()
        ex.set_timing(True)
        frame()
        ex.set_timing(False)
        k = ex.stats()
        kernels = {name: {"ms": k[f"ms_{name}"], "launches": k[f"n_{name}"]}
                   for name in ("raygen", "extend", "shade", "shadow", "resolve", "accumulate")}
        top = max(("extend", "shadow"), key=lambda n: kernels[n]["ms"])

    if dist:
        dist.barrier()
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        ex.dispose()
        return

    line: Dict[str, Any] = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(device_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene, no dataset)",
        "config": {"workload": bench.name, "triangles": bench.triangles, "width": w, "height": h, "spp": spp,
                   "rays_per_step": rays / args.steps, "l2": "flushed between steps (512 MiB write)",
                   "parallelism": "replicas" if world > 1 else "single GPU", "path_state_bytes": ex.stats()["path_bytes"],
                   "autotuned": tuned,
                   "compile_s": {"flatten_host": round(t_flat, 3), "gpu_bvh_compile": round(t_build, 3),
                                 "upload": round(t_upload, 3)}},
        "wall_s_timed": round(wall, 3),
        # Camera samples (pixels x spp) per second over all ranks, the second figure of the metric.
        "samples_per_s": round(w * h * spp * world / (device_ms / args.steps / 1e3)),
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
        "kernels": kernels,
    }
    peaks = measured_peaks()
    if world == 1 and not args.no_cpu_baseline and kernels is not None:
        from oracle import cpu

        threads = os.cpu_count() or 1
        from meercadraytracer_b200.compile import compile_scene

        base = oracle_sample(compiled, cam, bench, args.cpu_seconds, threads)
        bpq = bytes_per_query(base["counters"])
        rays_k = k["closest_rays"] if top == "extend" else k["any_rays"]
        per_launch_bytes = bpq["closest" if top == "extend" else "any"] * rays_k / max(1, kernels[top]["launches"])
        avg_ms = kernels[top]["ms"] / max(1, kernels[top]["launches"])
        achieved = per_launch_bytes / (avg_ms / 1000.0) / 1e9
        line["roofline"] = {"bound": "hbm", "kernel": f"k_{top}", "achieved": round(achieved, 1),
                            "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
                            "peak_source": peaks["source"], "traffic": traffic_from_profile(top),
                            "bytes_per_query": round(bpq["closest" if top == "extend" else "any"], 1),
                            "algorithmic_bytes_per_launch": round(per_launch_bytes)}
        line["cpu_baseline"] = {"value": round(base["mrays_s"], 3), "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{base['pixels']} random pixels x {spp} passes ({base['rays']} rays, "
                                          f"{base['seconds']:.1f} s) of the same workload on the oracle, a C++ "
                                          f"restatement of the reference's TypeScript path (no Node.js here)"}
    if world == 1 and not args.no_large:
        line["large"] = run_large(local, args.large_count, args.large_frames, tune=not args.no_tune,
                                  capacity=args.capacity, size=args.large_size)
    if world == 1 and not (args.no_batch and args.no_serve):
        # The batched and served forms of the same path, beside the plain number.
        from meercadraytracer_b200 import scenes as SC
        from meercadraytracer_b200.compile import compile_scene as _compile

        small = SC.small_scene()
        extra = {"mid": compiled, "small": _compile(small.scene, builder=ex.compile_sink)}
        if not args.no_batch:
            line["batched"] = run_batched(extra, local, args.batch_capacity)
        if not args.no_serve:
            t0 = time.perf_counter()
            big = SC.mid_scene(seed=SC.SEED_BASE + 13, grid=32, width=1280, height=720)
            extra["big"] = _compile(big.scene, builder=ex.compile_sink)
            extra["soup"] = _compile(SC.soup_scene().scene, builder=ex.compile_sink)
            t_scenes = time.perf_counter() - t0
            line["served"] = run_served(extra, local, args.serve_seconds, args.serve_capacity, args.serve_chunk,
                                        args.serve_target_ms)
            line["served"]["scene_build_s"] = round(t_scenes, 2)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    ex.dispose()


# ------------------------------------------------------------ batched renders
BATCH_RESOLUTIONS = ((256, 256), (512, 512), (640, 480), (1024, 1024))
BATCH_SPP = (4, 16, 64)


def batch_plan(seed: int, count: int = 64) -> List[Tuple[str, Tuple[float, float, float], Tuple[int, int], int]]:
    """The batched workload: `count` requests over the mid and small scenes (50/50), each with
    a camera on a sphere of radius U(10, 30) aimed at the origin, a resolution drawn from
    BATCH_RESOLUTIONS and a sample count from BATCH_SPP."""
    rng = np.random.default_rng(seed)
    plan = []
    for _ in range(count):
        scene = "mid" if rng.uniform() < 0.5 else "small"
        d = rng.normal(size=3)
        d /= max(float(np.linalg.norm(d)), 1e-12)
        pos = tuple(float(v) for v in d * rng.uniform(10.0, 30.0))
        res = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
        spp = BATCH_SPP[int(rng.integers(len(BATCH_SPP)))]
        plan.append((scene, pos, res, spp))
    return plan


def run_batched(compiled: Dict[str, Any], device: int, capacity: int, seed: int = 0x5EED0002) -> Dict[str, Any]:
    """64 requests rendered one by one through the plain path (mcrt_raytrace per request),
    then all together through the batch engine (one wavefront, CUDA-graph bounce loop).
    Both read every image back to the host; the batch's images must equal the plain ones."""
    from meercadraytracer_b200 import scene as S
    from meercadraytracer_b200.batch import BatchRenderer, RenderRequest
    from meercadraytracer_b200.compile import compile_camera
    from meercadraytracer_b200.executors import GpuExecutor
    from meercadraytracer_b200.raytrace import trace_settings

    settings = trace_settings({"global_illumination": True, "max_bounces": 4, "tone_mapping": S.ACESFilmicToneMapping})
    reqs = []
    for scene, pos, (w, h), spp in batch_plan(seed):
        cam = S.PerspectiveCamera(50, w / h, 0.1, 2000)
        cam.position.set(*pos)
        cam.look_at(0, 0, 0)
        cam.update_matrix_world()
        reqs.append(RenderRequest(compiled[scene], compile_camera(cam), w, h, settings, spp))
    renderer = BatchRenderer(device, capacity, memory_budget=4 << 30)
    try:
        # The autotuner picks the batch's traversal variant and chunk size on 8 of the requests.
        from meercadraytracer_b200 import autotune

        choice = autotune.tune_batch(renderer, reqs[:8])
        execs = {id(c): renderer.executor(c) for c in compiled.values()}
        for ex in execs.values():
            ex.set_capacity(capacity)
            ex.set_traversal(choice.block, choice.stack)
        # Warm-up, untimed, to the steady state of both arms: each executor renders its
        # scene's largest request, which grows its path pool to the size the timed loop
        # needs (a pool growth inside the loop would time a multi-GB cudaMalloc); the batch
        # renders the whole list once (graph instantiation, chunk tables sized).
        largest: Dict[int, Any] = {}
        for r in reqs:
            best = largest.get(id(r.scene))
            if best is None or r.width * r.height * r.samples > best.width * best.height * best.samples:
                largest[id(r.scene)] = r
        for r in largest.values():
            execs[id(r.scene)].raytrace(r.scene, r.camera, r.width, r.height, r.settings, r.samples, True)
        renderer.render(reqs)

        def compare(subset: List[Any]) -> Dict[str, Any]:
            # Plain: one raytraceCompiled per request, on executors that already hold the scenes.
            for ex in execs.values():
                ex.reset_stats()
            plain_imgs = []
            t0 = time.perf_counter()
            for r in subset:
                plain_imgs.append(execs[id(r.scene)].raytrace(r.scene, r.camera, r.width, r.height, r.settings,
                                                               r.samples, True))
            plain_wall = time.perf_counter() - t0
            pst = [ex.stats() for ex in execs.values()]
            plain_rays = sum(x["closest_rays"] + x["any_rays"] for x in pst)
            plain_ms = sum(x["ms_total"] for x in pst)
            # Batched: the same requests in one batch.
            st0 = renderer.stats()
            t0 = time.perf_counter()
            imgs = renderer.render(subset)
            batch_wall = time.perf_counter() - t0
            st1 = renderer.stats()
            rays = (st1["closest_rays"] - st0["closest_rays"]) + (st1["any_rays"] - st0["any_rays"])
            gpu_ms = st1["gpu_ms"] - st0["gpu_ms"]
            same = sum(int(np.array_equal(a, b)) for a, b in zip(imgs, plain_imgs))
            near = sum(int(np.abs(a.astype(np.int16) - b.astype(np.int16)).max(initial=0) <= 1)
                       for a, b in zip(imgs, plain_imgs))
            return {
                "requests": len(subset), "samples": int(sum(r.width * r.height * r.samples for r in subset)),
                "rays": int(rays), "plain_rays": int(plain_rays),
                "plain_mrays_s": round(plain_rays / plain_wall / 1e6, 1),
                "plain_device_mrays_s": round(plain_rays / (plain_ms / 1e3) / 1e6, 1),
                "batched_mrays_s": round(rays / batch_wall / 1e6, 1),
                "batched_device_mrays_s": round(rays / (gpu_ms / 1e3) / 1e6, 1),
                "speedup_vs_plain": round((rays / batch_wall) / (plain_rays / plain_wall), 3),
                "plain_wall_s": round(plain_wall, 4), "batched_wall_s": round(batch_wall, 4),
                "chunks": int(st1["chunks"] - st0["chunks"]),
                "graph_launches": int(st1["graph_launches"] - st0["graph_launches"]),
                "images_equal_to_plain": f"{same}/{len(subset)}",
                "images_within_one_level_of_plain": f"{near}/{len(subset)}",
            }

        out = compare(reqs)
        out["workload"] = ("64 requests, mid (1,310,720 tris) / small (22,530 tris) scenes 50/50, cameras on a "
                           "sphere of radius U(10,30) aimed at the origin, resolutions {256^2, 512^2, 640x480, "
                           "1024^2}, spp {4, 16, 64}, GI on, 4 bounces; images read back to the host")
        out["capacity"] = capacity
        out["autotuned"] = {"block": choice.block, "stack": choice.stack, "chunk": choice.chunk,
                            "timings_ms": choice.timings}
        # The requests of at most 512^2 pixels and 16 spp: each alone leaves most of the GPU idle.
        small = [r for r in reqs if r.width * r.height <= 512 * 512 and r.samples <= 16]
        if small:
            out["small_requests"] = compare(small)
        return out
    finally:
        renderer.dispose()


# ------------------------------------------------------------- serving loop
def run_served(compiled: Dict[str, Any], device: int, seconds: float, capacity: int, chunk: int,
               target_ms: float = 32.0) -> Dict[str, Any]:
    """The serving loop: 8 clients, two per resident scene, orbiting at 30 deg/s with Poisson
    camera moves (mean 100 ms); each move restarts the client's request: an 8x8 block preview,
    then 64 spp at 1280x720, GI on, 4 bounces. After `seconds` the moves stop and each
    client's last request runs to 64 spp."""
    from meercadraytracer_b200 import scene as S
    from meercadraytracer_b200.raytrace import trace_settings
    from meercadraytracer_b200.serve import Client, RenderServer, simulate_clients, simulate_clients_plain

    settings = trace_settings({"global_illumination": True, "max_bounces": 4, "tone_mapping": S.ACESFilmicToneMapping})
    orbits = {"small": (17.0, 6.0), "mid": (70.0, 32.0), "big": (130.0, 60.0), "soup": (34.0, 12.0)}
    names = [n for n in ("small", "mid", "big", "soup") if n in compiled]
    clients = [Client(names[i % len(names)], *orbits[names[i % len(names)]], phase=45.0 * i) for i in range(8)]
    server = RenderServer(device, capacity=capacity, memory_budget=2 << 30, chunk_paths=chunk)
    try:
        for n in names:
            server.add_scene(n, compiled[n])
        # The autotuner sizes chunks so one takes about `target_ms` on the slowest scene (a
        # new request's preview waits for at most the chunks in flight), unless given.
        # 32 ms with an 8M-path pool (a chunk fills half of it): p99 time-to-preview near
        # 40 ms (target 50). Measured 12 / 18 / 24 / 32 / 40 ms with 4M / 8M / 16M paths:
        # rays per second grow with the chunk, and 40 ms put p99 at 47 ms.
        from meercadraytracer_b200 import autotune
        from meercadraytracer_b200.batch import RenderRequest
        from meercadraytracer_b200.compile import compile_camera
        from meercadraytracer_b200.scenes import orbit_camera

        if not chunk:
            probes = [RenderRequest(compiled[c.scene], compile_camera(orbit_camera(c.radius, c.height, c.phase,
                                                                                   aspect=16 / 9)),
                                    1280, 720, settings, 1) for c in clients[: len(names)]]
            chunk = autotune.tune_serving_chunk(server.batch, probes, target_ms=target_ms).chunk
        # Warm-up: one short request per scene (graph instantiation, first-touch).
        simulate_clients(server, clients[: len(names)], {n: settings for n in names}, duration=0.2, width=320,
                         height=180, samples=2, seed=1)
        out = simulate_clients(server, clients, {n: settings for n in names}, duration=seconds)
        # The same clients and moves served by the plain path, one request at a time.
        out["plain_one_at_a_time"] = simulate_clients_plain(server, clients, {n: settings for n in names},
                                                            duration=seconds)
        out["scenes"] = {n: int(compiled[n].geometry.triangle_count) for n in names}
        out["capacity"], out["chunk_paths"] = capacity, chunk
        return out
    finally:
        server.close()


# ------------------------------------------------------ per-frame rebuild
def run_large(device: int, count: int, frames: int, bins: int = 32, tune: bool = True, capacity: int = 0,
              size: int = 0) -> Dict[str, Any]:
    """The large workload: `count` icospheres (20,480 triangles each) under rigid transforms
    re-drawn every frame; each frame compiles the instances on the GPU (flatten, binned-SAH
    BVH with `bins` bins, reorder, tangents) and renders 2048 x 2048 at 16 spp, GI on,
    8 bounces. Two untimed warm-up frames first (allocations); with `tune`, the second
    traces once per traversal variant and the fastest is kept for the timed frames."""
    import torch

    from meercadraytracer_b200 import scenes as SC
    from meercadraytracer_b200.compile import compile_camera
    from meercadraytracer_b200.executors import GpuExecutor
    from meercadraytracer_b200.raytrace import as_options, output_srgb, sample_count, trace_settings

    L = SC.large_scene(count=count, **({"width": size, "height": size} if size else {}))
    o = as_options(L.options)
    st, spp, srgb = trace_settings(o), sample_count(o), output_srgb(o)
    ex = GpuExecutor(device)
    if capacity:
        ex.set_capacity(capacity)
    try:
        free0, total_mem = torch.cuda.mem_get_info(device)
        ex.upload_meshes([L.mesh])
        sv = ex.send_shading_only(L.shading)
        cam = compile_camera(L.camera)
        image = torch.empty(L.width * L.height * 4, dtype=torch.uint8, device=f"cuda:{device}")
        rows = []
        warm = 2
        variant_ms: Dict[str, float] = {}
        for k in range(frames + warm):
            t0 = time.perf_counter()
            instances = L.frame(k)
            t_host = time.perf_counter() - t0
            info, _ = ex.compile_instances(instances, bins=bins)
            if tune and k == warm - 1:
                from meercadraytracer_b200._lib import traversal_variants

                for b_, s_ in traversal_variants():
                    ex.set_traversal(b_, s_)
                    ex.reset_stats()
                    ex.raytrace_resident((info["version"], sv), cam, L.width, L.height, st, spp, srgb,
                                         device_ptr=image.data_ptr())
                    variant_ms[f"{b_}x{s_}"] = round(ex.stats()["ms_total"], 1)
                best = min(variant_ms, key=variant_ms.get)
                ex.set_traversal(*(int(x) for x in best.split("x")))
            ex.reset_stats()
            ex.raytrace_resident((info["version"], sv), cam, L.width, L.height, st, spp, srgb,
                                 device_ptr=image.data_ptr())
            s = ex.stats()
            free1, _ = torch.cuda.mem_get_info(device)
            if k < warm:
                continue  # warm-up: first allocations of the builder, geometry and path buffers
            rays = s["closest_rays"] + s["any_rays"]
            rows.append({"frame": k, "instances_host_ms": round(1e3 * t_host, 2),
                         "build_ms": {"flatten": round(info["flatten_ms"], 2), "bvh": round(info["build_ms"], 2),
                                      "reorder_tangents": round(info["finish_ms"], 2),
                                      "total_with_pack": round(info["total_ms"], 2)},
                         "trace_ms": round(s["ms_total"], 2), "mrays_s": round(rays / (s["ms_total"] / 1e3) / 1e6, 1),
                         "rays": int(rays), "levels": info["levels"], "nodes": info["node_count"],
                         "hbm_bytes": {"geometry": int(info["geometry_bytes"]), "builder": int(info["build_bytes"]),
                                       "path_state": int(s["path_bytes"]), "device_used_by_process": int(free0 - free1)}})
        out = {"workload": L.name, "triangles": L.triangles, "bins": bins, "leaf_size": 4, "frames": rows,
               "hbm_total_bytes": int(total_mem)}
        if variant_ms:
            out["traversal_variant_ms"] = variant_ms
            out["traversal_variant"] = min(variant_ms, key=variant_ms.get)
        return out
    finally:
        ex.dispose()


def traffic_from_profile(kernel: str) -> Optional[float]:
    """DRAM bytes per launch of the kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    entry = d.get(f"k_{kernel}")
    return None if entry is None else float(entry["bytes_per_launch_full_frame"])


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", choices=("mid", "small"), default="mid")
    ap.add_argument("--capacity", type=int, default=0, help="path-state capacity (paths in flight)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="length of the CPU baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=10.0, help="length of each reference-arm step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end and kernel-breakdown passes")
    ap.add_argument("--width", type=int, default=0, help="override the image width (profiling runs)")
    ap.add_argument("--height", type=int, default=0, help="override the image height (profiling runs)")
    ap.add_argument("--spp", type=int, default=0, help="override samples per pixel (profiling runs)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-renders comparison")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default variant and pool)")
    ap.add_argument("--no-large", action="store_true", help="skip the per-frame rebuild workload")
    ap.add_argument("--large-count", type=int, default=4096, help="icospheres of the per-frame rebuild workload")
    ap.add_argument("--large-frames", type=int, default=2, help="timed frames of the per-frame rebuild workload")
    ap.add_argument("--large-only", action="store_true",
                    help="run only the per-frame rebuild workload and print its record (profiling runs)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop run")
    ap.add_argument("--batch-capacity", type=int, default=1 << 26,
                    help="path pool of the batch engine (two chunks of half of it run at once)")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="length of the served client simulation")
    ap.add_argument("--serve-capacity", type=int, default=1 << 23,
                    help="path pool of the serving loop (two chunks of half of it run at once)")
    ap.add_argument("--serve-chunk", type=int, default=0, help="paths per chunk in the serving loop (0: autotuned)")
    ap.add_argument("--serve-target-ms", type=float, default=32.0,
                    help="serving chunk autotune: device time of one chunk on the slowest resident scene")
    ap.add_argument("--large-size", type=int, default=0, help="image side of the per-frame rebuild workload "
                                                              "(0: 2048; smaller for profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be at least 3")
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
    elif args.large_only:
        if rank == 0:
            print(json.dumps({"large": run_large(local, args.large_count, args.large_frames, tune=not args.no_tune,
                                                 capacity=args.capacity, size=args.large_size)}), flush=True)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
