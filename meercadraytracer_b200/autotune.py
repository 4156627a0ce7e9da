"""Autotuner for the wavefront's launch parameters.

Three things are picked by timing short runs of the real workload on the
device, not by rules of thumb:

  * the traversal kernels' variant: threads per block and shared-memory
    short-stack entries per thread (the closest-hit and shadow kernels are
    compiled for several pairs, _lib.traversal_variants());
  * the path pool (queue size): paths in flight per launch series;
  * for the serving loop, the chunk size: the most paths one chunk may hold so
    that a chunk takes about `target_ms` on the slowest scene, which bounds
    how long a new request's preview waits behind the work in flight.

Choices never change results (every variant traces the same paths and
accumulates them in the same order); only time does. Results are cached in
memory per device and workload key, and in a JSON file when `cache_path` is
given.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import asdict, dataclass, field
from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple

from ._lib import traversal_variants
from .types import CompiledCamera, CompiledScene, TraceSettings

_memory: Dict[str, Dict[str, Any]] = {}


@dataclass
class Choice:
    """A tuned configuration and the timings it was chosen from (ms per run)."""

    block: int
    stack: int
    capacity: int
    chunk: int = 0
    timings: Dict[str, float] = field(default_factory=dict)

    def as_dict(self) -> Dict[str, Any]:
        return asdict(self)


def device_name(device: int = 0) -> str:
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:  # pragma: no cover - torch without CUDA
        return f"cuda:{device}"


def _load(cache_path: Optional[str], key: str) -> Optional[Dict[str, Any]]:
    if key in _memory:
        return _memory[key]
    if cache_path and os.path.exists(cache_path):
        try:
            with open(cache_path) as f:
                d = json.load(f)
            if key in d:
                _memory[key] = d[key]
                return d[key]
        except (OSError, ValueError):
            return None
    return None


def _store(cache_path: Optional[str], key: str, value: Dict[str, Any]) -> None:
    _memory[key] = value
    if not cache_path:
        return
    d: Dict[str, Any] = {}
    if os.path.exists(cache_path):
        try:
            with open(cache_path) as f:
                d = json.load(f)
        except (OSError, ValueError):
            d = {}
    d[key] = value
    os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
    tmp = cache_path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, cache_path)


def _best(timings: Dict[Any, float]) -> Any:
    return min(timings, key=lambda k: timings[k])


def tune_plain(executor: Any, scene: CompiledScene, camera: CompiledCamera, settings: TraceSettings, width: int,
               height: int, samples: int, capacities: Sequence[int] = (1 << 23, 1 << 24, 1 << 25),
               variants: Optional[Sequence[Tuple[int, int]]] = None, repeats: int = 2,
               key: Optional[str] = None, cache_path: Optional[str] = None,
               capacity_samples: Optional[int] = None) -> Choice:
    """Tunes an executor for raytraceCompiled on `scene`: each traversal variant is timed on
    the workload at the largest capacity, then the capacities with the best variant, at
    `capacity_samples` samples per pixel (default `samples`): a frame takes every pass of as
    many pixels as the pool holds, so the pool decides how many chunks a frame of the full
    sample count takes, which fewer samples do not show. The executor is left set to the
    choice. Times are device times of whole renders."""
    cap_spp = capacity_samples or samples
    key = key or (f"plain|{device_name(executor.device)}|{scene.geometry.triangle_count}|"
                  f"{width}x{height}x{samples}x{cap_spp}")
    hit = _load(cache_path, key)
    if hit is not None:
        choice = Choice(**hit)
        executor.set_traversal(choice.block, choice.stack)
        executor.set_capacity(choice.capacity)
        return choice

    def timed(spp: int = samples) -> float:
        best = float("inf")
        for _ in range(max(1, repeats)):
            executor.reset_stats()
            executor.raytrace(scene, camera, width, height, settings, spp, True)
            best = min(best, executor.stats()["ms_total"])
        return best

    variants = list(variants or traversal_variants())
    executor.set_capacity(max(capacities))
    executor.raytrace(scene, camera, width, height, settings, 1, True)  # warm-up: scene resident, buffers sized
    tv: Dict[Tuple[int, int], float] = {}
    for b, s in variants:
        executor.set_traversal(b, s)
        tv[(b, s)] = timed()
    block, stack = _best(tv)
    executor.set_traversal(block, stack)
    tc: Dict[int, float] = {}
    for c in capacities:
        executor.set_capacity(c)
        tc[c] = timed(cap_spp)
    capacity = _best(tc)
    executor.set_capacity(capacity)
    timings = {f"variant {b}x{s}": round(t, 3) for (b, s), t in tv.items()}
    timings.update({f"capacity {c}": round(t, 3) for c, t in tc.items()})
    choice = Choice(block, stack, capacity, 0, timings)
    _store(cache_path, key, choice.as_dict())
    return choice


def tune_batch(renderer: Any, requests: Sequence[Any], chunks: Optional[Sequence[int]] = None,
               variants: Optional[Sequence[Tuple[int, int]]] = None, key: Optional[str] = None,
               cache_path: Optional[str] = None) -> Choice:
    """Tunes a BatchRenderer on a sample of its requests: the traversal variant, then the
    chunk size (paths per chunk, up to the engine's pool). The renderer is left set."""
    capacity = int(renderer.capacity)
    key = key or f"batch|{device_name(renderer.device)}|{capacity}|{len(requests)}|" + ",".join(
        f"{r.scene.geometry.triangle_count}:{r.width}x{r.height}x{r.samples}" for r in requests[:8])
    hit = _load(cache_path, key)
    if hit is not None:
        choice = Choice(**hit)
        renderer.set_traversal(choice.block, choice.stack)
        renderer.set_chunk(choice.chunk)
        return choice

    def timed() -> float:
        s0 = renderer.stats()
        renderer.render(requests)
        return renderer.stats()["gpu_ms"] - s0["gpu_ms"]

    variants = list(variants or traversal_variants())
    renderer.render(requests[:1])  # warm-up: graph, scenes resident
    tv: Dict[Tuple[int, int], float] = {}
    for b, s in variants:
        renderer.set_traversal(b, s)
        tv[(b, s)] = timed()
    block, stack = _best(tv)
    renderer.set_traversal(block, stack)
    half = capacity // 2  # two chunks share the pool
    chunks = [c for c in (chunks or (half // 4, half // 2, half)) if 0 < c <= half]
    tc: Dict[int, float] = {}
    for c in chunks:
        renderer.set_chunk(c)
        tc[c] = timed()
    chunk = _best(tc)
    renderer.set_chunk(chunk)
    timings = {f"variant {b}x{s}": round(t, 3) for (b, s), t in tv.items()}
    timings.update({f"chunk {c}": round(t, 3) for c, t in tc.items()})
    choice = Choice(block, stack, capacity, chunk, timings)
    _store(cache_path, key, choice.as_dict())
    return choice


def tune_serving_chunk(renderer: Any, probes: Sequence[Any], target_ms: float = 12.0, key: Optional[str] = None,
                       cache_path: Optional[str] = None) -> Choice:
    """The serving loop's chunk size: each probe request (one per resident scene, one pass of
    the served resolution) is timed alone with chunks of half the pool (two chunks share it);
    the chunk is the number of paths the slowest scene traces in `target_ms`, rounded down to
    a multiple of 65,536 (at least 262,144, at most half the pool)."""
    capacity = int(renderer.capacity) // 2
    key = key or f"serve|{device_name(renderer.device)}|{capacity}|{target_ms}|" + ",".join(
        f"{r.scene.geometry.triangle_count}:{r.width}x{r.height}x{r.samples}" for r in probes)
    hit = _load(cache_path, key)
    if hit is not None:
        choice = Choice(**hit)
        renderer.set_chunk(choice.chunk)
        return choice
    renderer.set_chunk(capacity)
    per_path: Dict[str, float] = {}
    for i, r in enumerate(probes):
        renderer.render([r])  # warm-up
        s0 = renderer.stats()
        renderer.render([r])
        ms = renderer.stats()["gpu_ms"] - s0["gpu_ms"]
        per_path[f"probe {i} ({r.scene.geometry.triangle_count} tris) ms/Mpath"] = round(
            ms / (r.width * r.height * r.samples) * 1e6, 4)
    slowest = max(per_path.values()) / 1e6 if per_path else 1e-6
    chunk = int(target_ms / max(slowest, 1e-9))
    chunk = max(1 << 18, min(capacity, (chunk >> 16) << 16))
    renderer.set_chunk(chunk)
    choice = Choice(0, 0, capacity, chunk, per_path)
    _store(cache_path, key, choice.as_dict())
    return choice
