"""Builds libmcrt.so, the CUDA sm_100a library behind include/mcrt.h, in-tree.

    python -m meercadraytracer_b200.build [--force]

Each .cu file is compiled with nvcc for sm_100a (objects under _build/) and
linked into meercadraytracer_b200/libmcrt.so. scene_build.cu is compiled with
--fmad=false so its double-precision arithmetic rounds exactly as the
reference's JavaScript does.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmcrt.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = {
    "render.cu": [],
    "executor.cu": [],
    "batch.cu": [],
    "scene_build.cu": ["--fmad=false"],
}
HEADERS = ["mcrt_math.cuh", "device_scene.cuh", "traverse.cuh", "render.cuh", "scene_build.cuh", "batch.cuh", "dfg_lut.h"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build libmcrt.so")
    return path


def common_flags() -> List[str]:
    return ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
            f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}", "--expt-relaxed-constexpr"]


def _stale(target: str, deps: List[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra: List[str] = ()) -> str:
    """Compiles and links libmcrt.so if a source changed; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "mcrt.h"),
                                                          os.path.join(ROOT, "include", "mcrt_types.h")]
    objects = []
    commands = []
    for src, flags in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objects.append(obj)
        if force or _stale(obj, [path, *headers]):
            commands.append([nvcc(), *common_flags(), *flags, *extra, "-c", path, "-o", obj])
    changed = force or bool(commands)
    # The translation units are independent: compile them side by side.
    with ThreadPoolExecutor(max_workers=max(1, min(len(commands), os.cpu_count() or 1))) as pool:
        for cmd in commands:
            if verbose:
                print(" ".join(cmd), flush=True)
        for r in list(pool.map(lambda c: subprocess.run(c, capture_output=not verbose, text=True), commands)):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed: {' '.join(r.args)}\n{r.stdout or ''}{r.stderr or ''}")
            if extra and r.stderr:
                print(r.stderr, flush=True)
    if changed or _stale(LIB, objects):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objects, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv: List[str] = None) -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else []
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose, extra=extra))


if __name__ == "__main__":
    main(sys.argv[1:])
