"""The product's geometry builder: compileGeometry's BVH build, reorder,
tangents and epsilon (src/compile.ts:359-432) on the GPU through libmcrt."""
from __future__ import annotations

from typing import Optional

from .compile import TriangleSink
from .types import CompiledGeometry


def build_geometry_gpu(sink: TriangleSink, executor: Optional[object] = None) -> CompiledGeometry:
    from .executors import default_executor

    ex = executor or default_executor()
    return ex.compile_sink(sink)  # type: ignore[attr-defined]
