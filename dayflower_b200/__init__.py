"""dayflower_b200: a B200 (sm_100a) render path that stands in for Dayflower's
``GPURenderer``.

The renderer is ``libdayflower_cuda.so`` (C ABI in ``include/dayflower_cuda.h``);
this package holds its Python bindings (:class:`GPURenderer`, the per-job
drop-in, and :class:`RenderEngine`, the batch/serving engine), the scene model
and compiler that produce the compiled-scene arrays it consumes, and the
synthetic scene generators used by the tests and the benchmark.
"""
from .engine import RenderEngine  # noqa: F401
from .renderer import GPURenderer, RenderError, RenderingAlgorithm, UnsupportedSceneError  # noqa: F401

__all__ = ["GPURenderer", "RenderEngine", "RenderError", "RenderingAlgorithm", "UnsupportedSceneError"]
