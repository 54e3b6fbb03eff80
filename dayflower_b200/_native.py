"""ctypes loading of the in-tree native libraries.

The render path has no fallback: if ``libdayflower_cuda.so`` cannot be built
or loaded, :func:`load_renderer` raises.
"""
from __future__ import annotations

import ctypes
import threading

from . import build as _build

_lock = threading.Lock()
_cuda = None
_scene = None

_c_int, _c_i64, _c_f, _c_p, _c_u32 = ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_void_p, ctypes.c_uint32

# (name, restype, argtypes) for every entry point in include/dayflower_cuda.h
SIGNATURES = [
    ("dfc_create", _c_int, [_c_int, ctypes.POINTER(_c_p)]),
    ("dfc_destroy", _c_int, [_c_p]),
    ("dfc_last_error", ctypes.c_char_p, [_c_p]),
    ("dfc_scene_put", _c_int, [_c_p, ctypes.c_char_p, _c_p, _c_i64, _c_int]),
    ("dfc_scene_commit", _c_int, [_c_p, _c_int]),
    ("dfc_set_image", _c_int, [_c_p, _c_int, _c_int]),
    ("dfc_set_maximum_bounce", _c_int, [_c_p, _c_int]),
    ("dfc_set_minimum_bounce_russian_roulette", _c_int, [_c_p, _c_int]),
    ("dfc_set_rendering_algorithm", _c_int, [_c_p, _c_int]),
    ("dfc_set_samples", _c_int, [_c_p, _c_int]),
    ("dfc_set_maximum_distance", _c_int, [_c_p, _c_f]),
    ("dfc_set_tone_mapper", _c_int, [_c_p, _c_int]),
    ("dfc_set_preview_mode", _c_int, [_c_p, _c_int]),
    ("dfc_set_seed", _c_int, [_c_p, _c_u32]),
    ("dfc_set_stage_timing", _c_int, [_c_p, _c_int]),
    ("dfc_setup", _c_int, [_c_p]),
    ("dfc_render", _c_int, [_c_p, _c_int, ctypes.POINTER(_c_int)]),
    ("dfc_render_observed", _c_int, [_c_p, _c_int, _c_p, _c_p, ctypes.POINTER(_c_int)]),
    ("dfc_read_kernel_stats", _c_int, [_c_p, _c_p, _c_p, _c_p, _c_int]),
    ("dfc_render_shutdown", _c_int, [_c_p]),
    ("dfc_clear", _c_int, [_c_p]),
    ("dfc_update_camera", _c_int, [_c_p, _c_p]),
    ("dfc_update_matrices", _c_int, [_c_p, _c_p, _c_i64]),
    ("dfc_read_image_rgba8", _c_int, [_c_p, _c_p, _c_i64]),
    ("dfc_read_film", _c_int, [_c_p, _c_p, _c_i64]),
    ("dfc_set_film_filter", _c_int, [_c_p, _c_int]),
    ("dfc_read_pixel_film", _c_int, [_c_p, _c_p, _c_i64]),
    ("dfc_read_primary_hits", _c_int, [_c_p, _c_p, _c_p, _c_i64]),
    ("dfc_read_counters", _c_int, [_c_p, _c_p]),
    ("dfc_read_stage_times", _c_int, [_c_p, _c_p]),
    ("dfc_read_commit_times", _c_int, [_c_p, _c_p]),
    ("dfc_set_bvh_builder", _c_int, [_c_p, _c_int]),
    ("dfc_engine_set_bvh_builder", _c_int, [_c_p, _c_int]),
    ("dfc_trace_rays_noalloc", _c_int, [_c_p, _c_p, _c_p, _c_p, _c_i64]),
    # batch and serving engine
    ("dfc_engine_create", _c_int, [_c_int, _c_i64, ctypes.POINTER(_c_p)]),
    ("dfc_engine_destroy", _c_int, [_c_p]),
    ("dfc_engine_last_error", ctypes.c_char_p, [_c_p]),
    ("dfc_engine_scene_put", _c_int, [_c_p, ctypes.c_char_p, _c_p, _c_i64, _c_int]),
    ("dfc_engine_scene_commit", _c_int, [_c_p, _c_int, ctypes.POINTER(ctypes.c_int32)]),
    ("dfc_engine_scene_release", _c_int, [_c_p, ctypes.c_int32]),
    ("dfc_engine_configure", _c_int, [_c_p, _c_p]),
    ("dfc_engine_get_config", _c_int, [_c_p, _c_p]),
    ("dfc_engine_autotune", _c_int, [_c_p, _c_p, _c_int, ctypes.c_char_p, ctypes.c_char_p, _c_p]),
    ("dfc_job_submit", _c_int, [_c_p, _c_p, ctypes.POINTER(_c_i64)]),
    ("dfc_job_get_info", _c_int, [_c_p, _c_i64, _c_p]),
    ("dfc_job_wait", _c_int, [_c_p, _c_i64, ctypes.c_double]),
    ("dfc_job_cancel", _c_int, [_c_p, _c_i64]),
    ("dfc_job_read_film", _c_int, [_c_p, _c_i64, _c_p, _c_i64]),
    ("dfc_job_read_image_rgba8", _c_int, [_c_p, _c_i64, _c_int, _c_p, _c_i64]),
    ("dfc_job_release", _c_int, [_c_p, _c_i64]),
    ("dfc_engine_run", _c_int, [_c_p, ctypes.c_double]),
    ("dfc_engine_start", _c_int, [_c_p]),
    ("dfc_engine_stop", _c_int, [_c_p]),
    ("dfc_engine_get_stats", _c_int, [_c_p, _c_p]),
]


class PassEvent(ctypes.Structure):
    """``dfc_pass_event`` of ``dfc_render_observed``."""
    _fields_ = [("event", _c_int), ("render_pass", _c_int), ("progress", ctypes.c_double), ("millis", ctypes.c_double),
                ("rgba", ctypes.POINTER(ctypes.c_uint8)), ("width", _c_int), ("height", _c_int)]


OBSERVER_FN = ctypes.CFUNCTYPE(None, _c_p, ctypes.POINTER(PassEvent))


def load_renderer(build: bool = True) -> ctypes.CDLL:
    """Loads libdayflower_cuda.so (building it first if sources changed)."""
    global _cuda
    with _lock:
        if _cuda is None:
            path = _build.build_cuda() if build else _build.cuda_lib_path()
            lib = ctypes.CDLL(path)
            for name, res, args in SIGNATURES:
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _cuda = lib
        return _cuda


def load_scene_compiler() -> ctypes.CDLL:
    """Loads the scene-compiler host helper (libdayflower_scene.so)."""
    global _scene
    with _lock:
        if _scene is None:
            lib = ctypes.CDLL(_build.build_scene())
            lib.dfc_sc_build_mesh_bvh.restype = ctypes.c_longlong
            lib.dfc_sc_build_mesh_bvh.argtypes = [_c_p, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong, _c_p, _c_p,
                                                  ctypes.c_longlong]
            _scene = lib
        return _scene
