"""``RenderEngine``: many path-tracing jobs in one wavefront on one GPU.

The reference renders one image per ``GPURenderer`` (one pass per Aparapi
``execute``, renderer/gpu/AbstractGPURenderer.java:231-297).  A job here is
what one ``GPURenderer`` would do for ``setScene`` + ``setImage(w, h)`` +
``setMaximumBounce`` + ``setMinimumBounceRussianRoulette`` + ``setup()`` +
``render(samples)`` in PATH_TRACING, with the same random numbers for the same
seed.  The engine keeps scenes resident (reference-counted), admits jobs
against a device-memory budget, starts their paths in free path slots at every
bounce iteration and replays the iteration loop as a CUDA graph.

Two ways to drive it:

* batched: ``submit`` jobs, then ``run()`` renders until all are finished in
  the calling thread;
* served: ``start()`` runs the wavefront on an engine thread; ``submit`` from
  any thread, ``wait``/``info`` for completion and latency, ``film`` for a
  progressive image while a job runs, ``stop()`` to end.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Optional

import numpy as np

from . import _native
from .renderer import DFC_E_INVALID_ARG, DFC_E_OOM, DFC_E_TIMEOUT, DFC_E_UNSUPPORTED, DFC_OK, RenderError, UnsupportedSceneError
from .scene.compiler import CompiledScene, compile_scene
from .scene.model import Scene

JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_CANCELLED, JOB_FAILED = range(5)
JOB_STATE_NAMES = {JOB_QUEUED: "queued", JOB_RUNNING: "running", JOB_DONE: "done", JOB_CANCELLED: "cancelled", JOB_FAILED: "failed"}


class JobDesc(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_int32), ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("samples", ctypes.c_int32),
                ("maximum_bounce", ctypes.c_int32), ("minimum_bounce_russian_roulette", ctypes.c_int32),
                ("seed", ctypes.c_uint32), ("kind", ctypes.c_int32), ("ambient_occlusion_samples", ctypes.c_int32),
                ("maximum_distance", ctypes.c_float)]


# dfc_job_desc.kind: the RenderingAlgorithm of the job (GPURenderer.run dispatches on it, GPURenderer.java:65-77)
JOB_PATH_TRACING, JOB_RAY_CASTING, JOB_DEPTH_CAMERA, JOB_AMBIENT_OCCLUSION, JOB_RAY_TRACING = 0, 1, 2, 3, 4


class JobInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("scene", ctypes.c_int32), ("paths_total", ctypes.c_int64), ("paths_done", ctypes.c_int64),
                ("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double)]


SCHEDULE_ROUND_ROBIN, SCHEDULE_FIFO, SCHEDULE_SHORTEST_FIRST = 0, 1, 2


class EngineConfig(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int64), ("trace_blocks_per_sm", ctypes.c_int32), ("shade_blocks_per_sm", ctypes.c_int32),
                ("shade_threads", ctypes.c_int32), ("iterations_per_launch", ctypes.c_int32), ("policy", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("segment_paths", ctypes.c_int64), ("lookahead_paths", ctypes.c_int64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class EngineStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("graph_launches", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("paths_retired", ctypes.c_int64), ("rays", ctypes.c_int64), ("jobs_submitted", ctypes.c_int64),
                ("jobs_done", ctypes.c_int64), ("device_bytes_used", ctypes.c_int64), ("device_bytes_budget", ctypes.c_int64),
                ("overflow", ctypes.c_int64), ("busy_s", ctypes.c_double)]

    def as_dict(self):
        return {k: (float(getattr(self, k)) if k == "busy_s" else int(getattr(self, k))) for k, _ in self._fields_}


class RenderEngine:
    """Batch and serving engine over ``libdayflower_cuda``'s ``dfc_engine_*`` API."""

    def __init__(self, device: int = 0, memory_budget_bytes: int = 0):
        self._lib = _native.load_renderer()
        h = ctypes.c_void_p()
        rc = self._lib.dfc_engine_create(int(device), int(memory_budget_bytes), ctypes.byref(h))
        if rc != DFC_OK:
            raise RenderError(rc, "dfc_engine_create failed (device %d)" % device)
        self._h = h
        self._jobs = {}  # id -> (width, height)

    # -- helpers ---------------------------------------------------------------
    def _check(self, rc: int):
        if rc == DFC_OK:
            return
        msg = (self._lib.dfc_engine_last_error(self._h) or b"").decode()
        if rc == DFC_E_INVALID_ARG:
            raise ValueError(msg)
        if rc == DFC_E_UNSUPPORTED:
            raise UnsupportedSceneError(rc, msg)
        if rc == DFC_E_OOM:
            raise MemoryError(msg)
        if rc == DFC_E_TIMEOUT:
            raise TimeoutError(msg)
        raise RenderError(rc, msg)

    def close(self):
        if getattr(self, "_h", None) is not None:
            self._lib.dfc_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- scenes ------------------------------------------------------------------
    def add_scene(self, scene, layout_version: Optional[int] = None) -> int:
        """Uploads a scene (model or compiled) and returns its id."""
        if scene is None:
            raise TypeError("scene == null")
        if isinstance(scene, Scene):
            scene = compile_scene(scene, layout_version or 1)
        cs: CompiledScene = scene
        for name, arr in cs.arrays.items():
            a = np.ascontiguousarray(arr)
            typ = 1 if a.dtype == np.int32 else 0
            if typ == 0 and a.dtype != np.float32:
                a = a.astype(np.float32)
            self._check(self._lib.dfc_engine_scene_put(self._h, name.encode(), a.ctypes.data_as(ctypes.c_void_p), a.size, typ))
        sid = ctypes.c_int32(-1)
        self._check(self._lib.dfc_engine_scene_commit(self._h, int(layout_version or cs.layout_version), ctypes.byref(sid)))
        return int(sid.value)

    def release_scene(self, scene_id: int):
        self._check(self._lib.dfc_engine_scene_release(self._h, int(scene_id)))

    def set_bvh_builder(self, builder: int):
        """Builder of the mesh hierarchies of later ``add_scene`` calls (0 host SAH, 1 device)."""
        self._check(self._lib.dfc_engine_set_bvh_builder(self._h, int(builder)))

    # -- configuration -------------------------------------------------------------
    def configure(self, capacity=0, trace_blocks_per_sm=0, shade_blocks_per_sm=0, shade_threads=0, iterations_per_launch=0,
                  policy=SCHEDULE_ROUND_ROBIN, segment_paths=0, lookahead_paths=0, reserved=0):
        """Wavefront shape and scheduling (0 keeps a field's default); takes effect at the next run."""
        c = EngineConfig(int(capacity), int(trace_blocks_per_sm), int(shade_blocks_per_sm), int(shade_threads), int(iterations_per_launch),
                         int(policy), 0, int(segment_paths), int(lookahead_paths))
        self._check(self._lib.dfc_engine_configure(self._h, ctypes.byref(c)))

    def config(self) -> dict:
        c = EngineConfig()
        self._check(self._lib.dfc_engine_get_config(self._h, ctypes.byref(c)))
        return c.as_dict()

    def autotune(self, jobs: Iterable[dict], cache_path: Optional[str] = None, key: str = "") -> dict:
        """Times candidate wavefront shapes on the sample jobs and keeps the fastest."""
        descs = [self._desc(**j) for j in jobs]
        arr = (JobDesc * len(descs))(*descs)
        out = EngineConfig()
        self._check(self._lib.dfc_engine_autotune(self._h, arr, len(descs), cache_path.encode() if cache_path else None,
                                                  key.encode(), ctypes.byref(out)))
        return out.as_dict()

    # -- jobs ----------------------------------------------------------------------
    @staticmethod
    def _desc(scene, width, height, samples, maximum_bounce=20, minimum_bounce_russian_roulette=5, seed=0x5EED1234,
              kind=JOB_PATH_TRACING, ambient_occlusion_samples=10, maximum_distance=20.0):
        return JobDesc(int(scene), int(width), int(height), int(samples), int(maximum_bounce), int(minimum_bounce_russian_roulette),
                       int(seed) & 0xFFFFFFFF, int(kind), int(ambient_occlusion_samples), float(maximum_distance))

    def submit(self, scene: int, width: int, height: int, samples: int, maximum_bounce: int = 20,
               minimum_bounce_russian_roulette: int = 5, seed: int = 0x5EED1234, kind: int = JOB_PATH_TRACING,
               ambient_occlusion_samples: int = 10, maximum_distance: float = 20.0) -> int:
        """Queues a job of any rendering algorithm (``kind``: JOB_PATH_TRACING, JOB_RAY_CASTING,
        JOB_DEPTH_CAMERA, JOB_AMBIENT_OCCLUSION with its samples and maximum distance, or
        JOB_RAY_TRACING); returns its id.  ``samples`` is the render(samples) pass count."""
        d = self._desc(scene, width, height, samples, maximum_bounce, minimum_bounce_russian_roulette, seed, kind,
                       ambient_occlusion_samples, maximum_distance)
        jid = ctypes.c_int64(0)
        self._check(self._lib.dfc_job_submit(self._h, ctypes.byref(d), ctypes.byref(jid)))
        self._jobs[int(jid.value)] = (int(width), int(height))
        return int(jid.value)

    def info(self, job: int) -> dict:
        i = JobInfo()
        self._check(self._lib.dfc_job_get_info(self._h, int(job), ctypes.byref(i)))
        return {"state": JOB_STATE_NAMES.get(i.state, str(i.state)), "scene": int(i.scene), "paths_total": int(i.paths_total),
                "paths_done": int(i.paths_done), "submit_s": float(i.submit_s), "admit_s": float(i.admit_s), "done_s": float(i.done_s)}

    def wait(self, job: int, timeout_s: float = 0.0):
        self._check(self._lib.dfc_job_wait(self._h, int(job), float(timeout_s)))

    def cancel(self, job: int):
        self._check(self._lib.dfc_job_cancel(self._h, int(job)))

    def film(self, job: int):
        """(sum RGB, sum of squares RGB, sample count) per pixel, as ``GPURenderer.getFilm``."""
        w, h = self._jobs[job]
        out = np.empty((h, w, 7), dtype=np.float32)
        self._check(self._lib.dfc_job_read_film(self._h, int(job), out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out[..., 0:3], out[..., 3:6], out[..., 6]

    def radiance(self, job: int) -> np.ndarray:
        s, _, n = self.film(job)
        return s / np.maximum(n, 1.0)[..., None]

    def image(self, job: int, tone_mapper: int = 1) -> np.ndarray:
        w, h = self._jobs[job]
        out = np.empty((h, w, 4), dtype=np.uint8)
        self._check(self._lib.dfc_job_read_image_rgba8(self._h, int(job), int(tone_mapper), out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def release(self, job: int):
        self._check(self._lib.dfc_job_release(self._h, int(job)))
        self._jobs.pop(job, None)

    # -- driving -------------------------------------------------------------------
    def run(self, timeout_s: float = 0.0):
        """Renders until every submitted job is finished (batched mode)."""
        self._check(self._lib.dfc_engine_run(self._h, float(timeout_s)))

    def start(self):
        """Runs the wavefront on an engine thread (served mode)."""
        self._check(self._lib.dfc_engine_start(self._h))

    def stop(self):
        self._check(self._lib.dfc_engine_stop(self._h))

    def stats(self) -> dict:
        s = EngineStats()
        self._check(self._lib.dfc_engine_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()
