"""``GPURenderer``: the Python face of libdayflower_cuda, mirroring the Java API of
``org.dayflower.renderer.gpu.GPURenderer`` (renderer/gpu/GPURenderer.java and
AbstractGPURenderer.java) method by method.

Exceptions follow the reference: ``ValueError`` where Java throws
``IllegalArgumentException``, ``TypeError`` for ``NullPointerException``,
:class:`UnsupportedSceneError` for scene content the renderer does not
implement, :class:`RenderError` for CUDA failures.
"""
from __future__ import annotations

import ctypes
import enum
from typing import Optional

import numpy as np

from . import _native
from .scene.compiler import CompiledScene, compile_scene
from .scene.model import Scene

DFC_OK, DFC_E_INVALID_ARG, DFC_E_UNSUPPORTED, DFC_E_OOM, DFC_E_CUDA, DFC_E_TIMEOUT, DFC_E_STOPPED, DFC_E_STATE = range(8)


class RenderingAlgorithm(enum.IntEnum):
    """``renderer/RenderingAlgorithm.java:33-53`` (ordinal order)."""
    AMBIENT_OCCLUSION = 0
    DEPTH_CAMERA = 1
    PATH_TRACING = 2
    RAY_CASTING = 3
    RAY_TRACING = 4


class RenderError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("%s (status %d)" % (message, code))
        self.code = code


class UnsupportedSceneError(RenderError):
    pass


class GPURenderer:
    """Drop-in for ``GPURenderer`` over the compiled-scene arrays."""

    TONE_MAPPER_FILMIC_CURVE_ACES_MODIFIED_VERSION_1 = 0
    TONE_MAPPER_NONE = 1
    TONE_MAPPER_REINHARD = 2
    TONE_MAPPER_REINHARD_MODIFIED_VERSION_1 = 3
    TONE_MAPPER_REINHARD_MODIFIED_VERSION_2 = 4
    TONE_MAPPER_UNREAL_3 = 5

    def __init__(self, device: int = 0, renderer_observer=None):
        self._lib = _native.load_renderer()
        h = ctypes.c_void_p()
        rc = self._lib.dfc_create(int(device), ctypes.byref(h))
        if rc != DFC_OK:
            raise RenderError(rc, "dfc_create failed (no usable CUDA device %d)" % device)
        self._h = h
        self._observer = renderer_observer
        self._width, self._height = 800, 800
        self._scene: Optional[CompiledScene] = None
        self._render_pass = 0

    # -- helpers ---------------------------------------------------------------
    def _check(self, rc: int):
        if rc == DFC_OK:
            return
        msg = (self._lib.dfc_last_error(self._h) or b"").decode()
        if rc == DFC_E_INVALID_ARG:
            raise ValueError(msg)
        if rc == DFC_E_UNSUPPORTED:
            raise UnsupportedSceneError(rc, msg)
        raise RenderError(rc, msg)

    def _alive(self):
        if self._h is None:
            raise RenderError(DFC_E_STATE, "renderer disposed")

    # -- scene -----------------------------------------------------------------
    def setScene(self, scene, layout_version: Optional[int] = None):
        """``AbstractSceneKernel.setScene`` + ``doSetupScene``: accepts a model
        :class:`Scene` (compiled here) or an already compiled scene."""
        self._alive()
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
            self._check(self._lib.dfc_scene_put(self._h, name.encode(), a.ctypes.data_as(ctypes.c_void_p), a.size, typ))
        self._check(self._lib.dfc_scene_commit(self._h, int(layout_version or cs.layout_version)))
        self._scene = cs
        self._scene_version = getattr(cs, "version", 0)
        cam = cs.arrays["cameraArray"]
        self._width, self._height = int(cam[17]), int(cam[18])
        self._check(self._lib.dfc_set_image(self._h, self._width, self._height))

    def setImage(self, width: Optional[int] = None, height: Optional[int] = None):
        """``setImage()`` (resolution from the camera) / ``setImage(ImageF)``."""
        self._alive()
        if width is None or height is None:
            self._check(self._lib.dfc_set_image(self._h, 0, 0))
            if self._scene is not None:
                cam = self._scene.arrays["cameraArray"]
                self._width, self._height = int(cam[17]), int(cam[18])
        else:
            self._check(self._lib.dfc_set_image(self._h, int(width), int(height)))
            self._width, self._height = int(width), int(height)

    # -- settings (AbstractGPURenderer.java:448-526) -----------------------------
    def setMaximumBounce(self, v: int): self._check(self._lib.dfc_set_maximum_bounce(self._h, int(v)))
    def setMinimumBounceRussianRoulette(self, v: int): self._check(self._lib.dfc_set_minimum_bounce_russian_roulette(self._h, int(v)))
    def setSamples(self, v: int): self._check(self._lib.dfc_set_samples(self._h, int(v)))
    def setMaximumDistance(self, v: float): self._check(self._lib.dfc_set_maximum_distance(self._h, float(v)))
    def setToneMapper(self, v: int): self._check(self._lib.dfc_set_tone_mapper(self._h, int(v)))
    def setPreviewMode(self, v: bool): self._check(self._lib.dfc_set_preview_mode(self._h, 1 if v else 0))
    def setSeed(self, seed: int): self._check(self._lib.dfc_set_seed(self._h, int(seed) & 0xFFFFFFFF))

    FILM_BOX, FILM_GAUSSIAN = 0, 1

    def setFilmFilter(self, film: int):
        """0: per-pixel box film (getFilm); 1: the CPU renderer's Gaussian XYZ film
        (PixelImageF, getPixelFilm).  Takes effect at the next setup()."""
        self._check(self._lib.dfc_set_film_filter(self._h, int(film)))
    def setStageTiming(self, on: bool): self._check(self._lib.dfc_set_stage_timing(self._h, 1 if on else 0))

    def setRenderingAlgorithm(self, algorithm):
        if algorithm is None:
            raise TypeError("renderingAlgorithm == null")
        self._check(self._lib.dfc_set_rendering_algorithm(self._h, int(algorithm)))

    # -- lifecycle -----------------------------------------------------------------
    def setup(self):
        """``AbstractGPURenderer.setup()``."""
        self._alive()
        self._check(self._lib.dfc_setup(self._h))
        self._render_pass = 0

    def render(self, render_passes: Optional[int] = None) -> bool:
        """``render()`` / ``render(int)``: True if every pass completed."""
        self._alive()
        n = 1 if render_passes is None else int(render_passes)
        cs = self._scene
        if cs is not None and getattr(cs, "version", 0) != getattr(self, "_scene_version", 0):
            # AbstractGPURenderer.render: a compiled scene changed by a CompiledSceneModifier is uploaded again and the film cleared
            self.setScene(cs)
            self.setup()
        done = ctypes.c_int(0)
        if self._observer is None:
            rc = self._lib.dfc_render(self._h, n, ctypes.byref(done))
        else:
            # every pass notifies the observer as AbstractGPURenderer.render() does (:277-291)
            errors = []

            def on_event(_user, ev_p):
                ev = ev_p.contents
                try:
                    if ev.event == 0:
                        self._notify("onRenderPassProgress", ev.render_pass, ev.progress)
                    elif ev.event == 1:
                        img = np.ctypeslib.as_array(ev.rgba, shape=(ev.height, ev.width, 4)).copy()
                        self._notify("onRenderDisplay", img)
                    else:
                        self._notify("onRenderPassComplete", ev.render_pass, ev.millis)
                except BaseException as e:  # an exception must not unwind through the C frames
                    errors.append(e)
                    self._lib.dfc_render_shutdown(self._h)

            cb = _native.OBSERVER_FN(on_event)
            rc = self._lib.dfc_render_observed(self._h, n, cb, None, ctypes.byref(done))
            if errors:
                raise errors[0]
        self._render_pass += done.value
        if rc == DFC_E_STOPPED:
            return False
        self._check(rc)
        return True

    def _notify(self, method, *args):
        fn = getattr(self._observer, method, None)
        if fn is not None:
            fn(self, *args)

    def renderShutdown(self):
        if self._h is not None:
            self._lib.dfc_render_shutdown(self._h)

    def clear(self):
        self._alive()
        self._check(self._lib.dfc_clear(self._h))
        self._render_pass = 0

    def dispose(self):
        if self._h is not None:
            self._lib.dfc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    def updateCamera(self, camera19):
        a = np.ascontiguousarray(camera19, dtype=np.float32)
        if a.size != 19:
            raise ValueError("camera needs 19 floats")
        self._check(self._lib.dfc_update_camera(self._h, a.ctypes.data_as(ctypes.c_void_p)))

    def updateMatrix44Fs(self, matrices):
        a = np.ascontiguousarray(matrices, dtype=np.float32)
        if a.size % 32:
            raise ValueError("matrices need 32 floats per primitive")
        self._check(self._lib.dfc_update_matrices(self._h, a.ctypes.data_as(ctypes.c_void_p), a.size // 32))

    # -- outputs ---------------------------------------------------------------------
    @property
    def resolution(self):
        return self._width, self._height

    def getRenderPass(self) -> int:
        return self._render_pass

    def getImage(self) -> np.ndarray:
        """RGBA8 image (tone mapped, sRGB), shape (H, W, 4)."""
        out = np.empty((self._height, self._width, 4), dtype=np.uint8)
        self._check(self._lib.dfc_read_image_rgba8(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def getFilm(self):
        """(sum RGB, sum of squares RGB, sample count) per pixel, shapes (H, W, 3), (H, W, 3), (H, W)."""
        out = np.empty((self._height, self._width, 7), dtype=np.float32)
        self._check(self._lib.dfc_read_film(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out[..., 0:3], out[..., 3:6], out[..., 6]

    def getPixelFilm(self) -> np.ndarray:
        """The Gaussian XYZ film: per pixel X, Y, Z sums and the filter weight sum, (H, W, 4)."""
        out = np.empty((self._height, self._width, 4), dtype=np.float32)
        self._check(self._lib.dfc_read_pixel_film(self._h, out.ctypes.data_as(ctypes.c_void_p), out.size))
        return out

    def getRadiance(self) -> np.ndarray:
        s, _, n = self.getFilm()
        return s / np.maximum(n, 1.0)[..., None]

    def getPrimaryHits(self):
        prim = np.empty((self._height, self._width), dtype=np.int32)
        t = np.empty((self._height, self._width), dtype=np.float32)
        self._check(self._lib.dfc_read_primary_hits(self._h, prim.ctypes.data_as(ctypes.c_void_p), t.ctypes.data_as(ctypes.c_void_p), prim.size))
        return prim, t

    def getCounters(self):
        out = np.zeros(4, dtype=np.int64)
        self._check(self._lib.dfc_read_counters(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return {"passes": int(out[0]), "paths": int(out[1]), "rays": int(out[2]), "launches": int(out[3])}

    def traceRaysNoAlloc(self, d_origins: int, d_directions: int, d_hits: int, count: int):
        """Closest hits of ``count`` rays held in device memory (addresses of
        float4 arrays: origins, directions with tmax in w, hits out), with no
        device allocation by the library; at most 1,048,576 rays per call.

        It traces the scene of the last ``setScene``.  Edits made since then
        with a ``CompiledSceneModifier`` raise :class:`RenderError`
        (``DFC_E_STATE``): uploading them would allocate device memory, so the
        caller commits them first with ``setScene``."""
        self._alive()
        cs = self._scene
        if cs is not None and getattr(cs, "version", 0) != getattr(self, "_scene_version", 0):
            raise RenderError(DFC_E_STATE, "the compiled scene changed after setScene(); commit it with setScene() before "
                                           "traceRaysNoAlloc (which uploads nothing)")
        self._check(self._lib.dfc_trace_rays_noalloc(self._h, ctypes.c_void_p(d_origins), ctypes.c_void_p(d_directions),
                                                     ctypes.c_void_p(d_hits), int(count)))

    KERNELS = ("call", "raygen", "trace", "shade", "film", "sort_count", "sort_scatter", "ray_list")

    def kernelStats(self):
        """Per kernel kind: device milliseconds and launches of the last render call (with stage timing
        on) and the items processed since setup/clear (paths, rays, shade work items, listed rays)."""
        n = len(self.KERNELS)
        ms = np.zeros(n, dtype=np.float32)
        launches = np.zeros(n, dtype=np.int64)
        items = np.zeros(n, dtype=np.int64)
        self._check(self._lib.dfc_read_kernel_stats(self._h, ms.ctypes.data_as(ctypes.c_void_p), launches.ctypes.data_as(ctypes.c_void_p),
                                                    items.ctypes.data_as(ctypes.c_void_p), n))
        return {k: {"ms": float(ms[i]), "launches": int(launches[i]), "items": int(items[i])} for i, k in enumerate(self.KERNELS)}

    def lastRenderMillis(self) -> float:
        return self.stageMillis()["total"]

    def stageMillis(self):
        """Device milliseconds of the last render call: total and, with stage timing on, per stage."""
        out = np.zeros(5, dtype=np.float32)
        self._check(self._lib.dfc_read_stage_times(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return {"total": float(out[0]), "raygen": float(out[1]), "trace": float(out[2]), "shade": float(out[3]), "film": float(out[4])}

    BVH_HOST, BVH_DEVICE = 0, 1

    def setBVHBuilder(self, builder: int):
        """Builder of the mesh hierarchies of later ``setScene`` calls: ``BVH_HOST`` (binned SAH on
        the host) or ``BVH_DEVICE`` (built on the GPU from the uploaded triangles)."""
        self._alive()
        self._check(self._lib.dfc_set_bvh_builder(self._h, int(builder)))

    def commitMillis(self):
        """Host milliseconds of the last setScene commit: ingest (decode and builds), its bottom- and
        top-level builds, and the upload."""
        out = np.zeros(4, dtype=np.float32)
        self._check(self._lib.dfc_read_commit_times(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return {"ingest": float(out[0]), "blas": float(out[1]), "tlas": float(out[2]), "upload": float(out[3])}
