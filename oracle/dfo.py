"""ctypes binding of the CPU oracle (``oracle/dfo.cpp``).

TEST INFRASTRUCTURE ONLY.  The oracle restates Dayflower's CPURenderer
(``renderer/cpu/CPURenderer.java`` and ``scene/Scene.java``) over the compiled
scene arrays.  Only ``tests/``, ``__graft_entry__.smoke()`` and the benchmark's
CPU-baseline leg use it, as the checker; the renderer never calls it.

Pinning: the oracle's primitive math is checked against the golden vectors of
the reference's own unit tests (tests/test_oracle_golden.py).  No reference
test pins a rendered image, and the Java renderer cannot run here (no JVM), so
end-to-end image parity with the Java CPURenderer itself is unpinned.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libdfo.so")

_c_p, _c_f, _c_i, _c_u = ctypes.c_void_p, ctypes.c_float, ctypes.c_int, ctypes.c_uint


class Params(ctypes.Structure):
    _fields_ = [("algo", _c_i), ("width", _c_i), ("height", _c_i), ("spp", _c_i), ("sample_base", _c_i),
                ("max_bounce", _c_i), ("min_rr", _c_i), ("ao_samples", _c_i), ("ao_distance", _c_f), ("preview", _c_i),
                ("seed", _c_u), ("row_begin", _c_i), ("row_end", _c_i), ("row_step", _c_i)]


_lib = None


def build() -> str:
    src = [os.path.join(HERE, f) for f in ("dfo.cpp", "dfo_math.h", "Makefile")]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in src):
        r = subprocess.run(["make", "-C", HERE], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stdout)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        L = ctypes.CDLL(build())
        L.dfo_scene_new.restype = _c_p
        L.dfo_scene_free.argtypes = [_c_p]
        L.dfo_scene_put.argtypes = [_c_p, ctypes.c_char_p, _c_p, ctypes.c_longlong, _c_i]
        L.dfo_scene_commit.argtypes = [_c_p, _c_i]
        L.dfo_render.restype = ctypes.c_longlong
        L.dfo_render.argtypes = [_c_p, ctypes.POINTER(Params), _c_p, _c_p, _c_p, _c_p, _c_p, _c_i]
        L.dfo_render_pixel_film.restype = ctypes.c_longlong
        L.dfo_render_pixel_film.argtypes = [_c_p, ctypes.POINTER(Params), _c_p, _c_i]
        for n in ("dfo_plane_intersection", "dfo_sphere_intersection"):
            getattr(L, n).argtypes = [_c_p, _c_p, _c_f, _c_f, _c_p]
        L.dfo_sphere_intersection_t.restype = _c_f
        L.dfo_sphere_intersection_t.argtypes = [_c_p, _c_p, _c_f, _c_f]
        L.dfo_triangle_intersection_t.restype = _c_f
        L.dfo_triangle_intersection_t.argtypes = [_c_p, _c_p, _c_p, _c_f, _c_f]
        L.dfo_aabb_intersection.argtypes = [_c_p, _c_p, _c_p, _c_f, _c_f, _c_p]
        L.dfo_ray_transform.argtypes = [_c_p, _c_p, _c_p, _c_p]
        L.dfo_onb_from_w.argtypes = [_c_p, _c_p]
        L.dfo_onb_from_wv.argtypes = [_c_p, _c_p, _c_p]
        L.dfo_rgb_to_xyz.argtypes = [_c_p, _c_p]
        L.dfo_xyz_to_rgb.argtypes = [_c_p, _c_p]
        for n in ("dfo_srgb_redo", "dfo_srgb_undo"):
            getattr(L, n).restype = _c_f
            getattr(L, n).argtypes = [_c_f]
        L.dfo_gaussian_filter.restype = _c_f
        L.dfo_gaussian_filter.argtypes = [_c_f] * 5
        L.dfo_triangle_filter.restype = _c_f
        L.dfo_triangle_filter.argtypes = [_c_f] * 4
        L.dfo_rng_path_key.restype = _c_u
        L.dfo_rng_path_key.argtypes = [_c_u, _c_u, _c_u]
        L.dfo_rng_uniform.restype = _c_f
        L.dfo_rng_uniform.argtypes = [_c_u, _c_u]
        L.dfo_primary_ray.argtypes = [_c_p, _c_f, _c_f, _c_f, _c_f, _c_p]
        L.dfo_primary_prim_t.argtypes = [_c_p, _c_u, _c_i, _c_i, _c_i, _c_f, _c_f, _c_i, ctypes.POINTER(_c_f)]
        for n, args in (("dfo_perlin", [_c_f] * 3), ("dfo_simplex", [_c_f] * 3), ("dfo_perlin_turbulence", [_c_f] * 3 + [_c_i]),
                        ("dfo_simplex_fbm", [_c_f] * 7 + [_c_i])):
            getattr(L, n).restype = _c_f
            getattr(L, n).argtypes = args
        L.dfo_colorspace.argtypes = [_c_p, _c_i, _c_p, _c_p]
        L.dfo_onb_transform.argtypes = [_c_p, _c_p, _c_p]
        L.dfo_set_no_drift.argtypes = [_c_i]
        _lib = L
    return _lib


def f32(*v) -> np.ndarray:
    return np.asarray(v, dtype=np.float32).reshape(-1)


def ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleScene:
    """A compiled scene loaded into the oracle."""

    def __init__(self, compiled):
        L = lib()
        self._s = L.dfo_scene_new()
        for name, arr in compiled.arrays.items():
            a = np.ascontiguousarray(arr)
            L.dfo_scene_put(self._s, name.encode(), ptr(a), a.size, 1 if a.dtype == np.int32 else 0)
        rc = L.dfo_scene_commit(self._s, compiled.layout_version)
        if rc != 0:
            raise ValueError("oracle scene commit failed (%d)" % rc)
        cam = compiled.arrays["cameraArray"]
        self.width, self.height = int(cam[17]), int(cam[18])

    def __del__(self):
        try:
            lib().dfo_scene_free(self._s)
        except Exception:
            pass

    def render(self, algorithm: int, spp: int = 1, sample_base: int = 0, max_bounce: int = 20, min_rr: int = 5,
               ao_samples: int = 10, ao_distance: float = 20.0, seed: int = 0x5EED1234, rows=None, threads: int = 1,
               preview: bool = False, row_step: int = 1):
        """Returns dict(sum, sumsq, count, prim, t, rays) over rows r0, r0 + row_step, ... below r1
        (rows = (r0, r1), default the whole image); rows not rendered are left empty."""
        W, H = self.width, self.height
        r0, r1 = (0, H) if rows is None else rows
        p = Params(int(algorithm), W, H, int(spp), int(sample_base), int(max_bounce), int(min_rr), int(ao_samples),
                   float(ao_distance), 1 if preview else 0, int(seed) & 0xFFFFFFFF, int(r0), int(r1), int(row_step))
        s = np.zeros((H, W, 3), np.float32)
        q = np.zeros((H, W, 3), np.float32)
        n = np.zeros((H, W), np.int32)
        prim = np.full((H, W), -1, np.int32)
        t = np.full((H, W), np.nan, np.float32)
        rays = lib().dfo_render(self._s, ctypes.byref(p), ptr(s), ptr(q), ptr(n), ptr(prim), ptr(t), int(threads))
        if rays < 0:
            raise RuntimeError("oracle render failed (%d): the scene uses features the oracle does not restate" % rays)
        return {"sum": s, "sumsq": q, "count": n, "prim": prim, "t": t, "rays": int(rays)}

    def primary_prim_t(self, seed: int, x: int, y: int, prim: int, dpx: float = 0.0, dpy: float = 0.0):
        """World t at which pixel (x, y)'s first primary ray (its jitter moved by
        (dpx, dpy) pixels) hits primitive ``prim`` alone, or None on a miss."""
        t = _c_f(0.0)
        rc = lib().dfo_primary_prim_t(self._s, int(seed) & 0xFFFFFFFF, self.width, int(x), int(y), float(dpx), float(dpy), int(prim),
                                      ctypes.byref(t))
        if rc < 0:
            raise ValueError("bad primitive or pixel")
        return float(t.value) if rc == 1 else None

    def render_pixel_film(self, algorithm: int, spp: int = 1, sample_base: int = 0, max_bounce: int = 20, min_rr: int = 5,
                          ao_samples: int = 10, ao_distance: float = 20.0, seed: int = 0x5EED1234, threads: int = 1):
        """The CPU renderer's Gaussian XYZ film (PixelImageF): per pixel X, Y, Z sums and the filter weight sum, (H, W, 4)."""
        W, H = self.width, self.height
        p = Params(int(algorithm), W, H, int(spp), int(sample_base), int(max_bounce), int(min_rr), int(ao_samples),
                   float(ao_distance), 0, int(seed) & 0xFFFFFFFF, 0, H, 1)
        out = np.zeros((H, W, 4), np.float32)
        rays = lib().dfo_render_pixel_film(self._s, ctypes.byref(p), ptr(out), int(threads))
        if rays < 0:
            raise RuntimeError("oracle render failed (%d)" % rays)
        return out
