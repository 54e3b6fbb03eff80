"""dfc_trace_rays_noalloc against the existing render entry point.

The primary rays of a RAY_CASTING pass are restated on the host by the oracle
(same counter-based jitter, same camera), traced through the no-allocation
entry point twice in a row, and compared with the primary hits that
dfc_render + dfc_read_primary_hits report for the same pass.  The file sorts
last so that it runs both alone and after every other GPU test.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from dayflower_b200 import GPURenderer, RenderingAlgorithm
from dayflower_b200.scene import generators as G
from dayflower_b200.scene.compiler import compile_scene

SEED = 0x5EED1234
T_MIN = 1e-4
FLT_MAX = np.finfo(np.float32).max
MAX_RAYS = 1 << 20
ID_AGREEMENT = 0.999
T_RTOL = 1e-5

pytestmark = pytest.mark.gpu


def _primary_rays(oracle, compiled):
    """Origins (x, y, z, tmin) and directions (dx, dy, dz, tmax) of pass 0, one per pixel."""
    L = oracle.lib()
    sc = oracle.OracleScene(compiled)
    w, h = sc.width, sc.height
    org = np.zeros((h * w, 4), np.float32)
    dirs = np.zeros((h * w, 4), np.float32)
    out6 = np.zeros(6, np.float32)
    for y in range(h):
        for x in range(w):
            pix = y * w + x
            key = L.dfo_rng_path_key(SEED, pix, 0)
            px, py = L.dfo_rng_uniform(key, 0), L.dfo_rng_uniform(key, 1)
            assert L.dfo_primary_ray(sc._s, float(x), float(y), px, py, out6.ctypes.data_as(ctypes.c_void_p))
            org[pix] = (out6[0], out6[1], out6[2], T_MIN)
            dirs[pix] = (out6[3], out6[4], out6[5], FLT_MAX)
    return org, dirs


def _existing_entry(compiled):
    r = GPURenderer()
    try:
        r.setScene(compiled)
        r.setRenderingAlgorithm(RenderingAlgorithm.RAY_CASTING)
        r.setSeed(SEED)
        r.setup()
        assert r.render(1)
        return r.getPrimaryHits()
    finally:
        r.dispose()


@pytest.mark.parametrize("name", ["cornell", "mixed"])
def test_noalloc_matches_render_entry(oracle, name):
    import torch

    if name == "cornell":
        compiled = compile_scene(G.cornell_box(resolution=(128, 128)))
    else:
        compiled = compile_scene(G.small_mixed_scene(resolution=(96, 64)), layout_version=2)
    prim_ref, t_ref = _existing_entry(compiled)
    org, dirs = _primary_rays(oracle, compiled)
    n = org.shape[0]

    dev = torch.device("cuda:0")
    d_org = torch.from_numpy(org).to(dev)
    d_dir = torch.from_numpy(dirs).to(dev)
    d_hits = torch.full((n, 4), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    r = GPURenderer()
    try:
        r.setScene(compiled)
        r.traceRaysNoAlloc(0, 0, 0, 0)  # first-call set-up only
        calls = []
        for _ in range(2):
            d_hits.fill_(float("nan"))
            torch.cuda.synchronize()
            r.traceRaysNoAlloc(d_org.data_ptr(), d_dir.data_ptr(), d_hits.data_ptr(), n)
            calls.append(d_hits.cpu().numpy().copy())
    finally:
        r.dispose()

    # the two calls in a row agree bit for bit (the scratch is re-armed per call)
    assert np.array_equal(calls[0].view(np.uint32), calls[1].view(np.uint32))
    hits = calls[1]
    prim = hits[:, 1].copy().view(np.int32).reshape(prim_ref.shape)
    t = hits[:, 0].reshape(t_ref.shape)
    agree = prim == prim_ref
    assert agree.mean() >= ID_AGREEMENT, (name, agree.mean())
    both = agree & (prim_ref >= 0)
    assert both.sum() > 0.5 * both.size
    rel = np.abs(t[both] - t_ref[both]) / np.maximum(np.abs(t_ref[both]), 1e-30)
    assert rel.max() <= T_RTOL, (name, rel.max())


def test_noalloc_rejects_oversized_and_host_buffers():
    compiled = compile_scene(G.cornell_box(resolution=(16, 16)))
    r = GPURenderer()
    try:
        with pytest.raises(ValueError, match="limit"):
            r.traceRaysNoAlloc(16, 16, 16, MAX_RAYS + 1)
        host = np.zeros((4, 4), np.float32)
        with pytest.raises(Exception):
            r.traceRaysNoAlloc(0, 0, 0, 4)  # before setScene
        r.setScene(compiled)
        with pytest.raises(ValueError, match="aligned|device memory"):
            p = host.ctypes.data
            r.traceRaysNoAlloc(p, p, p, 4)
        # an edit made after setScene is not traced silently: the caller must commit it first
        from dayflower_b200.renderer import DFC_E_STATE, RenderError
        from dayflower_b200.scene import model as M
        from dayflower_b200.scene.compiler import CompiledSceneModifier
        assert CompiledSceneModifier(compiled).add_primitive(
            M.Primitive(M.Sphere(), M.Matte(kd=(0.5, 0.5, 0.5)), M.Transform.translate_scale((0.0, 10.0, 0.0), 2.0)))
        with pytest.raises(RenderError) as e:
            r.traceRaysNoAlloc(0, 0, 0, 0)
        assert e.value.code == DFC_E_STATE
        r.setScene(compiled)
        r.traceRaysNoAlloc(0, 0, 0, 0)
    finally:
        r.dispose()
