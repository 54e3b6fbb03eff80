"""Ray queries at the edges of the traversal's input range.

Rays given an infinite tmax must hit exactly what the same rays with
tmax = FLT_MAX hit, including rays whose direction has zero components (slab
planes parallel to the ray, inverse direction components clamped to
+-2^80) and rays that start outside the scene.
"""
from __future__ import annotations

import numpy as np
import pytest

from dayflower_b200 import GPURenderer
from dayflower_b200.scene import generators as G
from dayflower_b200.scene.compiler import compile_scene

pytestmark = pytest.mark.gpu

FLT_MAX = np.finfo(np.float32).max
T_MIN = 1e-4


def _rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    org = np.zeros((n, 4), np.float32)
    d = np.zeros((n, 4), np.float32)
    org[:, :3] = rng.uniform(lo, hi, size=(n, 3))
    org[:, 3] = T_MIN
    v = rng.normal(size=(n, 3))
    k = n // 4  # a quarter along the coordinate axes (zero direction components)
    axes = rng.integers(0, 3, size=k)
    v[:k] = 0.0
    v[np.arange(k), axes] = rng.choice([-1.0, 1.0], size=k)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    d[:, :3] = v
    return org, d


def _trace(r, org, dirs):
    import torch

    dev = torch.device("cuda:0")
    d_org = torch.from_numpy(org).to(dev)
    d_dir = torch.from_numpy(dirs).to(dev)
    d_hits = torch.full((org.shape[0], 4), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    r.traceRaysNoAlloc(d_org.data_ptr(), d_dir.data_ptr(), d_hits.data_ptr(), org.shape[0])
    return d_hits.cpu().numpy()


@pytest.mark.parametrize("name", ["cornell", "terrain"])
def test_infinite_tmax_hits_what_flt_max_hits(name):
    if name == "cornell":
        cs = compile_scene(G.cornell_box(resolution=(16, 16)))
        lo, hi = -20.0, 120.0
    else:
        cs = compile_scene(G.terrain_spheres(cells=64, n_spheres=200, resolution=(16, 16), seed=3), layout_version=2)
        lo, hi = -70.0, 70.0
    org, dirs = _rays(65536, lo, hi, seed=11)
    r = GPURenderer()
    try:
        r.setScene(cs)
        dirs[:, 3] = FLT_MAX
        a = _trace(r, org, dirs)
        dirs[:, 3] = np.inf
        b = _trace(r, org, dirs)
    finally:
        r.dispose()
    pa = a[:, 1].copy().view(np.int32)
    pb = b[:, 1].copy().view(np.int32)
    assert np.array_equal(pa, pb)
    hit = pa >= 0
    assert hit.mean() > 0.01, hit.mean()
    assert np.array_equal(a[hit, 0].view(np.uint32), b[hit, 0].view(np.uint32))
