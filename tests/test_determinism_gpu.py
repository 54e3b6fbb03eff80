"""Per-job renders are bitwise reproducible.

A render pass of the per-job renderer has one path per pixel and runs its
kernels in order on one stream, so each pixel of the box film has one writer
per pass and its sums are formed in pass order.  Two renders with the same
seed must therefore give the same film bit for bit, for every rendering
algorithm, and a different seed must give a different one.
"""
from __future__ import annotations

import numpy as np
import pytest

from dayflower_b200 import RenderingAlgorithm as RA
from dayflower_b200.scene import generators as G
from dayflower_b200.scene.compiler import compile_scene

from . import parity as PT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes():
    return {
        "cornell": compile_scene(G.cornell_box(resolution=(96, 96))),
        "terrain": compile_scene(G.terrain_spheres(cells=64, n_spheres=200, resolution=(128, 72), seed=3), layout_version=2),
    }


@pytest.mark.parametrize("name", ["cornell", "terrain"])
@pytest.mark.parametrize("algo,spp", [(RA.PATH_TRACING, 6), (RA.AMBIENT_OCCLUSION, 3), (RA.RAY_TRACING, 2), (RA.RAY_CASTING, 2)])
def test_same_seed_same_film(scenes, name, algo, spp):
    cs = scenes[name]
    a = PT.render_gpu(cs, algo, spp=spp, max_bounce=6, seed=77)
    b = PT.render_gpu(cs, algo, spp=spp, max_bounce=6, seed=77)
    for k in ("sum", "sumsq", "count"):
        assert np.array_equal(a[k].view(np.uint32), b[k].view(np.uint32)), k
    assert a["counters"]["rays"] == b["counters"]["rays"]
    if algo == RA.PATH_TRACING:
        c = PT.render_gpu(cs, algo, spp=spp, max_bounce=6, seed=78)
        assert not np.array_equal(a["sum"], c["sum"])
