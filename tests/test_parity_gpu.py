"""Device renderer against the CPU oracle on the same compiled scenes."""
import numpy as np
import pytest

from dayflower_b200 import RenderingAlgorithm as RA
from dayflower_b200.scene import generators as G
from dayflower_b200.scene.compiler import compile_scene

from . import parity as PT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cornell():
    return compile_scene(G.cornell_box(resolution=(128, 128)))


@pytest.fixture(scope="module")
def mixed():
    return compile_scene(G.small_mixed_scene(resolution=(96, 64)), layout_version=2)


@pytest.fixture(scope="module")
def quadrics():
    return compile_scene(G.quadrics_scene(resolution=(128, 96)))


@pytest.fixture(scope="module")
def disney():
    return compile_scene(G.disney_scene(resolution=(128, 72)))


@pytest.fixture(scope="module")
def materials():
    return compile_scene(G.materials_scene(resolution=(128, 72)), layout_version=2)


@pytest.fixture(scope="module")
def image_light():
    return compile_scene(G.image_light_scene(resolution=(128, 72)), layout_version=2)


@pytest.fixture(scope="module")
def instances():
    # the large scene's construction at test size: instanced blob meshes, Disney, image light
    return compile_scene(G.large_scene(cells=48, instances=120, resolution=(128, 72), env=(128, 64), extent=40.0), layout_version=2)


@pytest.fixture(scope="module")
def terrain():
    return compile_scene(G.terrain_spheres(cells=128, n_spheres=300, resolution=(160, 90), seed=11), layout_version=2)


@pytest.mark.parametrize("scene_name", ["cornell", "mixed", "terrain", "quadrics", "disney", "materials", "image_light", "instances"])
def test_ray_casting_hit_ids(scene_name, request):
    cs = request.getfixturevalue(scene_name)
    g = PT.render_gpu(cs, RA.RAY_CASTING)
    o = PT.render_oracle(cs, RA.RAY_CASTING)
    o_nd = PT.render_oracle_no_drift(cs, RA.RAY_CASTING)
    PT.check_primary(g, o, o_nd)
    # shading 0.5 |n_s . d| (Scene.java:675): absolute agreement with the drift-free oracle
    mg = g["sum"] / np.maximum(g["count"], 1)[..., None]
    mo = o_nd["sum"] / np.maximum(o_nd["count"], 1)[..., None]
    assert np.mean(np.all(np.abs(mg - mo) <= 1e-4, axis=-1)) >= 0.999


@pytest.mark.parametrize("scene_name", ["cornell", "mixed", "quadrics"])
def test_depth_camera(scene_name, request):
    cs = request.getfixturevalue(scene_name)
    g = PT.render_gpu(cs, RA.DEPTH_CAMERA)
    o = PT.render_oracle(cs, RA.DEPTH_CAMERA)
    PT.check_primary(g, o, PT.render_oracle_no_drift(cs, RA.DEPTH_CAMERA))
    mg = g["sum"] / np.maximum(g["count"], 1)[..., None]
    mo = o["sum"] / np.maximum(o["count"], 1)[..., None]
    assert np.mean(np.all(np.abs(mg - mo) <= 1e-4 + 1e-4 * np.abs(mo), axis=-1)) >= 0.999


@pytest.mark.parametrize("scene_name,spp", [("cornell", 16), ("mixed", 16), ("terrain", 8), ("quadrics", 16), ("disney", 16), ("materials", 16), ("image_light", 16), ("instances", 8)])
def test_path_tracing_sigma(scene_name, spp, request):
    cs = request.getfixturevalue(scene_name)
    g = PT.render_gpu(cs, RA.PATH_TRACING, spp=spp, max_bounce=8)
    o = PT.render_oracle(cs, RA.PATH_TRACING, spp=spp, max_bounce=8)
    ok, mg, mo = PT.sigma_test(g, o)
    assert ok >= PT.PIXEL_PASS, "3-sigma pass rate %.4f" % ok
    # same random numbers per sample: the bulk of the image must match closely
    assert abs(mg.mean() - mo.mean()) <= 0.02 * max(mo.mean(), 1e-3) + 1e-4


@pytest.mark.parametrize("scene_name", ["cornell", "mixed"])
def test_ambient_occlusion_sigma(scene_name, request):
    cs = request.getfixturevalue(scene_name)
    g = PT.render_gpu(cs, RA.AMBIENT_OCCLUSION, spp=4, ao_samples=16, ao_distance=200.0)
    o = PT.render_oracle(cs, RA.AMBIENT_OCCLUSION, spp=4, ao_samples=16, ao_distance=200.0)
    ok, _, _ = PT.sigma_test(g, o)
    assert ok >= PT.PIXEL_PASS, "3-sigma pass rate %.4f" % ok


@pytest.mark.parametrize("scene_name", ["cornell", "mixed", "materials"])
def test_ray_tracing_sigma(scene_name, request):
    # Whitted ray tracer (Scene.java:786): every light per hit, specular reflection and transmission recursively
    cs = request.getfixturevalue(scene_name)
    g = PT.render_gpu(cs, RA.RAY_TRACING, spp=8, max_bounce=8)
    o = PT.render_oracle(cs, RA.RAY_TRACING, spp=8, max_bounce=8)
    PT.check_primary(g, o, PT.render_oracle_no_drift(cs, RA.RAY_TRACING))
    ok, mg, mo = PT.sigma_test(g, o)
    assert ok >= PT.PIXEL_PASS, "3-sigma pass rate %.4f" % ok
    assert abs(mg.mean() - mo.mean()) <= 0.02 * max(mo.mean(), 1e-3) + 1e-4


@pytest.mark.parametrize("scene_name", ["cornell", "disney"])
def test_path_tracing_rmse_against_converged(scene_name, request):
    # PATH_TRACING criterion: at equal spp (16), the RMSE against a converged
    # 16,384-spp image is within 2% of the CPU oracle's RMSE.  The converged
    # image is rendered on the device with an independent seed.
    cs = request.getfixturevalue(scene_name)
    conv = PT.render_gpu(cs, RA.PATH_TRACING, spp=16384, max_bounce=8, seed=0xC0FFEE)
    ref = conv["sum"] / np.maximum(conv["count"], 1)[..., None]
    g = PT.render_gpu(cs, RA.PATH_TRACING, spp=16, max_bounce=8)
    o = PT.render_oracle(cs, RA.PATH_TRACING, spp=16, max_bounce=8)
    rmse_g = float(np.sqrt(np.mean((g["sum"] / np.maximum(g["count"], 1)[..., None] - ref) ** 2)))
    rmse_o = float(np.sqrt(np.mean((o["sum"] / np.maximum(o["count"], 1)[..., None] - ref) ** 2)))
    assert abs(rmse_g - rmse_o) <= 0.02 * rmse_o, "RMSE device %.5f oracle %.5f" % (rmse_g, rmse_o)
