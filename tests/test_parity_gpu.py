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
def textures():
    return compile_scene(G.textures_scene(resolution=(128, 72)))


@pytest.fixture(scope="module")
def terrain():
    return compile_scene(G.terrain_spheres(cells=128, n_spheres=300, resolution=(160, 90), seed=11), layout_version=2)


@pytest.mark.parametrize("scene_name", ["cornell", "mixed", "terrain", "quadrics", "disney", "materials", "image_light", "instances",
                                        "textures"])
def test_ray_casting_hit_ids(scene_name, request):
    cs = request.getfixturevalue(scene_name)
    g = PT.render_gpu(cs, RA.RAY_CASTING)
    o = PT.render_oracle(cs, RA.RAY_CASTING)
    o_nd = PT.render_oracle_no_drift(cs, RA.RAY_CASTING)
    PT.check_primary(g, o, o_nd)
    from oracle import dfo
    _, _, bad = PT.mismatch_near_ties(g, dfo.OracleScene(cs), o_nd, 0x5EED1234)
    assert not bad, "hit-id mismatches that are not near ties: %s" % bad[:5]
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


@pytest.mark.parametrize("scene_name,spp", [("cornell", 16), ("mixed", 16), ("terrain", 8), ("quadrics", 16), ("disney", 16), ("materials", 16), ("image_light", 16), ("instances", 8),
                                                 ("textures", 16)])
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


@pytest.mark.parametrize("scene_name", ["cornell", "mixed", "materials", "textures"])
def test_ray_tracing_sigma(scene_name, request):
    # Whitted ray tracer (Scene.java:786): every light per hit, specular reflection and transmission recursively
    cs = request.getfixturevalue(scene_name)
    g = PT.render_gpu(cs, RA.RAY_TRACING, spp=8, max_bounce=8)
    o = PT.render_oracle(cs, RA.RAY_TRACING, spp=8, max_bounce=8)
    PT.check_primary(g, o, PT.render_oracle_no_drift(cs, RA.RAY_TRACING))
    ok, mg, mo = PT.sigma_test(g, o)
    assert ok >= PT.PIXEL_PASS, "3-sigma pass rate %.4f" % ok
    assert abs(mg.mean() - mo.mean()) <= 0.02 * max(mo.mean(), 1e-3) + 1e-4


@pytest.mark.parametrize("scene_name", ["cornell", "mixed", "quadrics"])
def test_path_tracing_rmse_against_converged(scene_name, request):
    # PATH_TRACING criterion: at equal spp (16), the RMSE against a converged
    # 16,384-spp image is within 2% of the CPU oracle's RMSE.  The converged
    # image is rendered on the device with an independent seed; the RMSE is
    # the root of the mean squared error over four 16-spp renders with
    # different seeds (an estimate of the expected error, not of one draw).
    #
    # The oracle is the faithful one.  The reference carries each ray through
    # every primitive's space in list order, which moves a secondary ray's
    # origin by a few ulps and so decides whether a ray leaving a curved
    # surface hits that surface again at t ~ 1e-6 (the near root wins when its
    # lower bound is above 0, Sphere3F.java intersectionT).  A hierarchy cannot
    # follow that order per sample (per sample the device matches the
    # drift-free oracle, as the depth check shows), but in the aggregate the
    # device's image statistics are the faithful oracle's: measured device /
    # faithful RMSE 0.998-1.000 on these scenes, against 0.987-1.000 for the
    # drift-free oracle, whose glass and mirror spheres never re-hit
    # themselves.
    #
    # The Disney and materials scenes are not cases: their 16-spp error is
    # dominated by rare caustic paths (thin, glass and translucent spheres
    # under small bright lights) that ulp-level differences send elsewhere, so
    # two CPU oracles that differ only by the drift above give single-seed RMSE
    # ratios from 0.33 to 18 (Disney; 16 seeds: 1.13) and from 0.93 to 1.003
    # (materials).  They are held to the 3-sigma and mean checks.
    cs = request.getfixturevalue(scene_name)
    conv = PT.render_gpu(cs, RA.PATH_TRACING, spp=16384, max_bounce=8, seed=0xC0FFEE)
    ref = conv["sum"] / np.maximum(conv["count"], 1)[..., None]
    mse_g, mse_o = [], []
    for s in range(4):
        seed = 0x5EED1234 + 7919 * s
        g = PT.render_gpu(cs, RA.PATH_TRACING, spp=16, max_bounce=8, seed=seed)
        o = PT.render_oracle(cs, RA.PATH_TRACING, spp=16, max_bounce=8, seed=seed)
        mse_g.append(np.mean((g["sum"] / np.maximum(g["count"], 1)[..., None] - ref) ** 2))
        mse_o.append(np.mean((o["sum"] / np.maximum(o["count"], 1)[..., None] - ref) ** 2))
    rmse_g, rmse_o = float(np.sqrt(np.mean(mse_g))), float(np.sqrt(np.mean(mse_o)))
    assert abs(rmse_g - rmse_o) <= 0.02 * rmse_o, "RMSE device %.5f oracle %.5f" % (rmse_g, rmse_o)


def test_textures_direct_lighting_per_pixel():
    # Point light only, first bounce: each sample's radiance is kd(texture) f cos / d^2 at the
    # (possibly modified) hit, with no light sampling, so device and oracle agree per pixel.
    # Covers every texture, both modifiers, the composite materials and the textured emission.
    cs = compile_scene(G.textures_scene(resolution=(128, 72), point_light_only=True))
    g = PT.render_gpu(cs, RA.PATH_TRACING, spp=2, max_bounce=1)
    o = PT.render_oracle_no_drift(cs, RA.PATH_TRACING, spp=2, max_bounce=1)
    mg = g["sum"] / np.maximum(g["count"], 1)[..., None]
    mo = o["sum"] / np.maximum(o["count"], 1)[..., None]
    close = np.all(np.abs(mg - mo) <= 1e-3 * np.abs(mo) + 1e-4, axis=-1)
    assert close.mean() >= 0.999, "per-pixel agreement %.4f" % close.mean()
    assert mo.mean() > 0.05


def _reference_rgba8(mean, tone_mapper):
    """renderer/gpu/AbstractImageKernel.java:1104-1325 in numpy (exposure 1):
    tone mapper, sRGB redo-gamma (ColorSpaceF: break point 0.00304, gamma 2.4),
    clamp to [0, 1], * 255 + 0.5."""
    x = mean.astype(np.float32)
    if tone_mapper == 0:
        x = np.clip((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0)
    elif tone_mapper == 2:
        x = x / (1.0 + x)
    elif tone_mapper == 3:
        x = x * (1.0 + x / 16.0) / (1.0 + x)
    elif tone_mapper == 4:
        x = 1.0 - np.exp(-x)
    elif tone_mapper == 5:
        x = x / (x + 0.155) * 1.019
    slope, match, off = 12.923210180787857, 1.0553409, 0.0553409
    g = np.where(x <= 0.00304, x * slope, match * np.power(np.maximum(x, 0.0), 1.0 / 2.4) - off)
    return (np.clip(g, 0.0, 1.0) * 255.0 + 0.5).astype(np.int64)


@pytest.mark.parametrize("tone_mapper", [0, 1, 2, 3, 4, 5])
def test_tone_mappers_and_srgb_resolve(cornell, tone_mapper):
    from dayflower_b200 import GPURenderer
    r = GPURenderer()
    try:
        r.setScene(cornell)
        r.setRenderingAlgorithm(RA.PATH_TRACING)
        r.setMaximumBounce(6)
        r.setToneMapper(tone_mapper)
        r.setup()
        r.render(4)
        s, _, n = r.getFilm()
        img = r.getImage().astype(np.int64)
    finally:
        r.dispose()
    want = _reference_rgba8(s / np.maximum(n, 1)[..., None], tone_mapper)
    assert np.all(img[..., 3] == 255)
    assert np.abs(img[..., :3] - want).max() <= 1  # float rounding at a code boundary


def _gpu_pixel_film(cs, algorithm, spp, max_bounce=8, seed=0x5EED1234):
    from dayflower_b200 import GPURenderer
    r = GPURenderer()
    try:
        r.setScene(cs)
        r.setRenderingAlgorithm(algorithm)
        r.setMaximumBounce(max_bounce)
        r.setSeed(seed)
        r.setFilmFilter(GPURenderer.FILM_GAUSSIAN)
        r.setup()
        assert r.render(spp)
        return r.getPixelFilm(), r.getImage()
    finally:
        r.dispose()


def _film_render(xyzw):
    """PixelImageF.filmRender without splats: XYZ -> linear sRGB over the weight sum, negatives dropped."""
    from oracle import dfo
    m = np.array([[3.2404542, -1.5371385, -0.4985314], [-0.9692660, 1.8760108, 0.0415560], [0.0556434, -0.2040259, 1.0572252]])
    rgb = xyzw[..., :3] @ m.T
    w = xyzw[..., 3:4]
    return np.where(w != 0, np.maximum(rgb / np.where(w != 0, w, 1), 0), rgb)


def test_gaussian_pixel_film_matches_cpu_renderer_film(cornell):
    from oracle import dfo
    o = dfo.OracleScene(cornell)
    # RAY_CASTING: deterministic per sample, so the splatted films agree closely
    g, img = _gpu_pixel_film(cornell, RA.RAY_CASTING, 4)
    ref = o.render_pixel_film(RA.RAY_CASTING, spp=4, threads=8)
    assert np.allclose(g[..., 3], ref[..., 3], rtol=1e-4, atol=1e-6)
    close = np.all(np.abs(g[..., :3] - ref[..., :3]) <= 1e-3 * np.abs(ref[..., :3]) + 1e-5, axis=-1)
    assert close.mean() >= 0.999
    # the RGBA8 resolve of this film is PixelImageF.filmRender + sRGB
    want = _reference_rgba8(_film_render(ref.astype(np.float64)), 1)
    assert np.mean(np.abs(img[..., :3].astype(np.int64) - want) <= 1) >= 0.999
    # PATH_TRACING: same samples, the image means agree
    g, _ = _gpu_pixel_film(cornell, RA.PATH_TRACING, 8)
    ref = o.render_pixel_film(RA.PATH_TRACING, spp=8, max_bounce=8, threads=8)
    mg, mo = _film_render(g.astype(np.float64)).mean(), _film_render(ref.astype(np.float64)).mean()
    assert abs(mg - mo) <= 0.02 * mo
