"""The device builder of the mesh hierarchies against the host builder: the
same closest hits (primitive and distance) on every pixel, for scenes with
large meshes, instanced meshes and the degenerate cases a radix tree over
Morton codes meets (meshes of one to five triangles; every triangle with the
same centroid, so that all codes are equal)."""
import numpy as np
import pytest

from dayflower_b200 import GPURenderer, RenderingAlgorithm as RA
from dayflower_b200.scene import generators as G
from dayflower_b200.scene import model as M
from dayflower_b200.scene.compiler import compile_scene

pytestmark = pytest.mark.gpu


def _primary(cs, builder):
    r = GPURenderer()
    try:
        r.setBVHBuilder(builder)
        r.setScene(cs)
        r.setRenderingAlgorithm(RA.RAY_CASTING)
        r.setup()
        assert r.render(1)
        prim, t = r.getPrimaryHits()
        s, _, n = r.getFilm()
        return prim, t, s
    finally:
        r.dispose()


def _tiny_meshes_scene():
    sc = M.Scene(camera=M.Camera(eye=(0.0, 2.0, 9.0), look_at=(0.0, 0.5, 0.0), fov_x_deg=60.0, resolution=(96, 64)))
    rng = np.random.default_rng(4)
    for k, n in enumerate([1, 2, 3, 4, 5, 9]):
        pos = rng.uniform(-0.6, 0.6, size=(3 * n, 3)).astype(np.float32)
        idx = np.arange(3 * n).reshape(n, 3)
        mesh = M.TriangleMesh.from_positions(pos, idx)
        sc.add(M.Primitive(mesh, M.Matte(kd=(0.6, 0.5, 0.4)), M.Transform.translate_scale((-3.5 + 1.4 * k, 0.8, 0.0), 1.0)))
    # 200 triangles sharing one centroid: all Morton codes equal
    ang = np.linspace(0.0, np.pi, 200, endpoint=False)
    pos = []
    for a in ang:
        d = np.array([np.cos(a), np.sin(a), 0.3 * np.sin(3 * a)])
        e = np.array([-np.sin(a), np.cos(a), 0.1])
        pos += [d, -0.5 * d + 0.8 * e, -0.5 * d - 0.8 * e]
    mesh = M.TriangleMesh.from_positions(np.array(pos, dtype=np.float32), np.arange(600).reshape(200, 3))
    sc.add(M.Primitive(mesh, M.Matte(kd=(0.3, 0.6, 0.8)), M.Transform.translate_scale((0.0, 2.2, -1.0), 0.8)))
    sc.add(M.Primitive(M.Plane(), M.Matte(kd=(0.5, 0.5, 0.5)), G._rot_x(-90.0, (0.0, 0.0, 0.0))))
    sc.lights.append(M.PointLight((2.0, 6.0, 5.0), (40.0, 40.0, 40.0)))
    return sc


@pytest.mark.parametrize("name", ["terrain", "instances", "mixed", "tiny"])
def test_device_and_host_hierarchies_hit_alike(name):
    if name == "terrain":
        cs = compile_scene(G.terrain_spheres(cells=256, n_spheres=300, resolution=(320, 180), seed=11), layout_version=2)
    elif name == "instances":
        cs = compile_scene(G.large_scene(cells=48, instances=120, resolution=(128, 72), env=(128, 64), extent=40.0), layout_version=2)
    elif name == "mixed":
        cs = compile_scene(G.small_mixed_scene(resolution=(96, 64)), layout_version=2)
    else:
        cs = compile_scene(_tiny_meshes_scene(), layout_version=2)
    ph, th, sh = _primary(cs, GPURenderer.BVH_HOST)
    pd, td, sd = _primary(cs, GPURenderer.BVH_DEVICE)
    hit = ph >= 0
    assert hit.mean() > 0.2
    # the same closest primitive, at the same distance (ties between coplanar triangles of one mesh keep the primitive)
    assert np.array_equal(ph, pd)
    assert np.allclose(th[hit], td[hit], rtol=1e-6, atol=0.0)
    assert np.allclose(sh, sd, rtol=1e-5, atol=1e-7)
