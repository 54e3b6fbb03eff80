"""CompiledSceneModifier (scene/compiler/CompiledSceneModifier.java): adding a
primitive to a compiled scene gives the arrays of compiling the scene with it;
removing it gives back the primitive and matrix arrays; equal records and
lights are refused as the reference refuses them."""
import numpy as np

from dayflower_b200.scene import generators as G
from dayflower_b200.scene import model as M
from dayflower_b200.scene.compiler import CompiledSceneModifier, compile_scene


def _extra():
    mesh, _ = G.heightfield_mesh(6, 2.0, seed=9)
    return [M.Primitive(M.Sphere(), M.Plastic(kd=M.CheckerboardTexture(scale=(4.0, 2.0))), M.Transform.translate_scale((1.0, 2.0, 0.5), 0.5)),
            M.Primitive(mesh, M.Matte(kd=(0.3, 0.6, 0.2)), M.Transform.translate_scale((-1.0, 1.0, 0.0), 1.0)),
            M.Primitive(M.Torus(0.2, 0.6), M.Metal(), M.Transform.translate_scale((0.0, 3.0, 0.0), 1.0))]


def test_add_matches_a_full_compile():
    for lv in (1, 2):
        base = G.small_mixed_scene(resolution=(32, 24))
        extra = _extra()
        full = G.small_mixed_scene(resolution=(32, 24))
        for p in extra:
            full.add(p)
        cs = compile_scene(base, layout_version=lv)
        m = CompiledSceneModifier(cs)
        for p in extra:
            assert m.add_primitive(p)
        want = compile_scene(full, layout_version=lv).arrays
        for k in want:
            assert np.array_equal(cs.arrays[k], want[k]), k
        assert cs.version == len(extra)


def test_remove_and_refusals():
    sc = G.small_mixed_scene(resolution=(32, 24))
    cs = compile_scene(sc, layout_version=2)
    prims0 = cs.arrays["primitiveArray"].copy()
    mats0 = cs.arrays["primitiveMatrix44FArray"].copy()
    m = CompiledSceneModifier(cs)
    p = _extra()[0]
    assert m.add_primitive(p)
    assert not m.add_primitive(p)  # an equal record exists (CompiledPrimitiveCache.addPrimitive)
    assert cs.arrays["primitiveArray"].size == prims0.size + 8
    assert m.remove_primitive(p)
    assert np.array_equal(cs.arrays["primitiveArray"], prims0) and np.array_equal(cs.arrays["primitiveMatrix44FArray"], mats0)
    assert not m.remove_primitive(p)
    # removing a primitive of the original scene drops exactly its record and matrices
    victim = sc.primitives[3]
    assert m.remove_primitive(victim)
    rows = prims0.reshape(-1, 8)
    assert np.array_equal(cs.arrays["primitiveArray"].reshape(-1, 8), np.delete(rows, 3, axis=0))
    assert np.array_equal(cs.arrays["primitiveMatrix44FArray"].reshape(-1, 32), np.delete(mats0.reshape(-1, 32), 3, axis=0))
    # lights are neither added nor removed (CompiledSceneModifier.addLight / removeLight)
    assert not m.add_light(M.PointLight((0, 5, 0), (1, 1, 1)))
    assert not m.remove_light(sc.lights[0])


import pytest  # noqa: E402


@pytest.mark.gpu
def test_renderer_uploads_a_modified_scene():
    # AbstractGPURenderer.render -> updateCompiledScene: the next render sees the change and starts a new film
    from dayflower_b200 import GPURenderer, RenderingAlgorithm as RA
    sc = G.small_mixed_scene(resolution=(64, 48))
    victim = sc.primitives[-1]
    cs = compile_scene(sc, layout_version=2)
    r = GPURenderer()
    try:
        r.setScene(cs)
        r.setRenderingAlgorithm(RA.RAY_CASTING)
        r.setup()
        r.render(2)
        before, _, _ = r.getFilm()
        m = CompiledSceneModifier(cs)
        assert m.remove_primitive(victim)
        extra = _extra()
        for p in extra:
            assert m.add_primitive(p)
        r.render(2)
        after, _, n = r.getFilm()
    finally:
        r.dispose()
    assert np.all(n == 2)  # the film restarted
    fresh_scene = G.small_mixed_scene(resolution=(64, 48))
    fresh_scene.primitives.remove(fresh_scene.primitives[-1])
    for p in extra:
        fresh_scene.add(p)
    q = GPURenderer()
    try:
        q.setScene(compile_scene(fresh_scene, layout_version=2))
        q.setRenderingAlgorithm(RA.RAY_CASTING)
        q.setup()
        q.render(2)
        want, _, _ = q.getFilm()
    finally:
        q.dispose()
    assert np.allclose(after, want, rtol=1e-6, atol=1e-7)
    assert not np.allclose(before, want)
