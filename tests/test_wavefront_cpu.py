"""Wavefront OBJ input (TriangleMesh3F.readWavefrontObject semantics) on small
hand-written files."""
import io

import numpy as np
import pytest

from dayflower_b200.scene import model as M
from dayflower_b200.scene.compiler import compile_scene
from dayflower_b200.scene.wavefront import read_wavefront_obj

QUADS = """# two quads, two groups, one material change
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0 0 1
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
g front
usemtl red
f 1/1/1 2/2/1 3/3/1 4/4/1
g side
f 1//1 4//1 5//1
usemtl blue
o thing
f 2 3 5
"""


def test_fan_triangulation_groups_and_attributes():
    meshes = read_wavefront_obj(io.StringIO(QUADS))
    assert [(m.group_name, m.material_name) for m in meshes] == [("front", "red"), ("side", "red"), ("side", "blue")]
    assert [m.triangles.shape[0] for m in meshes] == [2, 1, 1]
    t = meshes[0].triangles
    # the quad fans around its first vertex: (1, 2, 3) and (1, 3, 4)
    assert np.allclose(t[0, 0:9], [0, 0, 0, 1, 0, 0, 1, 1, 0]) and np.allclose(t[1, 0:9], [0, 0, 0, 1, 1, 0, 0, 1, 0])
    assert np.allclose(t[1, 9:15], [0, 0, 1, 1, 0, 1])
    assert np.allclose(t[:, 15:24], np.tile([0, 0, 1], (2, 3)))
    # no texture coordinate reference: (0, 0)
    assert np.allclose(meshes[1].triangles[0, 9:15], 0.0)
    assert meshes[2].object_name == "thing"


def test_flip_and_scale():
    m = read_wavefront_obj(io.StringIO(QUADS), flip_texture_v=True, scale=2.0)[0].triangles
    assert np.allclose(m[0, 0:9], 2.0 * np.array([0, 0, 0, 1, 0, 0, 1, 1, 0]))
    assert np.allclose(m[0, 9:15], [0, 1, 1, 1, 1, 0])
    assert np.allclose(m[0, 15:18], [0, 0, 0.5])  # transpose of the inverse scale, not renormalised


def test_smooth_normals_without_vn():
    # a unit cube without normals: a corner's normal is the normalised sum of the normalised
    # normals of the triangles that use it (IndexedObjectModel.calculateNormals)
    verts = np.array([(x, y, z) for x in (0, 1) for y in (0, 1) for z in (0, 1)], dtype=np.float64)
    faces = [(1, 2, 4, 3), (5, 7, 8, 6), (1, 5, 6, 2), (3, 4, 8, 7), (1, 3, 7, 5), (2, 6, 8, 4)]
    src = "".join("v %d %d %d\n" % tuple(v) for v in verts) + "".join("f %d %d %d %d\n" % f for f in faces)
    m = read_wavefront_obj(io.StringIO(src))
    assert len(m) == 1 and m[0].triangles.shape[0] == 12
    tris = [(f[0] - 1, f[1 + i] - 1, f[2 + i] - 1) for f in faces for i in range(2)]
    acc = np.zeros((8, 3))
    for a, b, c in tris:
        n = np.cross(verts[b] - verts[a], verts[c] - verts[a])
        for v in (a, b, c):
            acc[v] += n / np.linalg.norm(n)
    want = acc / np.linalg.norm(acc, axis=1, keepdims=True)
    t = m[0].triangles
    for j, (a, b, c) in enumerate(tris):
        assert np.allclose(t[j, 15:24], np.concatenate([want[a], want[b], want[c]]), atol=1e-6)
    # every corner normal points out of the cube
    for k in range(3):
        assert np.all(np.sum((t[:, 3 * k:3 * k + 3] - 0.5) * t[:, 15 + 3 * k:18 + 3 * k], axis=1) > 0.0)


def test_bad_reference_and_compile():
    with pytest.raises(ValueError):
        read_wavefront_obj(io.StringIO("v 0 0 0\nf 1 2 3\n"))
    meshes = read_wavefront_obj(io.StringIO(QUADS))
    sc = M.Scene(camera=M.Camera((0.5, 0.5, 4), (0.5, 0.5, 0), resolution=(16, 16)))
    for mesh in meshes:
        sc.add(M.Primitive(mesh, M.Matte()))
    cs = compile_scene(sc)
    assert cs.arrays["shape3FTriangle3FArray"].size == 4 * 24
