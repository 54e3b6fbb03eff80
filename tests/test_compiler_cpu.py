"""Scene compiler (the producer of the reference's flattened arrays) and the
layout rules of scene/compiler/*.java, checked on the CPU."""
import numpy as np
import pytest

from dayflower_b200.scene import generators as G
from dayflower_b200.scene import model as M
from dayflower_b200.scene.compiler import compile_scene


def walk_mesh(stream, off):
    """Visits every node of a threaded mesh stream (CompiledShape3FCache.java:2652)."""
    tris, rel, seen = [], 0, 0
    while rel != -1:
        seen += 1
        assert seen <= len(stream) // 8 + 1
        o = off + rel
        nid, nxt, lc = stream[o], stream[o + 2], stream[o + 3]
        if nid == 1:
            tris += list(stream[o + 4:o + 4 + lc])
            assert lc < 4  # BVHNode3Fs.java:67, fewer than four items make a leaf
            rel = nxt
        else:
            assert nid == 2 and lc == rel + 8  # the left child follows in depth-first order
            rel = lc
    return tris


def test_cornell_layout():
    cs = compile_scene(G.cornell_box(resolution=(64, 64)))
    a = cs.arrays
    assert a["primitiveArray"].size == 9 * 8
    assert a["primitiveMatrix44FArray"].size == 9 * 32
    assert a["cameraArray"].size == 19 and a["cameraArray"][17] == 64
    assert a["shape3FRectangle3FArray"].size == 5 * 16
    assert a["lightDiffuseAreaLightArray"].size == 2 * 40
    ids = a["lightIDAndOffsetArray"].view(np.uint32)
    assert list(ids >> 16) == [1, 1] and list(ids & 0xFFFF) == [0, 1]
    prim = a["primitiveArray"].reshape(-1, 8)
    # area-light primitives reference their light with the same 16/16 pack
    assert set(prim[-2:, 1].view(np.uint32) >> 16) == {1}
    # material offsets are absolute (MatteMaterial records are 2 ints)
    matte = prim[prim[:, 4] == M.MAT_MATTE, 5]
    assert all(o % 2 == 0 for o in matte)


def test_mesh_stream_covers_every_triangle_once():
    mesh, _ = G.heightfield_mesh(16, 10.0, seed=1)
    sc = M.Scene(camera=M.Camera((0, 5, 10), (0, 0, 0), resolution=(8, 8)))
    sc.add(M.Primitive(mesh, M.Matte()))
    cs = compile_scene(sc)
    stream = cs.arrays["shape3FTriangleMesh3FArray"]
    offs = walk_mesh(stream, int(cs.arrays["primitiveArray"][7]))
    assert sorted(offs) == [24 * i for i in range(16 * 16 * 2)]
    # every node's box (relative index into the AABB array) contains its triangles
    boxes = cs.arrays["boundingVolume3FAxisAlignedBoundingBox3FArray"].reshape(-1, 8)
    tri = cs.arrays["shape3FTriangle3FArray"].reshape(-1, 24)
    n = stream.size // 8
    for k in range(n):
        node = stream[k * 8:(k + 1) * 8]
        if node[0] == 1:
            b = boxes[node[1]]
            for t in node[4:4 + node[3]]:
                p = tri[t // 24, 0:9].reshape(3, 3)
                assert np.all(p <= b[0:3] + 1e-6) and np.all(p >= b[3:6] - 1e-6)


def test_layout1_texture_overflow_raises_and_layout2_compiles():
    sc = G.terrain_spheres(cells=8, n_spheres=400, resolution=(16, 16), seed=5, extent=20.0)
    with pytest.raises(ValueError):
        compile_scene(sc, layout_version=1)
    cs = compile_scene(sc, layout_version=2)
    assert cs.stats["textures"] > 256


def test_layout2_widens_material_slots():
    sc = G.cornell_box(resolution=(8, 8))
    a1 = compile_scene(sc, 1).arrays
    a2 = compile_scene(sc, 2).arrays
    assert a2["materialMatteMaterialArray"].size == 4 * a1["materialMatteMaterialArray"].size
    v1 = a1["materialMatteMaterialArray"].view(np.uint32)
    v2 = a2["materialMatteMaterialArray"]
    for k in range(v1.size):
        assert [int((v1[k] >> (8 * j)) & 0xFF) for j in range(4)] == list(v2[4 * k:4 * k + 4])


def test_oracle_identical_on_both_layouts(oracle):
    sc = G.small_mixed_scene(resolution=(24, 16))
    r = []
    for layout in (1, 2):
        o = oracle.OracleScene(compile_scene(sc, layout))
        r.append(o.render(2, spp=2, max_bounce=4, threads=4))
    assert np.array_equal(r[0]["sum"], r[1]["sum"]) and np.array_equal(r[0]["prim"], r[1]["prim"])


def test_perez_record_layout():
    from dayflower_b200.scene.perez import perez_record
    rec = perez_record(2.5, (0.5, 0.6, 0.3))
    assert rec.size % 8 == 0
    assert rec[41] == np.float32(2.5) and rec[45] == 10.0
    # the distribution header: isUV, offset table length, marginal offset
    d = rec[48:]
    assert d[0] == 1.0 and d[1] == 33.0 and d[2] == 35.0
    marginal = int(d[2])
    assert d[marginal + 2] == 32 and d[marginal + 1] == 33  # 32 entries, 33 CDF values
    assert abs(d[marginal + 4 + 32] - 1.0) < 1e-6  # CDF ends at 1
    assert np.all(rec[32:35] > 0)  # the sun is above the horizon: a positive sun colour


def test_oracle_render_counts_and_guard(oracle):
    cs = compile_scene(G.cornell_box(resolution=(16, 16)))
    o = oracle.OracleScene(cs)
    r = o.render(2, spp=3, max_bounce=4, threads=2)
    assert r["count"].max() <= 3 and r["count"].min() >= 0
    assert np.all(np.isfinite(r["sum"]))
    assert r["rays"] > 16 * 16 * 3


def test_record_shapes_layout_and_oracle():
    """Disk ... torus and polygons compile into their reference records (CompiledShape3FCache.to*3F)
    and every one of them is hit by the oracle's primary rays."""
    import numpy as np

    from dayflower_b200.scene import generators as G
    from dayflower_b200.scene import model as M
    from dayflower_b200.scene.compiler import compile_scene
    from oracle import dfo

    cs = compile_scene(G.quadrics_scene(resolution=(64, 48)))
    a = cs.arrays
    assert a["shape3FDisk3FArray"].size == 4 and a["shape3FCylinder3FArray"].size == 8
    assert a["shape3FCone3FArray"].size == 4 and a["shape3FCone3FArray"][3] == 0.0
    assert a["shape3FHyperboloid3FArray"].size == 16 and a["shape3FRectangularCuboid3FArray"].size == 8
    assert a["shape3FTorus3FArray"].tolist() == [0.35, 1.0, 0.25, 0.800000011920929] or np.allclose(a["shape3FTorus3FArray"], [0.35, 1.0, 0.25, 0.8])
    assert np.float32(a["shape3FDisk3FArray"][0]) == np.float32(np.radians(300.0))
    prims = a["primitiveArray"].reshape(-1, 8)
    offsets = {int(sid): sorted(set(prims[prims[:, 6] == sid, 7].tolist())) for sid in np.unique(prims[:, 6])}
    assert offsets[M.SHAPE_CYLINDER] == [0, 4] and offsets[M.SHAPE_TORUS] == [0, 2]
    o = dfo.OracleScene(cs)
    res = o.render(3, spp=1, threads=4)
    hit = set(res["prim"].ravel().tolist())
    record_prims = [i for i, p in enumerate(prims) if p[6] in (M.SHAPE_DISK, M.SHAPE_CYLINDER, M.SHAPE_CONE, M.SHAPE_PARABOLOID,
                                                             M.SHAPE_HYPERBOLOID, M.SHAPE_CUBOID, M.SHAPE_TORUS, M.SHAPE_POLYGON)]
    assert len(record_prims) == 11
    pg = a["shape3FPolygon3FArray"]
    assert pg[12] == 5 and pg.size % 8 == 0  # 13 + 2 * 5 floats padded to 24, then the hexagon
    assert pg[24 + 12] == 6
    assert set(record_prims) <= hit


def test_hyperboloid_coefficients_match_reference_constructor():
    """Hyperboloid3F(phiMax, a, b) solves aH and cH so that b and c = a + 2 (b - a)
    (the constructor's first probe point) lie on aH (x^2 + y^2) - cH z^2 = 1
    (Hyperboloid3F.java:144-178)."""
    import numpy as np

    from dayflower_b200.scene import model as M

    h = M.Hyperboloid(360.0, (0.3, 0.3, 0.0), (1.0, 0.2, 2.0))
    c = h.a + 2.0 * (h.b - h.a)
    for p in (h.b, c):
        assert abs(h.aH * (p[0] ** 2 + p[1] ** 2) - h.cH * p[2] ** 2 - 1.0) < 1e-4
    assert h.z_min == 0.0 and h.z_max == 2.0 and np.isclose(h.r_max, np.sqrt(1.04))
