"""The CPU oracle's primitive math against the golden vectors of the
reference's own unit tests (src/test/java/org/dayflower/..., cited per test).
These pin the oracle before it is trusted as the checker."""
import math

import numpy as np
import pytest

from oracle import dfo

f32 = dfo.f32


def plane(o, d, tmin, tmax):
    out = np.zeros(18, np.float32)
    hit = dfo.lib().dfo_plane_intersection(dfo.ptr(f32(*o)), dfo.ptr(f32(*d)), tmin, tmax, dfo.ptr(out))
    return hit, out


def test_plane_intersection_golden():
    # geometry/shape/Plane3FUnitTests.java:152-171
    hit, s = plane((1, 3, 2), (0, 0, -1), 0.0, 3.0)
    assert hit == 1
    t, p, gw, gv, gu, sw, uv = s[0], s[1:4], s[4:7], s[7:10], s[10:13], s[13:16], s[16:18]
    assert t == 2.0
    assert list(p) == [1.0, 3.0, 0.0]
    assert list(gw) == [0.0, 0.0, 1.0] and list(gv) == [0.0, 1.0, 0.0] and list(gu) == [1.0, 0.0, 0.0]
    assert list(sw) == [0.0, 0.0, 1.0]
    assert list(uv) == [1.0, 3.0]
    assert plane((0, 0, 0), (1, 0, 0), 0.0, 1.0)[0] == 0


def sphere_t(o, d, tmin, tmax):
    return dfo.lib().dfo_sphere_intersection_t(dfo.ptr(f32(*o)), dfo.ptr(f32(*d)), tmin, tmax)


def test_sphere_intersection_t_golden():
    # geometry/shape/Sphere3DUnitTests.java:188-196 (double class; the float unit sphere agrees)
    assert math.isnan(sphere_t((0, 0, 2), (0, 0, -1), 0.0, 1.0))
    assert math.isnan(sphere_t((0, 0, 2), (0, 0, 1), 0.0, 1.0))
    assert math.isnan(sphere_t((0, 0, -2), (0, 0, -1), 0.0, 1.0))
    assert math.isnan(sphere_t((0, 0, -2), (0, 0, 1), 0.0, 1.0))
    assert math.isnan(sphere_t((2, 0, 0), (0, 0, 1), 0.0, 2.0))
    assert sphere_t((0, 0, 0), (0, 0, 1), 0.0, 2.0) == 1.0
    assert sphere_t((0, 0, 2), (0, 0, -1), 0.0, 2.0) == 1.0


def test_sphere_intersection_golden():
    # geometry/shape/Sphere3DUnitTests.java:149-176: point (0,0,1), normals (0,0,1), t = 1
    out = np.zeros(18, np.float32)
    assert dfo.lib().dfo_sphere_intersection(dfo.ptr(f32(0, 0, 2)), dfo.ptr(f32(0, 0, -1)), 0.0, 3.0, dfo.ptr(out)) == 1
    assert out[0] == 1.0
    # Sphere3F nudges a pole hit to x = 1e-5 r before computing phi (Sphere3F.java:276)
    assert np.allclose(out[1:4], [0, 0, 1], atol=2e-5)
    assert np.allclose(out[4:7], [0, 0, 1], atol=1e-4) and np.allclose(out[13:16], [0, 0, 1], atol=1e-4)
    assert dfo.lib().dfo_sphere_intersection(dfo.ptr(f32(1, 0, 0)), dfo.ptr(f32(1, 0, 0)), 0.0, 1.0, dfo.ptr(out)) == 0


def aabb(o, d, tmin, tmax):
    t = np.zeros(1, np.float32)
    bb = f32(5, 5, 10, -5, -5, 5, 0, 0)  # max xyz, min xyz (CompiledBoundingVolume3FCache layout)
    dfo.lib().dfo_aabb_intersection(dfo.ptr(bb), dfo.ptr(f32(*o)), dfo.ptr(f32(*d)), tmin, tmax, dfo.ptr(t))
    return float(t[0])


def test_aabb_intersection_golden():
    # geometry/boundingvolume/AxisAlignedBoundingBox3FUnitTests.java:284-306
    big = float(np.finfo(np.float32).max)
    assert aabb((0, 0, 0), (0, 0, 1), 0.0, big) == 5.0
    assert aabb((0, 0, 0), (0, 0, 1), 5.0, big) == 10.0
    assert math.isnan(aabb((0, 0, 0), (0, 0, 1), 10.0, big))
    assert math.isnan(aabb((0, 0, 0), (0, 0, 1), 0.0, 5.0))
    assert math.isnan(aabb((0, 0, 0), (1, 0, 0), 0.0, big))


def test_ray_transform_golden():
    # geometry/Ray3FUnitTests.java:169-184: the identity leaves a ray unchanged
    eye = np.eye(4, dtype=np.float32).reshape(-1)
    out = np.zeros(6, np.float32)
    dfo.lib().dfo_ray_transform(dfo.ptr(eye), dfo.ptr(f32(0, 0, 0)), dfo.ptr(f32(1, 0, 0)), dfo.ptr(out))
    assert list(out) == [0, 0, 0, 1, 0, 0]
    dfo.lib().dfo_ray_transform(dfo.ptr(eye), dfo.ptr(f32(0, 0, 0)), dfo.ptr(f32(0, 0, 0)), dfo.ptr(out))
    assert list(out[:3]) == [0, 0, 0] and np.all(np.isnan(out[3:]))  # a zero direction normalizes to NaN both times


def rot(axis, deg):
    a = np.float32(math.radians(deg))
    c, s = np.float32(math.cos(a)), np.float32(math.sin(a))
    m = np.eye(4, dtype=np.float32)
    i, j = {"x": (1, 2), "y": (2, 0), "z": (0, 1)}[axis]
    m[i, i], m[i, j], m[j, i], m[j, j] = c, -s, s, c
    return m.reshape(-1)


def onb_transform(m, onb):
    out = np.zeros(9, np.float32)
    dfo.lib().dfo_onb_transform(dfo.ptr(np.ascontiguousarray(m, np.float32)), dfo.ptr(f32(*onb)), dfo.ptr(out))
    return out


def test_onb_transform_golden():
    # geometry/OrthonormalBasis33FUnitTests.java:324-345 (w, v, u order)
    a = (0, 0, 1, 0, 1, 0, 1, 0, 0)
    e = 0.0000000874227766
    assert np.allclose(onb_transform(rot("x", 180), a), [0, e, -1, 0, -1, -e, 1, 0, 0], atol=1e-12)
    assert np.allclose(onb_transform(rot("y", 180), a), [-e, 0, -1, 0, 1, 0, -1, 0, e], atol=1e-12)
    assert np.allclose(onb_transform(rot("z", 180), a), [0, 0, 1, e, -1, 0, -1, -e, 0], atol=1e-12)
    b = onb_transform(rot("x", 180), a)
    assert np.allclose(onb_transform(rot("x", -180), b), a, atol=1e-7)


def test_onb_from_w():
    # OrthonormalBasis33F(w) builds a right-handed orthonormal frame around w
    out = np.zeros(9, np.float32)
    dfo.lib().dfo_onb_from_w(dfo.ptr(f32(0.3, -0.5, 0.8)), dfo.ptr(out))
    w, v, u = out[0:3], out[3:6], out[6:9]
    for x in (w, v, u):
        assert abs(np.linalg.norm(x) - 1) < 1e-6
    assert abs(w @ v) < 1e-6 and abs(w @ u) < 1e-6 and abs(u @ v) < 1e-6
    assert np.allclose(np.cross(v, w), u, atol=1e-6)


IDENTITY_CS = f32(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0, 1.0)  # color/ColorSpaceF.java:65


def cs(params, op, c):
    out = np.zeros(3, np.float32)
    dfo.lib().dfo_colorspace(dfo.ptr(params), op, dfo.ptr(f32(*c)), dfo.ptr(out))
    return out


def test_colorspace_golden():
    # color/ColorSpaceFUnitTests.java:58-128 (IDENTITY colour space)
    b = cs(IDENTITY_CS, 0, (0.5, 0.5, 0.5))
    assert list(b) == [0.5, 0.5, -0.5]
    assert list(cs(IDENTITY_CS, 1, b)) == [0.5, 0.5, 0.5]
    assert list(cs(IDENTITY_CS, 2, (0.5, 0.5, 0.5))) == [0.5, 0.5, 0.5]
    assert list(cs(IDENTITY_CS, 2, (2, 2, 2))) == [2, 2, 2]
    assert list(cs(IDENTITY_CS, 3, (0.5, 0.5, 0.5))) == [0.5, 0.5, 0.5]
    assert list(cs(IDENTITY_CS, 3, (2, 2, 2))) == [2, 2, 2]


def test_srgb_round_trip():
    L = dfo.lib()
    for v in (0.0, 0.001, 0.00304, 0.1, 0.5, 1.0):
        assert abs(L.dfo_srgb_undo(L.dfo_srgb_redo(v)) - v) <= 1e-6 + 1e-5 * v
    out = np.zeros(3, np.float32)
    back = np.zeros(3, np.float32)
    L.dfo_rgb_to_xyz(dfo.ptr(f32(0.2, 0.5, 0.9)), dfo.ptr(out))
    L.dfo_xyz_to_rgb(dfo.ptr(out), dfo.ptr(back))
    assert np.allclose(back, [0.2, 0.5, 0.9], atol=1e-5)


def test_gaussian_filter_golden():
    # filter/GaussianFilter2FUnitTests.java:89-104
    e0, e2, e8 = np.float32(math.exp(-0.0)), np.float32(math.exp(-2.0)), np.float32(math.exp(-8.0))
    g = dfo.lib().dfo_gaussian_filter
    assert g(0, 0, 2, 2, 2) == pytest.approx(float((e0 - e8) * (e0 - e8)), rel=1e-6)
    assert g(0, 1, 2, 2, 2) == pytest.approx(float((e0 - e8) * (e2 - e8)), rel=1e-6)
    assert g(1, 0, 2, 2, 2) == pytest.approx(float((e2 - e8) * (e0 - e8)), rel=1e-6)
    assert g(1, 1, 2, 2, 2) == pytest.approx(float((e2 - e8) * (e2 - e8)), rel=1e-6)


def test_triangle_filter_golden():
    # filter/TriangleFilter2FUnitTests.java:81-89 (default resolution 2 x 2)
    t = dfo.lib().dfo_triangle_filter
    assert t(0, 0, 2, 2) == 4.0 and t(0, 1, 2, 2) == 2.0 and t(1, 0, 2, 2) == 2.0 and t(1, 1, 2, 2) == 1.0


def test_triangle_watertight_edges():
    # geometry/shape/Triangle3F.java:505: a ray through a shared edge hits exactly one
    # of two adjacent triangles' interiors or both at the same t, never neither.
    tri_a = np.zeros(24, np.float32)
    tri_b = np.zeros(24, np.float32)
    tri_a[0:9] = [0, 0, 0, 1, 0, 0, 0, 1, 0]
    tri_b[0:9] = [1, 0, 0, 1, 1, 0, 0, 1, 0]
    L = dfo.lib()
    rng = np.random.default_rng(3)
    for _ in range(200):
        s = np.float32(rng.uniform(0.01, 0.99))
        o = f32(s, 1 - s, 5.0)
        ta = L.dfo_triangle_intersection_t(dfo.ptr(tri_a), dfo.ptr(o), dfo.ptr(f32(0, 0, -1)), 0.001, 100.0)
        tb = L.dfo_triangle_intersection_t(dfo.ptr(tri_b), dfo.ptr(o), dfo.ptr(f32(0, 0, -1)), 0.001, 100.0)
        assert not (math.isnan(ta) and math.isnan(tb))


def test_rng_streams_are_keyed():
    L = dfo.lib()
    k1, k2 = L.dfo_rng_path_key(1, 10, 0), L.dfo_rng_path_key(1, 10, 1)
    assert k1 != k2
    u = [L.dfo_rng_uniform(k1, d) for d in range(2000)]
    assert 0.0 <= min(u) and max(u) < 1.0
    assert abs(np.mean(u) - 0.5) < 0.03
