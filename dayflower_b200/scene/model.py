"""Scene model: the objects Dayflower's scene compiler flattens.

This mirrors the parts of ``org.dayflower.scene`` that the GPU render path
consumes (``scene/Scene.java``, ``scene/Primitive.java``, ``scene/Camera.java``,
the shapes under ``geometry/shape/``, the materials under ``scene/material/``
and the lights under ``scene/light/``).  It exists so that scenes can be built
and compiled without a JVM; the renderer itself only ever sees the compiled
arrays produced by :mod:`dayflower_b200.scene.compiler`.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

# Type ids: the ``public static final int ID`` of each reference class.
SHAPE_CONE, SHAPE_CYLINDER, SHAPE_DISK, SHAPE_HYPERBOLOID = 2, 5, 6, 7
SHAPE_PARABOLOID, SHAPE_PLANE, SHAPE_POLYGON, SHAPE_RECTANGLE = 9, 10, 11, 13
SHAPE_CUBOID, SHAPE_SPHERE, SHAPE_TORUS, SHAPE_TRIANGLE, SHAPE_MESH = 14, 15, 16, 17, 18
MAT_DISNEY, MAT_GLASS, MAT_MATTE, MAT_METAL, MAT_MIRROR, MAT_PLASTIC = 4, 7, 11, 12, 13, 14
MAT_CLEAR_COAT, MAT_GLOSSY, MAT_SUBSTRATE, MAT_TRANSLUCENT, MAT_UBER = 3, 8, 16, 18, 19
MAT_BULLSEYE, MAT_CHECKERBOARD, MAT_POLKA_DOT = 1, 2, 15
TEX_BLEND, TEX_BULLSEYE, TEX_CHECKERBOARD, TEX_CONSTANT, TEX_DOT_PRODUCT = 1, 2, 3, 4, 5
TEX_LDR_IMAGE, TEX_MARBLE, TEX_POLKA_DOT, TEX_SIMPLEX_FBM, TEX_SURFACE_NORMAL, TEX_UV = 7, 8, 9, 10, 11, 12
MOD_NOOP, MOD_NORMAL_MAP_LDR_IMAGE, MOD_SIMPLEX_NOISE_NORMAL_MAP = 2, 3, 4
LIGHT_DIFFUSE_AREA, LIGHT_DIRECTIONAL, LIGHT_IMAGE, LIGHT_PEREZ = 1, 2, 3, 4
LIGHT_POINT, LIGHT_SPOT = 5, 7
BV_AABB, BV_SPHERE, BV_INFINITE = 1, 2, 3


def _v(x) -> np.ndarray:
    return np.asarray(x, dtype=np.float32).reshape(3)


def normalize(v) -> np.ndarray:
    v = np.asarray(v, dtype=np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


class Transform:
    """``scene/Transform.java``: an object-to-world matrix and its inverse.

    Matrices are row-major 4x4 (``Matrix44F.toArray`` order)."""

    def __init__(self, object_to_world: Optional[np.ndarray] = None):
        m = np.eye(4, dtype=np.float64) if object_to_world is None else np.asarray(object_to_world, dtype=np.float64)
        self.object_to_world = m.astype(np.float32)
        self.world_to_object = np.linalg.inv(m).astype(np.float32)

    @staticmethod
    def translate_scale(position, scale=1.0) -> "Transform":
        m = np.eye(4)
        m[0, 0] = m[1, 1] = m[2, 2] = float(scale)
        m[:3, 3] = np.asarray(position, dtype=np.float64)
        return Transform(m)

    @staticmethod
    def from_matrix(m) -> "Transform":
        return Transform(np.asarray(m, dtype=np.float64))

    def to_array(self) -> np.ndarray:
        """``CompiledPrimitiveCache.toMatrix44Fs(Transform)``: O2W then W2O."""
        return np.concatenate([self.object_to_world.reshape(-1), self.world_to_object.reshape(-1)]).astype(np.float32)


# ---------------------------------------------------------------- shapes ----
class Shape:
    ID = 0


class Sphere(Shape):
    """``geometry/shape/Sphere3F``: the unit sphere; radius comes from the transform."""
    ID = SHAPE_SPHERE


class Plane(Shape):
    """``geometry/shape/Plane3F``: the plane z = 0 in object space."""
    ID = SHAPE_PLANE


class Triangle(Shape):
    """``geometry/shape/Triangle3F`` with per-vertex texture coordinates and normals."""
    ID = SHAPE_TRIANGLE

    def __init__(self, a, b, c, uv=((0, 0), (0, 1), (1, 1)), normals=None):
        self.a, self.b, self.c = _v(a), _v(b), _v(c)
        self.uv = np.asarray(uv, dtype=np.float32).reshape(3, 2)
        if normals is None:
            n = normalize(np.cross(normalize(self.b - self.a), normalize(self.c - self.a)))
            normals = (n, n, n)
        self.normals = np.asarray(normals, dtype=np.float32).reshape(3, 3)

    def to_array(self) -> np.ndarray:
        """``CompiledShape3FCache.toTriangle3F``: 24 floats."""
        out = np.zeros(24, dtype=np.float32)
        out[0:3], out[3:6], out[6:9] = self.a, self.b, self.c
        out[9:15] = self.uv.reshape(-1)
        out[15:24] = self.normals.reshape(-1)
        return out


class TriangleMesh(Shape):
    """``geometry/shape/TriangleMesh3F``: triangles given as (N, 24) compiled rows."""
    ID = SHAPE_MESH

    def __init__(self, triangles: np.ndarray):
        t = np.ascontiguousarray(triangles, dtype=np.float32)
        assert t.ndim == 2 and t.shape[1] == 24
        self.triangles = t

    @staticmethod
    def from_positions(positions: np.ndarray, indices: np.ndarray, uvs=None, normals=None) -> "TriangleMesh":
        """Builds the (N, 24) rows from an indexed vertex list."""
        p = np.asarray(positions, dtype=np.float32)
        idx = np.asarray(indices, dtype=np.int64).reshape(-1, 3)
        n = idx.shape[0]
        rows = np.zeros((n, 24), dtype=np.float32)
        rows[:, 0:3], rows[:, 3:6], rows[:, 6:9] = p[idx[:, 0]], p[idx[:, 1]], p[idx[:, 2]]
        if uvs is not None:
            uv = np.asarray(uvs, dtype=np.float32)
            rows[:, 9:11], rows[:, 11:13], rows[:, 13:15] = uv[idx[:, 0]], uv[idx[:, 1]], uv[idx[:, 2]]
        else:
            rows[:, 9:15] = np.array([0, 0, 0, 1, 1, 1], dtype=np.float32)
        if normals is not None:
            nn = np.asarray(normals, dtype=np.float32)
            rows[:, 15:18], rows[:, 18:21], rows[:, 21:24] = nn[idx[:, 0]], nn[idx[:, 1]], nn[idx[:, 2]]
        else:
            a, b, c = rows[:, 0:3].astype(np.float64), rows[:, 3:6].astype(np.float64), rows[:, 6:9].astype(np.float64)
            e1 = b - a
            e2 = c - a
            e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
            e2 /= np.linalg.norm(e2, axis=1, keepdims=True)
            g = np.cross(e1, e2)
            g /= np.linalg.norm(g, axis=1, keepdims=True)
            rows[:, 15:18] = rows[:, 18:21] = rows[:, 21:24] = g.astype(np.float32)
        return TriangleMesh(rows)


class Rectangle(Shape):
    """``geometry/shape/Rectangle3F`` given by corners a, b, c (d = a + (c - b))."""
    ID = SHAPE_RECTANGLE

    def __init__(self, a, b, c):
        self.a, self.b, self.c = _v(a), _v(b), _v(c)
        self.d = self.a + (self.c - self.b)
        self.normal = normalize(np.cross(normalize(self.b - self.a), normalize(self.c - self.a)))

    def to_array(self) -> np.ndarray:
        """``CompiledShape3FCache.toRectangle3F``: 16 floats."""
        out = np.zeros(16, dtype=np.float32)
        out[0:3] = self.a
        out[3:6] = self.b - self.a
        out[6:9] = self.c - self.b
        out[9:12] = self.normal
        return out

    def corners(self) -> np.ndarray:
        return np.stack([self.a, self.b, self.c, self.d])


def _rad(degrees) -> float:
    """``AngleF.degrees(d).getRadians()``: the float of d * pi / 180."""
    return float(np.float32(math.radians(degrees)))


def _box_corners(lo, hi) -> np.ndarray:
    lo, hi = _v(lo), _v(hi)
    return np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])], dtype=np.float32)


class Disk(Shape):
    """``geometry/shape/Disk3F``: the annulus ri <= r <= ro at z = zMax, phi <= phiMax."""
    ID = SHAPE_DISK

    def __init__(self, phi_max_degrees=360.0, radius_inner=0.0, radius_outer=1.0, z_max=0.0):
        self.phi_max, self.ri, self.ro, self.z_max = _rad(phi_max_degrees), radius_inner, radius_outer, z_max

    def to_array(self):
        """``CompiledShape3FCache.toDisk3F``: phiMax, radiusInner, radiusOuter, zMax."""
        return np.array([self.phi_max, self.ri, self.ro, self.z_max], dtype=np.float32)

    def corners(self):
        return _box_corners((-self.ro, -self.ro, self.z_max), (self.ro, self.ro, self.z_max))


class Cylinder(Shape):
    """``geometry/shape/Cylinder3F``: radius r about z, zMin <= z <= zMax."""
    ID = SHAPE_CYLINDER

    def __init__(self, phi_max_degrees=360.0, radius=1.0, z_max=1.0, z_min=-1.0):
        self.phi_max, self.radius, self.z_max, self.z_min = _rad(phi_max_degrees), radius, z_max, z_min

    def to_array(self):
        """``CompiledShape3FCache.toCylinder3F``: phiMax, radius, zMax, zMin."""
        return np.array([self.phi_max, self.radius, self.z_max, self.z_min], dtype=np.float32)

    def corners(self):
        return _box_corners((-self.radius, -self.radius, self.z_min), (self.radius, self.radius, self.z_max))


class Cone(Shape):
    """``geometry/shape/Cone3F``: apex at z = zMax, base radius r at z = 0."""
    ID = SHAPE_CONE

    def __init__(self, phi_max_degrees=360.0, radius=1.0, z_max=1.0):
        self.phi_max, self.radius, self.z_max = _rad(phi_max_degrees), radius, z_max

    def to_array(self):
        """``CompiledShape3FCache.toCone3F``: phiMax, radius, zMax, 0."""
        return np.array([self.phi_max, self.radius, self.z_max, 0.0], dtype=np.float32)

    def corners(self):
        return _box_corners((-self.radius, -self.radius, 0.0), (self.radius, self.radius, self.z_max))


class Paraboloid(Shape):
    """``geometry/shape/Paraboloid3F``: z = zMax (x^2 + y^2) / r^2, zMin <= z <= zMax."""
    ID = SHAPE_PARABOLOID

    def __init__(self, phi_max_degrees=360.0, radius=1.0, z_max=1.0, z_min=0.0):
        self.phi_max, self.radius, self.z_max, self.z_min = _rad(phi_max_degrees), radius, z_max, z_min

    def to_array(self):
        """``CompiledShape3FCache.toParaboloid3F``: phiMax, radius, zMax, zMin."""
        return np.array([self.phi_max, self.radius, self.z_max, self.z_min], dtype=np.float32)

    def corners(self):
        return _box_corners((-self.radius, -self.radius, self.z_min), (self.radius, self.radius, self.z_max))


class Hyperboloid(Shape):
    """``geometry/shape/Hyperboloid3F``: the surface swept by the segment a-b about z.
    The coefficients follow the reference constructor (``Hyperboloid3F.java:144-178``),
    evaluated in float."""
    ID = SHAPE_HYPERBOLOID

    def __init__(self, phi_max_degrees=360.0, a=(0.0001, 0.0001, 0.0), b=(1.0, 1.0, 1.0)):
        f = np.float32
        a, b = _v(a), _v(b)
        pa = a if a[2] == 0 else (b if b[2] == 0 else a)
        pb = b if a[2] == 0 else (a if b[2] == 0 else b)
        pc = pa.copy()
        aH = cH = f(np.inf)
        with np.errstate(all="ignore"):
            for _ in range(10):
                if np.isfinite(aH):
                    break
                pc = (pc + (pb - pa) * f(2.0)).astype(np.float32)
                c = f(pc[0] * pc[0] + pc[1] * pc[1])
                d = f(pb[0] * pb[0] + pb[1] * pb[1])
                aH = f((f(1.0) / c - (pc[2] * pc[2]) / (c * pb[2] * pb[2])) / (f(1.0) - (d * pc[2] * pc[2]) / (c * pb[2] * pb[2])))
                cH = f((aH * d - f(1.0)) / (pb[2] * pb[2]))
        if not np.isfinite(aH):
            raise ValueError("degenerate hyperboloid")
        self.phi_max, self.a, self.b, self.aH, self.cH = _rad(phi_max_degrees), pa, pb, float(aH), float(cH)
        self.r_max = float(max(np.sqrt(f(a[0] * a[0] + a[1] * a[1])), np.sqrt(f(b[0] * b[0] + b[1] * b[1]))))
        self.z_max, self.z_min = float(max(a[2], b[2])), float(min(a[2], b[2]))

    def to_array(self):
        """``CompiledShape3FCache.toHyperboloid3F``: 16 floats."""
        out = np.zeros(16, dtype=np.float32)
        out[0] = self.phi_max
        out[1:4], out[4:7] = self.a, self.b
        out[7], out[8], out[9], out[10], out[11] = self.aH, self.cH, self.r_max, self.z_max, self.z_min
        return out

    def corners(self):
        return _box_corners((-self.r_max, -self.r_max, self.z_min), (self.r_max, self.r_max, self.z_max))


class RectangularCuboid(Shape):
    """``geometry/shape/RectangularCuboid3F``: an axis-aligned box in object space."""
    ID = SHAPE_CUBOID

    def __init__(self, minimum=(-0.5, -0.5, -0.5), maximum=(0.5, 0.5, 0.5)):
        self.minimum, self.maximum = _v(np.minimum(minimum, maximum)), _v(np.maximum(minimum, maximum))

    def to_array(self):
        """``CompiledShape3FCache.toRectangularCuboid3F``: maximum, minimum, 0, 0."""
        return np.concatenate([self.maximum, self.minimum, [0.0, 0.0]]).astype(np.float32)

    def corners(self):
        return _box_corners(self.minimum, self.maximum)


class Torus(Shape):
    """``geometry/shape/Torus3F``: tube radius ri around a circle of radius ro in z = 0."""
    ID = SHAPE_TORUS

    def __init__(self, radius_inner=0.25, radius_outer=1.0):
        self.ri, self.ro = radius_inner, radius_outer

    def to_array(self):
        """``CompiledShape3FCache.toTorus3F``: radiusInner, radiusOuter."""
        return np.array([self.ri, self.ro], dtype=np.float32)

    def corners(self):
        r = self.ri + self.ro  # the reference bounds it by a sphere of this radius
        return _box_corners((-r, -r, -r), (r, r, r))


class Polygon(Shape):
    """``geometry/shape/Polygon3F``: a planar polygon of n >= 3 coplanar points."""
    ID = SHAPE_POLYGON

    def __init__(self, points):
        pts = np.asarray(points, dtype=np.float32).reshape(-1, 3)
        if pts.shape[0] < 3:
            raise ValueError("a polygon needs at least 3 points")
        self.points = pts
        a, b, c = (pts[0].astype(np.float32), pts[1].astype(np.float32), pts[2].astype(np.float32))
        # Vector3F.normalNormalized(a, b, c) = normalize(cross(normalize(b - a), normalize(c - a)))
        n = np.cross(normalize(b - a), normalize(c - a))
        self.normal = normalize(n).astype(np.float32)
        u = normalize(b - a)
        v = np.cross(self.normal, u)
        d = pts - a
        if np.abs(d @ self.normal).max() > 1e-4 * max(1.0, float(np.abs(pts).max())):
            raise ValueError("The provided Point3F instances are not coplanar.")
        self.projected = np.stack([d @ u, d @ v], axis=1).astype(np.float32)  # Polygon3F.doCreateProjectedPolygon

    def to_array(self):
        """``CompiledShape3FCache.toPolygon3F``: points 0, 1, n-1, normal, count, projected points, padded to 8."""
        rec = np.concatenate([self.points[0], self.points[1], self.points[-1], self.normal, [len(self.points)],
                              self.projected.reshape(-1)]).astype(np.float32)
        return np.concatenate([rec, np.zeros((-len(rec)) % 8, dtype=np.float32)])

    def corners(self):
        return self.points


# -------------------------------------------------------------- textures ----
# A material parameter is a number, a colour or one of these (``scene/texture/``).
# Children of the pattern textures are textures or plain colours.
class Texture:
    ID = 0


@dataclass(eq=False)
class ConstantTexture(Texture):
    """``scene/texture/ConstantTexture``."""
    color: Sequence[float] = (0.5, 0.5, 0.5)
    ID = TEX_CONSTANT


@dataclass(eq=False)
class BlendTexture(Texture):
    """``scene/texture/BlendTexture``: per-channel lerp(a, b, t)."""
    a: object = (0.5, 0.5, 0.5)
    b: object = (1.0, 1.0, 1.0)
    t: Sequence[float] = (0.5, 0.5, 0.5)
    ID = TEX_BLEND


@dataclass(eq=False)
class BullseyeTexture(Texture):
    """``scene/texture/BullseyeTexture``: rings around ``origin`` (object space)."""
    a: object = (0.5, 0.5, 0.5)
    b: object = (1.0, 1.0, 1.0)
    origin: Sequence[float] = (0.0, 10.0, 0.0)
    scale: float = 1.0
    ID = TEX_BULLSEYE


@dataclass(eq=False)
class CheckerboardTexture(Texture):
    """``scene/texture/CheckerboardTexture`` over the texture coordinates."""
    a: object = (0.5, 0.5, 0.5)
    b: object = (1.0, 1.0, 1.0)
    angle_deg: float = 0.0
    scale: Sequence[float] = (1.0, 1.0)
    ID = TEX_CHECKERBOARD


@dataclass(eq=False)
class DotProductTexture(Texture):
    """``scene/texture/DotProductTexture``: |n_s . d|."""
    ID = TEX_DOT_PRODUCT


@dataclass(eq=False)
class LDRImageTexture(Texture):
    """``scene/texture/LDRImageTexture``: a packed-ARGB image, bilinear, wrapping."""
    resolution_x: int = 1
    resolution_y: int = 1
    image: object = None  # uint32 ARGB, row-major, resolution_x * resolution_y
    angle_deg: float = 0.0
    scale: Sequence[float] = (1.0, 1.0)
    ID = TEX_LDR_IMAGE


@dataclass(eq=False)
class MarbleTexture(Texture):
    """``scene/texture/MarbleTexture`` (Perlin turbulence); colours are packed to 8 bits."""
    color_a: Sequence[float] = (0.8, 0.8, 0.8)
    color_b: Sequence[float] = (0.4, 0.2, 0.1)
    color_c: Sequence[float] = (0.06, 0.04, 0.02)
    frequency: float = 1.0
    scale: float = 5.0
    stripes: float = 0.15
    octaves: int = 8
    ID = TEX_MARBLE


@dataclass(eq=False)
class PolkaDotTexture(Texture):
    """``scene/texture/PolkaDotTexture`` over the texture coordinates."""
    a: object = (0.5, 0.5, 0.5)
    b: object = (1.0, 1.0, 1.0)
    angle_deg: float = 0.0
    cell_resolution: float = 10.0
    radius: float = 0.25
    ID = TEX_POLKA_DOT


@dataclass(eq=False)
class SimplexFBMTexture(Texture):
    """``scene/texture/SimplexFractionalBrownianMotionTexture``; the colour is packed to 8 bits."""
    color: Sequence[float] = (0.75, 0.5, 0.75)
    frequency: float = 5.0
    gain: float = 0.5
    octaves: int = 16
    ID = TEX_SIMPLEX_FBM


@dataclass(eq=False)
class SurfaceNormalTexture(Texture):
    """``scene/texture/SurfaceNormalTexture``: (n_s + 1) / 2, n_s facing the ray."""
    ID = TEX_SURFACE_NORMAL


@dataclass(eq=False)
class UVTexture(Texture):
    """``scene/texture/UVTexture``: (u, v, 0)."""
    ID = TEX_UV


# ------------------------------------------------------------- modifiers ----
class Modifier:
    ID = 0


@dataclass(eq=False)
class NoOpModifier(Modifier):
    ID = MOD_NOOP


@dataclass(eq=False)
class NormalMapLDRImageModifier(Modifier):
    """``scene/modifier/NormalMapLDRImageModifier``: shading normal from an image, in the geometric frame."""
    resolution_x: int = 1
    resolution_y: int = 1
    image: object = None
    angle_deg: float = 0.0
    scale: Sequence[float] = (1.0, 1.0)
    ID = MOD_NORMAL_MAP_LDR_IMAGE


@dataclass(eq=False)
class SimplexNoiseNormalMapModifier(Modifier):
    """``scene/modifier/SimplexNoiseNormalMapModifier``: shading normal perturbed by simplex fBm."""
    frequency: float = 16.0
    scale: float = 1.0
    ID = MOD_SIMPLEX_NOISE_NORMAL_MAP


# ------------------------------------------------------------- materials ----
@dataclass(eq=False)
class Material:
    emission: Sequence[float] = (0.0, 0.0, 0.0)
    modifier: Optional[Modifier] = None
    ID = 0


@dataclass(eq=False)
class Matte(Material):
    """``scene/material/MatteMaterial``."""
    kd: Sequence[float] = (0.5, 0.5, 0.5)
    angle: float = 0.0
    ID = MAT_MATTE


@dataclass(eq=False)
class Mirror(Material):
    """``scene/material/MirrorMaterial``."""
    kr: Sequence[float] = (0.5, 0.5, 0.5)
    ID = MAT_MIRROR


@dataclass(eq=False)
class Glass(Material):
    """``scene/material/GlassMaterial``."""
    kr: Sequence[float] = (1.0, 1.0, 1.0)
    kt: Sequence[float] = (1.0, 1.0, 1.0)
    eta: float = 1.5
    roughness_u: float = 0.0
    roughness_v: float = 0.0
    remap_roughness: bool = True
    ID = MAT_GLASS


@dataclass(eq=False)
class Metal(Material):
    """``scene/material/MetalMaterial``: conductor with eta and k colours (copper defaults)."""
    eta: Sequence[float] = (0.2004, 0.9240, 1.1022)
    k: Sequence[float] = (3.9129, 2.4528, 2.1421)
    roughness_u: float = 0.01
    roughness_v: float = 0.01
    remap_roughness: bool = True
    ID = MAT_METAL


@dataclass(eq=False)
class Plastic(Material):
    """``scene/material/PlasticMaterial``."""
    kd: Sequence[float] = (0.2, 0.2, 0.5)
    ks: Sequence[float] = (0.5, 0.5, 0.5)
    roughness: float = 0.05
    remap_roughness: bool = True
    ID = MAT_PLASTIC


@dataclass(eq=False)
class Disney(Material):
    """``scene/material/DisneyMaterial`` with constant textures; the defaults are
    those of its constructor chain (DisneyMaterial.java:111-520)."""
    color: Sequence[float] = (0.5, 0.5, 0.5)
    scatter_distance: Sequence[float] = (0.0, 0.0, 0.0)
    anisotropic: float = 0.0
    clear_coat: float = 0.0
    clear_coat_gloss: float = 1.0
    diffuse_transmission: float = 1.0
    eta: float = 1.5
    flatness: float = 0.0
    metallic: float = 0.0
    roughness: float = 0.5
    sheen: float = 0.0
    sheen_tint: float = 0.5
    specular_tint: float = 0.0
    specular_transmission: float = 0.0
    thin: bool = False
    ID = MAT_DISNEY


@dataclass(eq=False)
class ClearCoat(Material):
    """``scene/material/ClearCoatMaterial`` (defaults ClearCoatMaterial.java:86-146)."""
    kd: Sequence[float] = (0.5, 0.5, 0.5)
    ks: Sequence[float] = (1.0, 1.0, 1.0)
    ID = MAT_CLEAR_COAT


@dataclass(eq=False)
class Glossy(Material):
    """``scene/material/GlossyMaterial`` (defaults GlossyMaterial.java:81-141)."""
    kr: Sequence[float] = (0.5, 0.5, 0.5)
    roughness: float = 0.2
    ID = MAT_GLOSSY


@dataclass(eq=False)
class Substrate(Material):
    """``scene/material/SubstrateMaterial`` (defaults SubstrateMaterial.java:86-215)."""
    kd: Sequence[float] = (0.5, 0.5, 0.5)
    ks: Sequence[float] = (0.5, 0.5, 0.5)
    roughness_u: float = 0.1
    roughness_v: float = 0.1
    remap_roughness: bool = True
    ID = MAT_SUBSTRATE


@dataclass(eq=False)
class Translucent(Material):
    """``scene/material/TranslucentMaterial`` (defaults TranslucentMaterial.java:94-274)."""
    kd: Sequence[float] = (0.25, 0.25, 0.25)
    ks: Sequence[float] = (0.25, 0.25, 0.25)
    roughness: float = 0.1
    reflectance: Sequence[float] = (0.5, 0.5, 0.5)
    transmittance: Sequence[float] = (0.5, 0.5, 0.5)
    remap_roughness: bool = True
    ID = MAT_TRANSLUCENT


@dataclass(eq=False)
class Uber(Material):
    """``scene/material/UberMaterial`` (defaults UberMaterial.java:97-332)."""
    kd: Sequence[float] = (0.25, 0.25, 0.25)
    kr: Sequence[float] = (0.0, 0.0, 0.0)
    ks: Sequence[float] = (0.25, 0.25, 0.25)
    kt: Sequence[float] = (0.0, 0.0, 0.0)
    opacity: Sequence[float] = (1.0, 1.0, 1.0)
    eta: float = 1.5
    roughness_u: float = 0.1
    roughness_v: float = 0.1
    remap_roughness: bool = True
    ID = MAT_UBER


@dataclass(eq=False)
class BullseyeMaterial(Material):
    """``scene/material/BullseyeMaterial``: material ``a`` where the object-space
    distance to ``origin`` times ``scale`` has a fractional part above 0.5."""
    a: Optional[Material] = None
    b: Optional[Material] = None
    origin: Sequence[float] = (0.0, 10.0, 0.0)
    scale: float = 1.0
    ID = MAT_BULLSEYE


@dataclass(eq=False)
class CheckerboardMaterial(Material):
    """``scene/material/CheckerboardMaterial`` over the texture coordinates."""
    a: Optional[Material] = None
    b: Optional[Material] = None
    angle_deg: float = 0.0
    scale: Sequence[float] = (1.0, 1.0)
    ID = MAT_CHECKERBOARD


@dataclass(eq=False)
class PolkaDotMaterial(Material):
    """``scene/material/PolkaDotMaterial`` over the texture coordinates."""
    a: Optional[Material] = None
    b: Optional[Material] = None
    angle_deg: float = 0.0
    cell_resolution: float = 10.0
    radius: float = 0.25
    ID = MAT_POLKA_DOT


# ---------------------------------------------------------------- lights ----
class Light:
    ID = 0


class DiffuseAreaLight(Light):
    """``scene/light/DiffuseAreaLight``: emits from a shape attached to a primitive."""
    ID = LIGHT_DIFFUSE_AREA

    def __init__(self, shape: Shape, radiance, transform: Optional[Transform] = None, two_sided: bool = False):
        self.shape = shape
        self.radiance = _v(radiance)
        self.transform = transform or Transform()
        self.two_sided = two_sided


class PointLight(Light):
    ID = LIGHT_POINT

    def __init__(self, position, intensity):
        self.position, self.intensity = _v(position), _v(intensity)


class SpotLight(Light):
    """``scene/light/SpotLight``: cone about +z of its transform."""
    ID = LIGHT_SPOT

    def __init__(self, position, look_at, intensity, cone_angle_deg=30.0, cone_delta_deg=5.0):
        self.position = _v(position)
        self.intensity = _v(intensity)
        w = normalize(_v(look_at) - self.position)
        up = np.array([0, 1, 0], dtype=np.float32) if abs(w[1]) < 0.99 else np.array([1, 0, 0], dtype=np.float32)
        u = normalize(np.cross(up, w))
        v = np.cross(w, u)
        m = np.eye(4)
        m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = u, v, w, self.position
        self.transform = Transform(m)
        self.cos_cone = math.cos(math.radians(cone_angle_deg))
        self.cos_cone_minus_delta = math.cos(math.radians(cone_angle_deg - cone_delta_deg))


class DirectionalLight(Light):
    ID = LIGHT_DIRECTIONAL

    def __init__(self, direction, radiance, radius=10.0):
        self.direction, self.radiance, self.radius = normalize(direction), _v(radiance), float(radius)


class PerezLight(Light):
    """``scene/light/PerezLight``: Preetham sun and sky (precomputed in :mod:`perez`)."""
    ID = LIGHT_PEREZ

    def __init__(self, turbidity=2.0, sun_direction_world=(1.0, 1.0, -1.0)):
        self.turbidity = float(turbidity)
        self.sun_direction_world = normalize(sun_direction_world)


class ImageLight(Light):
    """``scene/light/ImageLight``: an environment image (float RGB, rows from
    theta = 0 at the top), rotated by ``angle_deg`` and scaled by ``scale`` in
    spherical texture space (ImageLight.java:134-146)."""
    ID = LIGHT_IMAGE

    def __init__(self, image, angle_deg=0.0, scale=(1.0, 1.0)):
        img = np.ascontiguousarray(image, dtype=np.float32)
        if img.ndim != 3 or img.shape[2] != 3:
            raise ValueError("image must be (height, width, 3)")
        self.image = img
        self.angle_deg = float(angle_deg)
        self.scale = (float(scale[0]), float(scale[1]))


# ------------------------------------------------------ camera, primitives ----
class Camera:
    """``scene/Camera.java`` reduced to what ``CompiledCameraCache.toCamera`` stores."""

    def __init__(self, eye, look_at, up=(0, 1, 0), fov_x_deg=40.0, resolution=(800, 800), aperture_radius=0.0,
                 focal_distance=40.0, lens_fisheye=False):
        self.eye = _v(eye)
        self.w = normalize(_v(look_at) - self.eye)
        self.u = normalize(np.cross(self.w, _v(up)))
        # u points to the image's right and v up: Camera.createPrimaryRay maps
        # image x to +u and image row 0 (top) to +v through the negated tan(fovY/2).
        self.v = np.cross(self.u, self.w).astype(np.float32)
        self.fov_x_deg = float(fov_x_deg)
        self.resolution = (int(resolution[0]), int(resolution[1]))
        self.aperture_radius = float(aperture_radius)
        self.focal_distance = float(focal_distance)
        self.lens = 0 if lens_fisheye else 1

    def to_array(self, resolution=None) -> np.ndarray:
        rx, ry = resolution or self.resolution
        fx = math.radians(self.fov_x_deg)
        fy = 2.0 * math.atan(math.tan(fx * 0.5) * (ry / rx))  # AngleF.fieldOfViewY
        out = np.zeros(19, dtype=np.float32)
        out[0] = math.tan(+fx * 0.5)
        out[1] = math.tan(-fy * 0.5)
        out[2] = self.lens
        out[3:6], out[6:9], out[9:12] = self.u, self.v, self.w
        out[12:15] = self.eye
        out[15] = self.aperture_radius
        out[16] = self.focal_distance
        out[17], out[18] = rx, ry
        return out


class Primitive:
    """``scene/Primitive.java``: shape + material + transform (+ optional area light)."""

    def __init__(self, shape: Shape, material: Material, transform: Optional[Transform] = None,
                 area_light: Optional[DiffuseAreaLight] = None, instance_id: int = 0):
        self.shape = shape
        self.material = material
        self.transform = transform or Transform()
        self.area_light = area_light
        self.instance_id = instance_id


@dataclass
class Scene:
    camera: Camera
    primitives: List[Primitive] = field(default_factory=list)
    lights: List[Light] = field(default_factory=list)
    name: str = "scene"

    def add(self, p: Primitive) -> Primitive:
        self.primitives.append(p)
        return p
