"""Scene compiler: flattens a :class:`~dayflower_b200.scene.model.Scene` into the
named arrays that ``renderer/gpu/AbstractSceneKernel.java:1777-1852``
(``doSetupScene``) uploads, i.e. the ``CompiledScene`` caches of
``scene/compiler/SceneCompiler.java:81``.

Two layouts are produced:

* ``layout_version = 1`` is the reference packing.  Texture and modifier
  references are packed four to an int with ``utility/Ints.java:258``
  (8-bit ids and 8-bit relative offsets), light references 16/16 with
  ``Ints.java:237``.  Compiling a scene that needs more than 256 textures
  raises ``ValueError``, as ``Ints.pack`` throws ``IllegalArgumentException``.
* ``layout_version = 2`` widens the material records: each 32-bit slot of a v1
  material becomes four int32 lanes (the four packed bytes, or the plain value
  followed by three zeros), and material offsets count lanes.  Everything else
  is identical.  Large scenes (thousands of distinct textures) need it.

Offsets follow the reference: shape and material offsets are absolute array
indices, bounding-volume, texture and light offsets are relative structure
indices (the device multiplies them by the structure length).
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, List

import numpy as np

from . import model as M
from .perez import image_light_record, perez_record

ARRAY_NAMES_F32 = [
    "boundingVolume3FAxisAlignedBoundingBox3FArray", "boundingVolume3FBoundingSphere3FArray",
    "shape3FCone3FArray", "shape3FCylinder3FArray", "shape3FDisk3FArray", "shape3FHyperboloid3FArray",
    "shape3FParaboloid3FArray", "shape3FPolygon3FArray", "shape3FRectangle3FArray", "shape3FRectangularCuboid3FArray",
    "shape3FTorus3FArray", "shape3FTriangle3FArray",
    "textureBlendTextureArray", "textureBullseyeTextureArray", "textureCheckerboardTextureArray",
    "textureConstantTextureArray", "textureLDRImageTextureArray", "textureMarbleTextureArray",
    "texturePolkaDotTextureArray", "textureSimplexFractionalBrownianMotionTextureArray",
    "modifierNormalMapLDRImageModifierArray", "modifierSimplexNoiseNormalMapModifierArray",
    "materialBullseyeMaterialArray", "materialCheckerboardMaterialArray", "materialPolkaDotMaterialArray",
    "lightDiffuseAreaLightArray", "lightDirectionalLightArray", "lightImageLightArray", "lightPerezLightArray",
    "lightPointLightArray", "lightSpotLightArray", "cameraArray", "primitiveMatrix44FArray",
]
ARRAY_NAMES_I32 = [
    "shape3FTriangleMesh3FArray", "textureLDRImageTextureOffsetArray",
    "materialClearCoatMaterialArray",
    "materialDisneyMaterialArray", "materialGlassMaterialArray", "materialGlossyMaterialArray",
    "materialMatteMaterialArray", "materialMetalMaterialArray", "materialMirrorMaterialArray",
    "materialPlasticMaterialArray", "materialSubstrateMaterialArray",
    "materialTranslucentMaterialArray", "materialUberMaterialArray",
    "modifierNormalMapLDRImageModifierOffsetArray", "lightIDAndOffsetArray", "lightImageLightOffsetArray",
    "lightPerezLightOffsetArray", "primitiveArray",
]


class CompiledScene:
    """The compiled arrays plus bookkeeping (``scene/compiler/CompiledScene.java``)."""

    def __init__(self, arrays: Dict[str, np.ndarray], layout_version: int, stats: Dict[str, int]):
        self.arrays = arrays
        self.layout_version = layout_version
        self.stats = stats
        self.version = 0       # bumped by every change a CompiledSceneModifier makes
        self.compiler = None   # the SceneCompiler that made it (None for arrays from elsewhere)

    def nbytes(self) -> int:
        return int(sum(a.nbytes for a in self.arrays.values()))


def _scene_lib():
    from .._native import load_scene_compiler
    return load_scene_compiler()


def build_mesh_bvh_stream(tris: np.ndarray, tri_offset_base: int, aabb_base: int):
    """Returns (int32 stream, float32 aabbs) for one mesh (host helper in csrc/scene_compiler.cpp)."""
    lib = _scene_lib()
    n = tris.shape[0]
    cap = 2 * n + 1
    stream = np.zeros(cap * 8, dtype=np.int32)
    boxes = np.zeros(cap * 8, dtype=np.float32)
    t = np.ascontiguousarray(tris, dtype=np.float32)
    nodes = lib.dfc_sc_build_mesh_bvh(t.ctypes.data_as(ctypes.c_void_p), ctypes.c_longlong(n), ctypes.c_longlong(tri_offset_base),
                                      ctypes.c_longlong(aabb_base), stream.ctypes.data_as(ctypes.c_void_p),
                                      boxes.ctypes.data_as(ctypes.c_void_p), ctypes.c_longlong(cap))
    if nodes <= 0:
        raise RuntimeError("mesh BVH build failed")
    return stream[: nodes * 8].copy(), boxes[: nodes * 8].copy()


def _pack8(a, b, c, d) -> int:
    """``utility/Ints.java:258``."""
    for v in (a, b, c, d):
        if not 0 <= v <= 255:
            raise ValueError("texture/modifier reference out of range for layout 1: %d (use layout_version=2)" % v)
    x = (a & 0xFF) | ((b & 0xFF) << 8) | ((c & 0xFF) << 16) | ((d & 0xFF) << 24)
    return int(np.int32(np.uint32(x)))


def _pack16(a, b) -> int:
    """``utility/Ints.java:237``."""
    if not (0 <= a <= 65535 and 0 <= b <= 65535):
        raise ValueError("reference out of range for a 16/16 pack: %d %d" % (a, b))
    return int(np.int32(np.uint32(((a & 0xFFFF) << 16) | (b & 0xFFFF))))


def _world_aabb(points_obj: np.ndarray, o2w: np.ndarray):
    p = np.asarray(points_obj, dtype=np.float64).reshape(-1, 3)
    lo, hi = p.min(axis=0), p.max(axis=0)
    corners = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
    m = o2w.astype(np.float64)
    w = corners @ m[:3, :3].T + m[:3, 3]
    return w.min(axis=0), w.max(axis=0)


def _packf(a, b) -> float:
    """A 16/16 packed reference stored in a float array (exact below 2^24)."""
    return float(_pack16(a, b))


def _argb(color) -> float:
    """``Color3F.pack()`` (ARGB, alpha 255) stored in a float array.  The 8-bit
    rounding (saturate, * 255, + 0.5, truncate) stands in for
    ``org.macroing.java.lang.Ints.saturateAndScaleToInt``, whose source is not
    part of the reference; every reader unpacks the stored value."""
    c = [int(min(max(float(x), 0.0), 1.0) * 255.0 + 0.5) for x in np.broadcast_to(np.asarray(color, dtype=np.float64), (3,))]
    return float(np.int32(np.uint32((255 << 24) | (c[0] << 16) | (c[1] << 8) | c[2])))


def _rad(degrees) -> float:
    return float(np.float32(float(np.float32(degrees)) * (math.pi / 180.0)))


def _image_record(t) -> list:
    """``CompiledTextureCache.toLDRImageTexture`` / ``CompiledModifierCache.toNormalMapLDRImageModifier``:
    angle (radians), scale (2), resolution x, y, the packed ARGB pixels, zero padding to 8."""
    img = np.asarray(t.image, dtype=np.uint32).reshape(-1)
    if img.size != t.resolution_x * t.resolution_y:
        raise ValueError("image size does not match its resolution")
    px = img.view(np.int32).astype(np.float64)
    head = [_rad(t.angle_deg), t.scale[0], t.scale[1], t.resolution_x, t.resolution_y]
    n = 5 + img.size
    return head + px.tolist() + [0.0] * ((8 - n % 8) % 8)


# Shapes stored as one fixed-length record each (CompiledShape3FCache.java:90-310).
_RECORD_SHAPES = {M.Disk: "shape3FDisk3FArray", M.Cylinder: "shape3FCylinder3FArray", M.Cone: "shape3FCone3FArray",
                  M.Paraboloid: "shape3FParaboloid3FArray", M.Hyperboloid: "shape3FHyperboloid3FArray",
                  M.RectangularCuboid: "shape3FRectangularCuboid3FArray", M.Torus: "shape3FTorus3FArray",
                  M.Polygon: "shape3FPolygon3FArray"}


class SceneCompiler:
    """Appends scene objects to the compiled arrays: the state of one compile, kept so that
    primitives can be added and removed afterwards (:class:`CompiledSceneModifier`)."""

    def __init__(self, layout_version: int = 1):
        if layout_version not in (1, 2):
            raise ValueError("layout_version must be 1 or 2")
        lanes = 4 if layout_version == 2 else 1
        f32: Dict[str, List[np.ndarray]] = {k: [] for k in ARRAY_NAMES_F32}
        i32: Dict[str, List[np.ndarray]] = {k: [] for k in ARRAY_NAMES_I32}
        sizes = {k: 0 for k in ARRAY_NAMES_F32 + ARRAY_NAMES_I32}

        def push(name, arr):
            bucket = f32 if name in f32 else i32
            a = np.asarray(arr, dtype=np.float32 if name in f32 else np.int32).reshape(-1)
            off = sizes[name]
            bucket[name].append(a)
            sizes[name] += a.size
            return off

        # ---- textures (CompiledTextureCache.java:1530-2144): records of the pattern
        # textures hold their children as Ints.pack(id, relative offset) in a float
        tex_index: Dict[tuple, int] = {}
        tex_objects: Dict[int, tuple] = {}

        def tex(color) -> int:
            c = tuple(float(np.float32(x)) for x in (np.broadcast_to(np.asarray(color, dtype=np.float32), (3,))))
            if c not in tex_index:
                tex_index[c] = sizes["textureConstantTextureArray"] // 4
                push("textureConstantTextureArray", [c[0], c[1], c[2], 0.0])
            return tex_index[c]

        def texture(t) -> tuple:
            """(texture id, relative offset) of a texture, a colour or a number."""
            if not isinstance(t, M.Texture):
                return (M.TEX_CONSTANT, tex(t))
            key = id(t)
            if key in tex_objects:
                return tex_objects[key]
            if isinstance(t, M.ConstantTexture):
                ref = (M.TEX_CONSTANT, tex(t.color))
            elif isinstance(t, (M.DotProductTexture, M.SurfaceNormalTexture, M.UVTexture)):
                ref = (t.ID, 0)
            elif isinstance(t, M.BlendTexture):
                a, b = _packf(*texture(t.a)), _packf(*texture(t.b))
                tt = np.broadcast_to(np.asarray(t.t, dtype=np.float32), (3,))
                ref = (t.ID, push("textureBlendTextureArray", [a, b, tt[0], tt[1], tt[2], 0, 0, 0]) // 8)
            elif isinstance(t, M.BullseyeTexture):
                a, b = _packf(*texture(t.a)), _packf(*texture(t.b))
                o = t.origin
                ref = (t.ID, push("textureBullseyeTextureArray", [o[0], o[1], o[2], a, b, t.scale, 0, 0]) // 8)
            elif isinstance(t, M.CheckerboardTexture):
                a, b = _packf(*texture(t.a)), _packf(*texture(t.b))
                rec = [t.angle_deg, _rad(t.angle_deg), a, b, t.scale[0], t.scale[1], 0, 0]
                ref = (t.ID, push("textureCheckerboardTextureArray", rec) // 8)
            elif isinstance(t, M.PolkaDotTexture):
                a, b = _packf(*texture(t.a)), _packf(*texture(t.b))
                rec = [t.angle_deg, _rad(t.angle_deg), a, b, t.cell_resolution, t.radius, 0, 0]
                ref = (t.ID, push("texturePolkaDotTextureArray", rec) // 8)
            elif isinstance(t, M.MarbleTexture):
                rec = [_argb(t.color_a), _argb(t.color_b), _argb(t.color_c), t.frequency, t.scale, t.stripes, t.octaves, 0]
                ref = (t.ID, push("textureMarbleTextureArray", rec) // 8)
            elif isinstance(t, M.SimplexFBMTexture):
                rec = [_argb(t.color), t.frequency, t.gain, t.octaves]
                ref = (t.ID, push("textureSimplexFractionalBrownianMotionTextureArray", rec) // 4)
            elif isinstance(t, M.LDRImageTexture):
                off = push("textureLDRImageTextureArray", _image_record(t))
                ref = (t.ID, sizes["textureLDRImageTextureOffsetArray"])
                push("textureLDRImageTextureOffsetArray", [off])
            else:
                raise ValueError("unsupported texture %r" % type(t).__name__)
            tex_objects[key] = ref
            return ref

        mod_objects: Dict[int, tuple] = {}

        def modifier(m) -> tuple:
            """(modifier id, relative offset) (CompiledModifierCache.java:445-530)."""
            if m is None or isinstance(m, M.NoOpModifier):
                return (M.MOD_NOOP, 0)
            key = id(m)
            if key not in mod_objects:
                if isinstance(m, M.NormalMapLDRImageModifier):
                    off = push("modifierNormalMapLDRImageModifierArray", _image_record(m))
                    mod_objects[key] = (m.ID, sizes["modifierNormalMapLDRImageModifierOffsetArray"])
                    push("modifierNormalMapLDRImageModifierOffsetArray", [off])
                elif isinstance(m, M.SimplexNoiseNormalMapModifier):
                    mod_objects[key] = (m.ID, push("modifierSimplexNoiseNormalMapModifierArray", [m.frequency, m.scale]) // 2)
                else:
                    raise ValueError("unsupported modifier %r" % type(m).__name__)
            return mod_objects[key]

        def slot(a=(0, 0), b=(0, 0)):
            if layout_version == 2:
                return [a[0], a[1], b[0], b[1]]
            return [_pack8(a[0], a[1], b[0], b[1])]

        def plain(v):
            return [int(v), 0, 0, 0] if layout_version == 2 else [int(v)]

        def pad_to(rec, length):
            return rec + [0] * (length * lanes - len(rec))

        def ft(v):
            """A float parameter: a texture, or a number as a grey constant texture."""
            return texture(v if isinstance(v, M.Texture) else [v] * 3)

        T = texture
        mat_offsets: Dict[int, tuple] = {}
        composite_arrays = {M.BullseyeMaterial: "materialBullseyeMaterialArray",
                            M.CheckerboardMaterial: "materialCheckerboardMaterialArray",
                            M.PolkaDotMaterial: "materialPolkaDotMaterialArray"}

        def material(m: M.Material):
            key = id(m)
            if key in mat_offsets:
                return mat_offsets[key]
            if type(m) in composite_arrays:  # CompiledMaterialCache.java toBullseyeMaterial etc.: absolute offsets
                if m.a is None or m.b is None:
                    raise ValueError("%s needs two materials" % type(m).__name__)
                a, b = _packf(*material(m.a)), _packf(*material(m.b))
                if isinstance(m, M.BullseyeMaterial):
                    o = m.origin
                    rec = [o[0], o[1], o[2], a, b, m.scale, 0, 0]
                elif isinstance(m, M.CheckerboardMaterial):
                    rec = [m.angle_deg, _rad(m.angle_deg), a, b, m.scale[0], m.scale[1], 0, 0]
                else:
                    rec = [m.angle_deg, _rad(m.angle_deg), a, b, m.cell_resolution, m.radius, 0, 0]
                mat_offsets[key] = (m.ID, push(composite_arrays[type(m)], rec))
                return mat_offsets[key]
            head = slot(T(m.emission), modifier(m.modifier))
            if isinstance(m, M.Matte):
                rec, name, length = head + slot(ft(m.angle), T(m.kd)), "materialMatteMaterialArray", 2
            elif isinstance(m, M.Mirror):
                rec, name, length = head + slot(T(m.kr)), "materialMirrorMaterialArray", 2
            elif isinstance(m, M.Glass):
                rec = head + slot(ft(m.eta)) + slot(T(m.kr), T(m.kt)) + \
                    slot(ft(m.roughness_u), ft(m.roughness_v)) + plain(m.remap_roughness)
                name, length = "materialGlassMaterialArray", 8
            elif isinstance(m, M.Metal):
                rec = head + slot(T(m.eta), T(m.k)) + slot(ft(m.roughness_u), ft(m.roughness_v)) + plain(m.remap_roughness)
                name, length = "materialMetalMaterialArray", 4
            elif isinstance(m, M.Plastic):
                rec = head + slot(T(m.kd), T(m.ks)) + slot(ft(m.roughness)) + plain(m.remap_roughness)
                name, length = "materialPlasticMaterialArray", 4
            elif isinstance(m, M.ClearCoat):  # CompiledMaterialCache.java:2639-2646
                rec, name, length = head + slot(T(m.kd), T(m.ks)), "materialClearCoatMaterialArray", 2
            elif isinstance(m, M.Glossy):  # :2932-2939
                rec, name, length = head + slot(T(m.kr), ft(m.roughness)), "materialGlossyMaterialArray", 2
            elif isinstance(m, M.Substrate):  # :3373-3383
                rec = head + slot(T(m.kd), T(m.ks)) + slot(ft(m.roughness_u), ft(m.roughness_v)) + plain(m.remap_roughness)
                name, length = "materialSubstrateMaterialArray", 4
            elif isinstance(m, M.Translucent):  # :3466-3477
                rec = head + slot(T(m.kd), T(m.ks)) + slot(T(m.reflectance), T(m.transmittance)) + \
                    slot(ft(m.roughness), (1 if m.remap_roughness else 0, 0))
                name, length = "materialTranslucentMaterialArray", 4
            elif isinstance(m, M.Uber):  # :3563-3577
                rec = head + slot(T(m.kd), T(m.kr)) + slot(T(m.ks), T(m.kt)) + slot(ft(m.eta), T(m.opacity)) + \
                    slot(ft(m.roughness_u), ft(m.roughness_v)) + plain(m.remap_roughness)
                name, length = "materialUberMaterialArray", 8
            elif isinstance(m, M.Disney):
                # CompiledMaterialCache.toDisneyMaterial (:2717-2760): nine packed slots of a 16-slot record
                rec = head + slot(ft(m.anisotropic)) + slot(ft(m.clear_coat), ft(m.clear_coat_gloss)) + \
                    slot(T(m.color), ft(m.diffuse_transmission)) + slot(ft(m.eta), ft(m.flatness)) + \
                    slot(ft(m.metallic), ft(m.roughness)) + slot(T(m.scatter_distance), ft(m.sheen)) + \
                    slot(ft(m.sheen_tint), ft(m.specular_tint)) + slot(ft(m.specular_transmission), (1 if m.thin else 0, 0))
                name, length = "materialDisneyMaterialArray", 16
            else:
                raise ValueError("unsupported material %r" % type(m).__name__)
            off = push(name, pad_to(rec, length))
            mat_offsets[key] = (m.ID, off)
            return mat_offsets[key]

        # ---- shapes
        shape_offsets: Dict[int, tuple] = {}
        mesh_jobs = []

        def shape(s: M.Shape):
            key = id(s)
            if key in shape_offsets:
                return shape_offsets[key]
            if isinstance(s, M.Triangle):
                off = push("shape3FTriangle3FArray", s.to_array())
            elif isinstance(s, M.Rectangle):
                off = push("shape3FRectangle3FArray", s.to_array())
            elif isinstance(s, (M.Sphere, M.Plane)):
                off = 0
            elif isinstance(s, tuple(_RECORD_SHAPES)):
                off = push(_RECORD_SHAPES[type(s)], s.to_array())
            elif isinstance(s, M.TriangleMesh):
                tri_base = push("shape3FTriangle3FArray", s.triangles)
                aabb_base = sizes["boundingVolume3FAxisAlignedBoundingBox3FArray"] // 8
                stream, boxes = build_mesh_bvh_stream(s.triangles, tri_base, aabb_base)
                push("boundingVolume3FAxisAlignedBoundingBox3FArray", boxes)
                off = push("shape3FTriangleMesh3FArray", stream)
                mesh_jobs.append(off)
            else:
                raise ValueError("unsupported shape %r" % type(s).__name__)
            shape_offsets[key] = (s.ID, off)
            return shape_offsets[key]


        # ---- lights: the record, and its (id, relative offset) in lightIDAndOffsetArray
        light_refs: Dict[int, tuple] = {}
        rel_count = {M.LIGHT_DIFFUSE_AREA: 0, M.LIGHT_DIRECTIONAL: 0, M.LIGHT_POINT: 0, M.LIGHT_SPOT: 0, M.LIGHT_PEREZ: 0, M.LIGHT_IMAGE: 0}

        def add_light(L) -> tuple:
            if id(L) in light_refs:
                return light_refs[id(L)]
            if isinstance(L, M.DiffuseAreaLight):
                sid, soff = shape(L.shape)
                if isinstance(L.shape, M.Triangle):
                    area = 0.5 * float(np.linalg.norm(np.cross(L.shape.b - L.shape.a, L.shape.c - L.shape.a)))
                elif isinstance(L.shape, M.Sphere):
                    area = 4.0 * np.pi
                else:
                    area = 0.0
                rec = np.zeros(40, dtype=np.float32)
                rec[0:16] = L.transform.object_to_world.reshape(-1)
                rec[16:32] = L.transform.world_to_object.reshape(-1)
                rec[32:35] = L.radiance
                rec[35], rec[36], rec[37], rec[38] = sid, soff, area, 1.0 if L.two_sided else 0.0
                push("lightDiffuseAreaLightArray", rec)
            elif isinstance(L, M.PointLight):
                push("lightPointLightArray", np.concatenate([L.intensity, L.position, [0, 0]]))
            elif isinstance(L, M.SpotLight):
                rec = np.zeros(24, dtype=np.float32)
                rec[0:16] = L.transform.world_to_object.reshape(-1)
                rec[16:19] = L.intensity
                rec[19:22] = L.position
                rec[22], rec[23] = L.cos_cone, L.cos_cone_minus_delta
                push("lightSpotLightArray", rec)
            elif isinstance(L, M.DirectionalLight):
                push("lightDirectionalLightArray", np.concatenate([L.radiance, L.direction, [L.radius, 0.0]]))
            elif isinstance(L, M.PerezLight):
                off = push("lightPerezLightArray", perez_record(L.turbidity, L.sun_direction_world))
                push("lightPerezLightOffsetArray", [off])
            elif isinstance(L, M.ImageLight):
                off = push("lightImageLightArray", image_light_record(L.image, L.angle_deg, L.scale))
                push("lightImageLightOffsetArray", [off])
            else:
                raise ValueError("unsupported light %r" % type(L).__name__)
            rel = rel_count[L.ID]
            rel_count[L.ID] += 1
            light_refs[id(L)] = (L.ID, rel)
            push("lightIDAndOffsetArray", [_pack16(L.ID, rel)])
            return light_refs[id(L)]

        # ---- primitives: one 8-int record (CompiledPrimitiveCache.java:53-93) and two matrices each
        mesh_bounds: Dict[int, np.ndarray] = {}
        aabb_index: Dict[tuple, int] = {}

        def aabb(lo, hi) -> int:  # CompiledBoundingVolume3FCache.addAxisAlignedBoundingBox3F: equal boxes shared
            rec = tuple(float(np.float32(v)) for v in (hi[0], hi[1], hi[2], lo[0], lo[1], lo[2]))
            if rec not in aabb_index:
                aabb_index[rec] = sizes["boundingVolume3FAxisAlignedBoundingBox3FArray"] // 8
                push("boundingVolume3FAxisAlignedBoundingBox3FArray", list(rec) + [0, 0])
            return aabb_index[rec]

        def primitive_record(p) -> list:
            sid, soff = shape(p.shape)
            mid, moff = material(p.material)
            o2w = p.transform.object_to_world
            if isinstance(p.shape, M.Plane):
                bvid, bvoff = M.BV_INFINITE, 0
            else:
                if isinstance(p.shape, M.Sphere):
                    pts = np.array([[-1, -1, -1], [1, 1, 1]], dtype=np.float32)
                elif isinstance(p.shape, M.Triangle):
                    pts = np.stack([p.shape.a, p.shape.b, p.shape.c])
                elif isinstance(p.shape, M.Rectangle) or isinstance(p.shape, tuple(_RECORD_SHAPES)):
                    pts = p.shape.corners()
                else:
                    key = id(p.shape)
                    if key not in mesh_bounds:  # the mesh's object-space box, shared by its instances
                        q = p.shape.triangles[:, 0:9].reshape(-1, 3)
                        mesh_bounds[key] = np.stack([q.min(axis=0), q.max(axis=0)])
                    pts = mesh_bounds[key]
                lo, hi = _world_aabb(pts, o2w)
                bvid, bvoff = M.BV_AABB, aabb(lo, hi)
            al = 0
            if p.area_light is not None:
                lid, lrel = add_light(p.area_light)
                al = _pack16(lid, lrel)
            return [p.instance_id, al, bvid, bvoff, mid, moff, sid, soff]

        def add_primitive(p):
            push("primitiveArray", primitive_record(p))
            push("primitiveMatrix44FArray", p.transform.to_array())

        def remove_primitive(p) -> bool:
            """CompiledPrimitiveCache.removePrimitive: the first record equal to p's, and its matrices."""
            rec = np.asarray(primitive_record(p), dtype=np.int32)
            prim = self._flat("primitiveArray").reshape(-1, 8)
            hit = np.nonzero(np.all(prim == rec, axis=1))[0]
            if hit.size == 0:
                return False
            k = int(hit[0])
            mats = self._flat("primitiveMatrix44FArray").reshape(-1, 32)
            self._set("primitiveArray", np.delete(prim, k, axis=0).reshape(-1))
            self._set("primitiveMatrix44FArray", np.delete(mats, k, axis=0).reshape(-1))
            return True

        self.layout_version = layout_version
        self._f32, self._i32, self._sizes, self._push = f32, i32, sizes, push
        self.add_light, self.add_primitive, self.remove_primitive = add_light, add_primitive, remove_primitive
        self.camera = None
        self._tex_index, self._tex_objects, self._mesh_jobs = tex_index, tex_objects, mesh_jobs

    def _flat(self, name) -> np.ndarray:
        bucket = self._f32 if name in self._f32 else self._i32
        parts = bucket[name]
        dt = np.float32 if bucket is self._f32 else np.int32
        return np.concatenate(parts).astype(dt) if parts else np.zeros(0, dtype=dt)

    def _set(self, name, arr):
        bucket = self._f32 if name in self._f32 else self._i32
        bucket[name] = [np.asarray(arr)]
        self._sizes[name] = int(np.asarray(arr).size)

    def set_camera(self, camera, resolution=None):
        self.camera = np.asarray(camera.to_array(resolution), dtype=np.float32)

    def arrays(self) -> Dict[str, np.ndarray]:
        out = {k: self._flat(k) for k in list(self._f32) + list(self._i32)}
        out["cameraArray"] = self.camera.copy() if self.camera is not None else np.zeros(19, dtype=np.float32)
        return out

    def compiled_scene(self, n_lights: int = 0) -> CompiledScene:
        a = self.arrays()
        stats = {"primitives": int(a["primitiveArray"].size // 8), "lights": int(a["lightIDAndOffsetArray"].size),
                 "triangles": int(a["shape3FTriangle3FArray"].size // 24), "textures": len(self._tex_index) + len(self._tex_objects),
                 "meshes": len(self._mesh_jobs)}
        cs = CompiledScene(a, self.layout_version, stats)
        cs.compiler = self
        return cs


def compile_scene(scene: M.Scene, layout_version: int = 1, resolution=None) -> CompiledScene:
    c = SceneCompiler(layout_version)
    for L in scene.lights:
        c.add_light(L)
    for p in scene.primitives:
        c.add_primitive(p)
    c.set_camera(scene.camera, resolution)
    return c.compiled_scene()


class CompiledSceneModifier:
    """``scene/compiler/CompiledSceneModifier.java``: adds primitives to and
    removes them from an already compiled scene.  A renderer holding the
    scene sees the new version at its next ``render`` and uploads it
    (``AbstractGPURenderer.render`` -> ``updateCompiledScene``, which also
    clears the film).

    ``add_primitive`` appends the primitive's shape, material, bounding volume
    and area light (each shared with an equal one already compiled) and its
    record; like ``CompiledPrimitiveCache.addPrimitive`` it returns False when
    an equal record exists.  ``remove_primitive`` removes the first equal
    record and its matrices; the shape and material records stay.  Lights are
    not added or removed (the reference's ``addLight`` and ``removeLight``
    return false)."""

    def __init__(self, compiled: CompiledScene):
        if compiled.compiler is None:
            raise ValueError("the compiled scene was not made by compile_scene")
        self.compiled = compiled

    def _changed(self):
        c = self.compiled
        c.arrays = c.compiler.arrays()
        c.stats["primitives"] = int(c.arrays["primitiveArray"].size // 8)
        c.stats["triangles"] = int(c.arrays["shape3FTriangle3FArray"].size // 24)
        c.version += 1

    def add_primitive(self, primitive: M.Primitive) -> bool:
        comp = self.compiled.compiler
        before = comp._flat("primitiveArray").reshape(-1, 8)
        comp.add_primitive(primitive)
        after = comp._flat("primitiveArray").reshape(-1, 8)
        rec = after[-1]
        if before.shape[0] and np.any(np.all(before == rec, axis=1)):
            comp._set("primitiveArray", before.reshape(-1))  # an equal record exists: undo
            mats = comp._flat("primitiveMatrix44FArray").reshape(-1, 32)
            comp._set("primitiveMatrix44FArray", mats[:-1].reshape(-1))
            self._changed()
            return False
        self._changed()
        return True

    def remove_primitive(self, primitive: M.Primitive) -> bool:
        ok = self.compiled.compiler.remove_primitive(primitive)
        if ok:
            self._changed()
        return ok

    def add_light(self, light: M.Light) -> bool:
        return False

    def remove_light(self, light: M.Light) -> bool:
        return False
