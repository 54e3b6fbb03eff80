// Device-resident scene layout of libdayflower_cuda (shared by the host-side
// ingest in dfc_ingest.cpp and the kernels).
//
// The compiled arrays of the reference (renderer/gpu/AbstractSceneKernel.java:
// 1777-1852) are decoded once on the host into these records:
//   * DPrim      one 128-byte record per primitive: 3x4 object-to-world and
//                world-to-object rows, shape kind and data index, resolved
//                material index and area-light index;
//   * DMaterial  one record per distinct compiled material with its constant
//                textures already evaluated (only ConstantTexture is supported);
//   * DLight     one record per entry of lightIDAndOffsetArray, in its order;
//   * BVH4Node   128-byte 4-wide nodes, child boxes stored as SoA float4
//                (one 128-byte line per node fetch).  The top level is built
//                over primitive world boxes, every mesh gets its own
//                object-space bottom level;
//   * triangles  float4 x3 per triangle (positions, v0.w = triangle index),
//                reordered by the bottom-level builds, and the compiled
//                24-float rows kept in their original order for shading.
#pragma once

#include <cstdint>

namespace dfc {

// 16-byte vector with the layout of CUDA's float4 (device code reads it as float4).
struct alignas(16) F4 { float x, y, z, w; };

// Reference type ids (each class's public static final int ID).
enum : int {
  kShapeCone = 2, kShapeCylinder = 5, kShapeDisk = 6, kShapeHyperboloid = 7, kShapeParaboloid = 9, kShapePlane = 10,
  kShapePolygon = 11, kShapeRectangle = 13, kShapeCuboid = 14, kShapeSphere = 15, kShapeTorus = 16, kShapeTriangle = 17,
  kShapeMesh = 18
};
enum : int { kLightDiffuseArea = 1, kLightDirectional = 2, kLightImage = 3, kLightPerez = 4, kLightPoint = 5, kLightSpot = 7 };

// Resolved material kinds (one shading routine each).
enum : int {
  kMatNone = 0,        // no BSDF: rays pass through (Scene.java:494-500)
  kMatLambert = 1,     // MatteMaterial, angle 0
  kMatOrenNayar = 2,   // MatteMaterial, angle > 0
  kMatMirror = 3,      // MirrorMaterial
  kMatGlassSpec = 4,   // GlassMaterial, zero roughness (FresnelSpecularBXDF)
  kMatGlassRough = 5,  // GlassMaterial, rough (TorranceSparrow BRDF + BTDF)
  kMatMetal = 6,       // MetalMaterial
  kMatPlastic = 7,     // PlasticMaterial
  kMatDisney = 8,      // DisneyMaterial
  kMatClearCoat = 9,   // ClearCoatMaterial (picks its lobe with a random number per hit)
  kMatGlossy = 10,     // GlossyMaterial
  kMatSubstrate = 11,  // SubstrateMaterial (FresnelBlendBRDF)
  kMatTranslucent = 12,  // TranslucentMaterial
  kMatUber = 13,       // UberMaterial
  kMatTextured = 14,   // a material with a non-constant texture or a modifier: DMaterial.flags indexes DTexMaterial
  kMatComposite = 15,  // Bullseye/Checkerboard/PolkaDotMaterial: DMaterial.flags indexes DComposite
  kMatKinds = 16
};

// Reference texture ids (scene/texture/*Texture.java ID); DTexture.kind.
enum : int {
  kTexBlend = 1, kTexBullseye = 2, kTexCheckerboard = 3, kTexConstant = 4, kTexDotProduct = 5, kTexLDRImage = 7,
  kTexMarble = 8, kTexPolkaDot = 9, kTexSimplexFBM = 10, kTexSurfaceNormal = 11, kTexUV = 12
};
enum : int { kModNoOp = 2, kModNormalMapLDRImage = 3, kModSimplexNoiseNormalMap = 4 };  // DModifier.kind
enum : int { kCompBullseye = 1, kCompCheckerboard = 2, kCompPolkaDot = 15 };           // DComposite.kind
constexpr int kTexPositions = 18;  // texture positions of a material record: slot s texture A at 2s, B at 2s + 1
constexpr int kMaxBlendDepth = 3;  // BlendTexture nesting the device evaluates (checked at ingest)

// One node of a texture tree (CompiledTextureCache.java records, resolved):
//   Constant      p[0..2] colour
//   Blend         a, b children; p[0..2] per-channel t
//   Bullseye      a, b; p[0..2] origin (object space), p[3] scale
//   Checkerboard  a, b; p[0] cos, p[1] sin of the angle, p[2..3] scale
//   PolkaDot      a, b; p[0] cos, p[1] sin, p[2] cell resolution, p[3] dot radius
//   LDRImage      a, b resolution x, y; c first texel (SceneView.texels); p[0] cos, p[1] sin, p[2..3] scale
//   Marble        a octaves; p[0..8] colours A, B, C; p[9] frequency, p[10] scale
//   SimplexFBM    a octaves; p[0..2] colour; p[3] frequency, p[4] gain
//   DotProduct, SurfaceNormal, UV: no parameters
struct alignas(16) DTexture {
  int kind, a, b, c;
  float p[12];
};
static_assert(sizeof(DTexture) == 64, "DTexture layout");

// A material modifier (scene/modifier): NormalMapLDRImage (texel, rx, ry; p cos, sin, scale x, y) or
// SimplexNoiseNormalMap (p[0] frequency, p[1] scale).
struct alignas(16) DModifier {
  int kind, texel, rx, ry;
  float p[4];
};
static_assert(sizeof(DModifier) == 32, "DModifier layout");

// A composite material: a, b are DMaterial indices; Bullseye p[0..2] origin (object space), p[3] scale;
// Checkerboard p[0] cos, p[1] sin, p[2..3] scale; PolkaDot p[0] cos, p[1] sin, p[2] cell resolution, p[3] radius.
struct alignas(16) DComposite {
  int kind, a, b, pad;
  float p[4];
};
static_assert(sizeof(DComposite) == 32, "DComposite layout");

// A material evaluated per hit: the reference material id, its modifier
// (DModifier index, -1 for none), the plain int of its record (roughness
// remapping, DisneyMaterial isThin) and one DTexture per texture position
// (-1 where the record has none).
struct alignas(16) DTexMaterial {
  int ref_id, modifier, plain, pad;
  int tex[kTexPositions];
  int pad2[2];
};
static_assert(sizeof(DTexMaterial) == 96, "DTexMaterial layout");

// DisneyMaterial flags (DMaterial.flags); TranslucentMaterial and UberMaterial
// use DMaterial.flags as a bit set of the lobes they build (dfc_ingest.cpp).
enum : int { kDisneyThin = 1, kDisneyScatter = 2, kDisneyHasSheen = 4, kDisneyHasClearCoat = 8, kDisneyHasTransmission = 16 };

struct alignas(16) DPrim {
  float o2w[12];
  float w2o[12];
  int shape;       // reference shape id
  int data;        // triangle index / rectangle index / bottom-level root node
  int material;    // DMaterial index
  int light;       // DLight index of its DiffuseAreaLight, -1 if none
  int identity;    // 1 if both matrices are the identity
  int tri_first;   // mesh: first triangle (in the reordered intersection array)
  int tri_count;   // mesh: triangle count
  int pad;
};
static_assert(sizeof(DPrim) == 128, "DPrim is one 128-byte line");

// One compiled material with its constant textures evaluated.  DisneyMaterial
// keeps the per-material quantities of DisneyMaterial.computeScatteringFunctions
// (scene/material/DisneyMaterial.java:1121-1210), computed once at ingest.
struct alignas(16) DMaterial {
  int kind;
  int has_kr, has_kt;
  int flags;       // Disney: kDisney* bits
  float emission[3];
  float eta;
  float c0[3];     // kd (matte/plastic), kr (mirror/glass), unused (metal), Disney colour
  float ax;
  float c1[3];     // ks (plastic), kt (glass), metal eta, Disney specular R0 (DisneyFresnel)
  float ay;
  float c2[3];     // metal k; Disney (flatness, diffuse transmission / 2, specular transmission)
  float on_a;      // Oren-Nayar A; Disney thin transmission alpha x
  float on_b;      // Oren-Nayar B; Disney thin transmission alpha y
  float d_rough, d_met, d_dw;  // Disney roughness, metallic, diffuse weight (1 - metallic)(1 - specular transmission)
  float c3[3];     // Disney sheen lobe scale
  float d_cc;      // Disney clear coat weight
  float c4[3];     // Disney transmission scale sqrt(colour) * specular transmission
  float d_gloss;   // Disney clear coat alpha lerp(0.1, 0.001, gloss)
};
static_assert(sizeof(DMaterial) == 128, "DMaterial layout");

struct alignas(16) DLight {
  int type;
  int shape;       // DiffuseAreaLight: shape id
  int shape_data;  // DiffuseAreaLight: triangle index (triangle shapes)
  int two_sided;
  float radiance[3];  // area radiance / point & spot intensity / directional radiance / Perez sun colour
  float area;
  float pos[3];       // point/spot position
  float radius;       // directional and Perez radius
  float dir[3];       // directional direction
  float cos_cone;
  float o2w[12];
  float w2o[12];
  float cos_cone_delta;
  int perez;          // PerezLight / ImageLight: float offset of its record in the sky pool (SceneView.perez)
  float pad[2];
};

struct alignas(16) BVH4Node {
  float lox[4], loy[4], loz[4];
  float hix[4], hiy[4], hiz[4];
  // As built: child >= 0 an internal node, < 0 a leaf whose first item is
  // ~child, with count[] items (0 for internal or empty slots).  In device
  // memory, once uploaded (encode_node_entries), child[] holds the traversal's
  // stack entries instead: an internal node's index, or
  // 0x80000000 | first << 2 | (count - 1) for a leaf.
  int child[4];
  int count[4];
};
static_assert(sizeof(BVH4Node) == 128, "BVH4Node is one 128-byte line");

// Everything a kernel needs to read the scene (passed by value).
struct SceneView {
  const DPrim* prims;
  int prim_count;
  const DMaterial* materials;
  const DLight* lights;
  int light_count;
  const BVH4Node* nodes;        // top level and all bottom levels
  int tlas_root;                // -1 if no bounded primitive
  const int* tlas_items;        // primitive index per top-level leaf item
  const F4* tlas_bound;         // per leaf item: world bounding sphere (centre, radius); radius < 0 for meshes
  const int* unbounded;         // primitives with an infinite bounding volume (planes)
  int unbounded_count;
  const F4* tri_pos;            // 3 per triangle, reordered; v0.w holds the triangle index
  const float* tri_attr;        // shape3FTriangle3FArray, 24 floats per triangle, original order
  const float* rects;           // shape3FRectangle3FArray
  const float* shapes;          // disk, cylinder, cone, paraboloid, hyperboloid, cuboid and torus records
  const float* perez;           // sky pool: lightPerezLightArray, then lightImageLightArray
  const float* camera;          // 19 floats
  const DTexture* textures;     // texture nodes of the per-hit materials
  const unsigned* texels;       // packed ARGB pixels of LDRImageTexture and NormalMapLDRImageModifier images
  const DModifier* modifiers;
  const DComposite* composites;
  const DTexMaterial* texmats;
};

}  // namespace dfc
