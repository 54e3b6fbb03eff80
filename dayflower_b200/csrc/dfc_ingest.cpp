// Host-side decoding of the reference's compiled scene arrays into the device
// records of dfc_scene.h, plus the acceleration-structure builds.
//
// Input: the arrays renderer/gpu/AbstractSceneKernel.java:1777-1852 puts, by
// the same names.  Layouts are those of scene/compiler/Compiled*Cache.java:
//   primitiveArray        8 ints per primitive (CompiledPrimitiveCache.java:53-93)
//   primitiveMatrix44FArray 32 floats per primitive (object-to-world, world-to-object)
//   material arrays       packed (texture id, relative offset) bytes, Ints.java:258
//                         (layout 2: one int32 lane per packed byte)
//   lightIDAndOffsetArray (light id << 16) | relative offset, Ints.java:237
//   shape3FTriangleMesh3FArray threaded BVH stream (CompiledShape3FCache.java:2652)
#include "dfc_ingest.h"

#include <algorithm>
#include <chrono>
#include <thread>

#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <sstream>

#include "dfc_blas.h"
#include "dfc_bvh.h"
#include "dfc_matderive.h"

namespace dfc {
namespace {

enum {
  kMatClearCoatId = 3, kMatDisneyId = 4, kMatGlassId = 7, kMatGlossyId = 8, kMatMatteId = 11, kMatMetalId = 12, kMatMirrorId = 13,
  kMatPlasticId = 14, kMatSubstrateId = 16, kMatTranslucentId = 18, kMatUberId = 19
};
enum { kTexConstantId = 4 };
enum { kBVAabbId = 1, kBVSphereId = 2, kBVInfiniteId = 3 };

// Runs f(begin, end) over [0, n) in contiguous chunks on the host's threads.
template <typename F>
void parallel_for(size_t n, F&& f) {
  const unsigned hw = std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
  const size_t parts = n < (1u << 16) ? 1 : hw;
  if (parts == 1) { f((size_t)0, n); return; }
  std::vector<std::thread> ws;
  for (size_t p = 1; p < parts; ++p) ws.emplace_back([&, p] { f(n * p / parts, n * (p + 1) / parts); });
  f((size_t)0, n / parts);
  for (auto& w : ws) w.join();
}

template <typename V, typename T>
void stage_copy_into(V& dst, const T* src, size_t count) {
  dst.resize(count);
  T* out = dst.data();
  parallel_for(count, [&](size_t a, size_t b) { std::memcpy(out + a, src + a, (b - a) * sizeof(T)); });
}

struct Fail {
  int code;
  std::string msg;
};

template <typename V>
const V& get(const std::map<std::string, V>& m, const char* name) {
  static const V empty;
  auto it = m.find(name);
  return it == m.end() ? empty : it->second;
}

struct Decoder {
  const Staged& st;
  int layout;
  HostScene& hs;
  std::map<std::pair<int, int>, int> material_index;
  std::map<int, int> light_by_key;  // (id << 16 | rel) -> index

  bool device_blas = false;

  Decoder(const Staged& s, int l, HostScene& h, bool dev) : st(s), layout(l), hs(h), device_blas(dev) {}

  const StagedF& F(const char* n) { return get(st.f32, n); }
  const StagedI& I(const char* n) { return get(st.i32, n); }

  void texref(const StagedI& arr, int base, int slot, int* ida, int* offa, int* idb, int* offb) {
    if (layout == 2) {
      size_t k = (size_t)base + (size_t)slot * 4;
      if (k + 4 > arr.size()) throw Fail{DFC_E_INVALID_ARG, "material record out of range"};
      *ida = arr[k]; *offa = arr[k + 1]; *idb = arr[k + 2]; *offb = arr[k + 3];
    } else {
      size_t k = (size_t)base + slot;
      if (k >= arr.size()) throw Fail{DFC_E_INVALID_ARG, "material record out of range"};
      uint32_t v = (uint32_t)arr[k];
      *ida = v & 0xFF; *offa = (v >> 8) & 0xFF; *idb = (v >> 16) & 0xFF; *offb = (v >> 24) & 0xFF;
    }
  }
  int plain(const StagedI& arr, int base, int slot) {
    size_t k = (size_t)base + (size_t)slot * (layout == 2 ? 4 : 1);
    if (k >= arr.size()) throw Fail{DFC_E_INVALID_ARG, "material record out of range"};
    return arr[k];
  }
  // renderer/gpu/AbstractTextureKernel.java:152 (ConstantTexture)
  void color(int id, int off, float out[3]) {
    if (id != kTexConstantId) {
      std::ostringstream os;
      os << "texture id " << id << " is not supported (ConstantTexture only)";
      throw Fail{DFC_E_UNSUPPORTED, os.str()};
    }
    const auto& C = F("textureConstantTextureArray");
    size_t k = (size_t)off * 4;
    if (off < 0 || k + 3 > C.size()) throw Fail{DFC_E_INVALID_ARG, "constant texture offset out of range"};
    out[0] = C[k]; out[1] = C[k + 1]; out[2] = C[k + 2];
  }

  // ---- textures (renderer/gpu/AbstractTextureKernel.java:152-435, scene/texture/*.java getColor)
  std::map<std::pair<int, int>, int> texture_index;
  std::vector<int> texture_blend_depth;  // BlendTexture nesting below each node

  static float jcos(float a) { return (float)std::cos((double)a); }  // utility/Floats.java cos, sin: Math in double
  static float jsin(float a) { return (float)std::sin((double)a); }
  static void unpack_argb(float f, float* out) {  // Color3F.unpack(ARGB) of a packed colour stored in a float
    const int c = (int)f;
    out[0] = (float)((c >> 16) & 0xFF) / 255.0f; out[1] = (float)((c >> 8) & 0xFF) / 255.0f; out[2] = (float)(c & 0xFF) / 255.0f;
  }
  const float* record(const char* name, size_t off, size_t len) {
    const auto& A = F(name);
    if (off + len > A.size()) throw Fail{DFC_E_INVALID_ARG, std::string(name) + ": record out of range"};
    return A.data() + off;
  }
  // An LDR image record (angle, scale x, y, resolution x, y, ARGB pixels): its texels go to the pool.
  void image(const char* name, const char* offsets, int rel, int* texel, int* rx, int* ry, float* p4) {
    const auto& O = I(offsets);
    if (rel < 0 || (size_t)rel >= O.size()) throw Fail{DFC_E_INVALID_ARG, std::string(offsets) + ": index out of range"};
    const float* q = record(name, (size_t)O[rel], 5);
    *rx = (int)q[3]; *ry = (int)q[4];
    if (*rx <= 0 || *ry <= 0) throw Fail{DFC_E_INVALID_ARG, "image resolution must be positive"};
    q = record(name, (size_t)O[rel], 5 + (size_t)*rx * (size_t)*ry);
    *texel = (int)hs.texels.size();
    for (size_t k = 0; k < (size_t)*rx * (size_t)*ry; ++k) hs.texels.push_back((unsigned)(int)q[5 + k]);
    p4[0] = jcos(q[0]); p4[1] = jsin(q[0]); p4[2] = q[1]; p4[3] = q[2];
  }
  static void unpack16(float f, int* id, int* off) { const int v = (int)f; *id = (v >> 16) & 0xFFFF; *off = v & 0xFFFF; }

  int texture_node(int id, int off, int depth) {
    const auto key = std::make_pair(id, off);
    auto it = texture_index.find(key);
    if (it != texture_index.end()) return it->second;
    if (depth > 64) throw Fail{DFC_E_UNSUPPORTED, "texture tree deeper than 64 (or cyclic)"};
    DTexture t{};
    t.kind = id; t.a = t.b = t.c = -1;
    int blend = 0;
    auto children = [&](float fa, float fb) {
      int ia, oa, ib, ob;
      unpack16(fa, &ia, &oa);
      unpack16(fb, &ib, &ob);
      t.a = texture_node(ia, oa, depth + 1);
      t.b = texture_node(ib, ob, depth + 1);
      blend = std::max(texture_blend_depth[t.a], texture_blend_depth[t.b]);
    };
    switch (id) {
      case kTexConstant: color(id, off, t.p); break;
      case kTexBlend: {
        const float* q = record("textureBlendTextureArray", (size_t)off * 8, 8);
        children(q[0], q[1]);
        t.p[0] = q[2]; t.p[1] = q[3]; t.p[2] = q[4];
        blend += 1;
        break;
      }
      case kTexBullseye: {
        const float* q = record("textureBullseyeTextureArray", (size_t)off * 8, 8);
        children(q[3], q[4]);
        t.p[0] = q[0]; t.p[1] = q[1]; t.p[2] = q[2]; t.p[3] = q[5];
        break;
      }
      case kTexCheckerboard: case kTexPolkaDot: {
        const float* q = record(id == kTexCheckerboard ? "textureCheckerboardTextureArray" : "texturePolkaDotTextureArray", (size_t)off * 8, 8);
        children(q[2], q[3]);
        t.p[0] = jcos(q[1]); t.p[1] = jsin(q[1]); t.p[2] = q[4]; t.p[3] = q[5];
        break;
      }
      case kTexLDRImage:
        image("textureLDRImageTextureArray", "textureLDRImageTextureOffsetArray", off, &t.c, &t.a, &t.b, t.p);
        break;
      case kTexMarble: {
        const float* q = record("textureMarbleTextureArray", (size_t)off * 8, 8);
        unpack_argb(q[0], t.p); unpack_argb(q[1], t.p + 3); unpack_argb(q[2], t.p + 6);
        t.p[9] = q[3]; t.p[10] = q[4]; t.a = (int)q[6];
        break;
      }
      case kTexSimplexFBM: {
        const float* q = record("textureSimplexFractionalBrownianMotionTextureArray", (size_t)off * 4, 4);
        unpack_argb(q[0], t.p);
        t.p[3] = q[1]; t.p[4] = q[2]; t.a = (int)q[3];
        break;
      }
      case kTexDotProduct: case kTexSurfaceNormal: case kTexUV: break;
      default: {
        std::ostringstream os;
        os << "texture id " << id << " is not supported";
        throw Fail{DFC_E_UNSUPPORTED, os.str()};
      }
    }
    const int idx = (int)hs.textures.size();
    hs.textures.push_back(t);
    texture_blend_depth.push_back(blend);
    texture_index[key] = idx;
    return idx;
  }

  // ---- modifiers (renderer/gpu/AbstractModifierKernel.java:75, scene/modifier/*.java modify)
  std::map<std::pair<int, int>, int> modifier_index;
  int modifier(int id, int off) {
    if (id == kModNoOp || id == 0) return -1;
    const auto key = std::make_pair(id, off);
    auto it = modifier_index.find(key);
    if (it != modifier_index.end()) return it->second;
    DModifier d{};
    d.kind = id;
    if (id == kModNormalMapLDRImage) {
      image("modifierNormalMapLDRImageModifierArray", "modifierNormalMapLDRImageModifierOffsetArray", off, &d.texel, &d.rx, &d.ry, d.p);
    } else if (id == kModSimplexNoiseNormalMap) {
      const float* q = record("modifierSimplexNoiseNormalMapModifierArray", (size_t)off * 2, 2);
      d.p[0] = q[0]; d.p[1] = q[1];
    } else {
      throw Fail{DFC_E_UNSUPPORTED, "modifier id " + std::to_string(id) + " is not supported"};
    }
    const int idx = (int)hs.modifiers.size();
    hs.modifiers.push_back(d);
    modifier_index[key] = idx;
    return idx;
  }

  int material(int mid, int moff, int depth = 0) {
    auto key = std::make_pair(mid, moff);
    auto it = material_index.find(key);
    if (it != material_index.end()) return it->second;
    if (depth > 64) throw Fail{DFC_E_UNSUPPORTED, "composite materials nested deeper than 64 (or cyclic)"};
    if (moff < 0) throw Fail{DFC_E_INVALID_ARG, "negative material offset"};
    DMaterial m{};
    if (mid == kRefBullseye || mid == kRefCheckerboard || mid == kRefPolkaDot) {
      // CompiledMaterialCache.java toBullseyeMaterial / toCheckerboardMaterial / toPolkaDotMaterial (absolute offsets)
      const char* name = mid == kRefBullseye ? "materialBullseyeMaterialArray"
                         : mid == kRefCheckerboard ? "materialCheckerboardMaterialArray" : "materialPolkaDotMaterialArray";
      const float* q = record(name, (size_t)moff, 8);
      DComposite c{};
      c.kind = mid;
      int ia, oa, ib, ob;
      if (mid == kRefBullseye) {
        unpack16(q[3], &ia, &oa); unpack16(q[4], &ib, &ob);
        c.p[0] = q[0]; c.p[1] = q[1]; c.p[2] = q[2]; c.p[3] = q[5];
      } else {
        unpack16(q[2], &ia, &oa); unpack16(q[3], &ib, &ob);
        c.p[0] = jcos(q[1]); c.p[1] = jsin(q[1]); c.p[2] = q[4]; c.p[3] = q[5];
      }
      c.a = material(ia, oa, depth + 1);
      c.b = material(ib, ob, depth + 1);
      m.kind = kMatComposite;
      m.flags = (int)hs.composites.size();
      hs.composites.push_back(c);
    } else {
      const char* name = nullptr;
      switch (mid) {
        case kMatMatteId: name = "materialMatteMaterialArray"; break;
        case kMatMirrorId: name = "materialMirrorMaterialArray"; break;
        case kMatGlassId: name = "materialGlassMaterialArray"; break;
        case kMatMetalId: name = "materialMetalMaterialArray"; break;
        case kMatPlasticId: name = "materialPlasticMaterialArray"; break;
        case kMatDisneyId: name = "materialDisneyMaterialArray"; break;
        case kMatClearCoatId: name = "materialClearCoatMaterialArray"; break;
        case kMatGlossyId: name = "materialGlossyMaterialArray"; break;
        case kMatSubstrateId: name = "materialSubstrateMaterialArray"; break;
        case kMatTranslucentId: name = "materialTranslucentMaterialArray"; break;
        case kMatUberId: name = "materialUberMaterialArray"; break;
        default: throw Fail{DFC_E_UNSUPPORTED, "material id " + std::to_string(mid) + " is not supported"};
      }
      const auto& A = I(name);
      const MatShape sh = mat_shape(mid);
      int ids[kTexPositions], offs[kTexPositions];
      for (int slot = 0; slot < kTexPositions / 2; ++slot) {
        const bool needed = ((sh.tex_mask >> (2 * slot)) & 3u) != 0 || slot == 0 || 2 * slot + 1 == sh.plain_pos;
        if (needed) texref(A, moff, slot, &ids[2 * slot], &offs[2 * slot], &ids[2 * slot + 1], &offs[2 * slot + 1]);
        else ids[2 * slot] = ids[2 * slot + 1] = offs[2 * slot] = offs[2 * slot + 1] = 0;
      }
      int plain_v = 0;
      if (sh.plain_slot >= 0) plain_v = plain(A, moff, sh.plain_slot);
      if (sh.plain_pos >= 0) plain_v = ids[sh.plain_pos];
      const int mod = modifier(ids[1], offs[1]);
      bool all_constant = mod < 0;
      for (int p = 0; p < kTexPositions; ++p)
        if (((sh.tex_mask >> p) & 1u) && ids[p] != kTexConstantId) all_constant = false;
      if (all_constant) {
        MatInputs in{};
        for (int p = 0; p < kTexPositions; ++p)
          if ((sh.tex_mask >> p) & 1u) color(ids[p], offs[p], in.c[p]);
        in.plain = plain_v;
        derive_material(mid, in, &m);
      } else {
        DTexMaterial tm{};
        tm.ref_id = mid;
        tm.modifier = mod;
        tm.plain = plain_v;
        for (int p = 0; p < kTexPositions; ++p) {
          tm.tex[p] = -1;
          if (!((sh.tex_mask >> p) & 1u)) continue;
          tm.tex[p] = texture_node(ids[p], offs[p], 0);
          if (texture_blend_depth[tm.tex[p]] > kMaxBlendDepth)
            throw Fail{DFC_E_UNSUPPORTED, "BlendTexture nested deeper than " + std::to_string(kMaxBlendDepth)};
        }
        m.kind = kMatTextured;
        m.flags = (int)hs.texmats.size();
        hs.texmats.push_back(tm);
      }
    }
    int idx = (int)hs.materials.size();
    hs.materials.push_back(m);
    material_index[key] = idx;
    return idx;
  }

  void copy34(const float* m16, float* out12) { std::memcpy(out12, m16, 12 * sizeof(float)); }
  bool affine(const float* m16) { return m16[12] == 0.0f && m16[13] == 0.0f && m16[14] == 0.0f && m16[15] == 1.0f; }
  bool is_identity(const float* m16) {
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c)
        if (m16[r * 4 + c] != (r == c ? 1.0f : 0.0f)) return false;
    return true;
  }

  void lights() {
    const auto& L = I("lightIDAndOffsetArray");
    for (size_t k = 0; k < L.size(); ++k) {
      uint32_t v = (uint32_t)L[k];
      int id = (v >> 16) & 0xFFFF, rel = v & 0xFFFF;
      DLight lt;
      std::memset(&lt, 0, sizeof lt);
      lt.type = id;
      lt.perez = -1;
      switch (id) {
        case kLightDiffuseArea: {  // CompiledLightCache.java:68-103
          const auto& A = F("lightDiffuseAreaLightArray");
          size_t o = (size_t)rel * 40;
          if (o + 40 > A.size()) throw Fail{DFC_E_INVALID_ARG, "diffuse area light offset out of range"};
          const float* q = A.data() + o;
          if (!affine(q) || !affine(q + 16)) throw Fail{DFC_E_UNSUPPORTED, "projective light transforms are not supported"};
          copy34(q, lt.o2w); copy34(q + 16, lt.w2o);
          lt.radiance[0] = q[32]; lt.radiance[1] = q[33]; lt.radiance[2] = q[34];
          lt.shape = (int)q[35];
          int soff = (int)q[36];
          lt.shape_data = lt.shape == kShapeTriangle ? soff / 24 : 0;
          lt.area = q[37];
          lt.two_sided = q[38] != 0.0f;
          if (lt.shape == kShapeTriangle) {
            const auto& T = F("shape3FTriangle3FArray");
            if (soff < 0 || soff % 24 != 0 || (size_t)soff + 24 > T.size()) throw Fail{DFC_E_INVALID_ARG, "area light triangle offset out of range"};
            const float* t = T.data() + soff;
            double e1[3] = {t[3] - t[0], t[4] - t[1], t[5] - t[2]}, e2[3] = {t[6] - t[0], t[7] - t[1], t[8] - t[2]};
            double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            float cf[3] = {(float)c[0], (float)c[1], (float)c[2]};
            lt.area = std::sqrt(cf[0] * cf[0] + cf[1] * cf[1] + cf[2] * cf[2]) * 0.5f;  // Triangle3F.getSurfaceArea
          } else if (lt.shape == kShapeSphere) {
            lt.area = 4.0f * 3.14159265358979323846f;
          }
          break;
        }
        case kLightPoint: {
          const auto& A = F("lightPointLightArray");
          size_t o = (size_t)rel * 8;
          if (o + 8 > A.size()) throw Fail{DFC_E_INVALID_ARG, "point light offset out of range"};
          std::memcpy(lt.radiance, A.data() + o, 12);
          std::memcpy(lt.pos, A.data() + o + 3, 12);
          break;
        }
        case kLightSpot: {
          const auto& A = F("lightSpotLightArray");
          size_t o = (size_t)rel * 24;
          if (o + 24 > A.size()) throw Fail{DFC_E_INVALID_ARG, "spot light offset out of range"};
          const float* q = A.data() + o;
          copy34(q, lt.w2o);
          std::memcpy(lt.radiance, q + 16, 12);
          std::memcpy(lt.pos, q + 19, 12);
          lt.cos_cone = q[22];
          lt.cos_cone_delta = q[23];
          break;
        }
        case kLightDirectional: {
          const auto& A = F("lightDirectionalLightArray");
          size_t o = (size_t)rel * 8;
          if (o + 8 > A.size()) throw Fail{DFC_E_INVALID_ARG, "directional light offset out of range"};
          const float* q = A.data() + o;
          std::memcpy(lt.radiance, q, 12);
          std::memcpy(lt.dir, q + 3, 12);
          lt.radius = q[6];
          break;
        }
        case kLightPerez: {
          const auto& O = I("lightPerezLightOffsetArray");
          const auto& A = F("lightPerezLightArray");
          if (rel < 0 || (size_t)rel >= O.size()) throw Fail{DFC_E_INVALID_ARG, "Perez light offset out of range"};
          int off = O[rel];
          if (off < 0 || (size_t)off + 48 > A.size()) throw Fail{DFC_E_INVALID_ARG, "Perez light record out of range"};
          validate_distribution2(A, (size_t)off + 48);
          lt.perez = off;
          lt.radius = A[off + 45];
          std::memcpy(lt.radiance, A.data() + off + 32, 12);
          break;
        }
        case kLightImage: {  // CompiledLightCache.java:1393-1460; kept after the Perez records in the sky pool
          const auto& O = I("lightImageLightOffsetArray");
          const auto& A = F("lightImageLightArray");
          if (rel < 0 || (size_t)rel >= O.size()) throw Fail{DFC_E_INVALID_ARG, "image light offset out of range"};
          const int off = O[rel];
          if (off < 0 || (size_t)off + 2352 > A.size()) throw Fail{DFC_E_INVALID_ARG, "image light record out of range"};
          const float rx = A[off + 36], ry = A[off + 37];
          if (!(rx >= 1.0f && ry >= 1.0f) || rx != std::floor(rx) || ry != std::floor(ry) ||
              (size_t)off + 2352 + (size_t)rx * (size_t)ry * 3 > A.size())
            throw Fail{DFC_E_INVALID_ARG, "image light resolution out of range"};
          validate_distribution2(A, (size_t)off + 40);
          lt.perez = (int)F("lightPerezLightArray").size() + off;
          lt.radius = A[off + 35];
          break;
        }
        default:
          throw Fail{DFC_E_UNSUPPORTED, "light id " + std::to_string(id) + " is not supported"};
      }
      light_by_key[(id << 16) | rel] = (int)hs.lights.size();
      hs.lights.push_back(lt);
    }
  }

  // Checks a packed Distribution2F (sampler/Distribution2F.java toArray) so that
  // every offset and count the device follows stays inside the array.
  void validate_distribution1(const StagedF& A, size_t off) {
    if (off + 4 > A.size()) throw Fail{DFC_E_INVALID_ARG, "distribution out of range"};
    const float len = A[off], cdf = A[off + 1], cnt = A[off + 2];
    if (!(cnt >= 1.0f && cdf == cnt + 1.0f && len == 4.0f + cdf + cnt) || off + (size_t)len > A.size())
      throw Fail{DFC_E_INVALID_ARG, "malformed Distribution1F"};
  }
  void validate_distribution2(const StagedF& A, size_t base) {
    if (base + 3 > A.size()) throw Fail{DFC_E_INVALID_ARG, "distribution out of range"};
    const float tab = A[base + 1];  // offset table length = 1 + conditionals
    if (!(tab >= 2.0f && tab < 1.0e6f) || base + 2 + (size_t)tab > A.size()) throw Fail{DFC_E_INVALID_ARG, "malformed Distribution2F"};
    const size_t n = (size_t)tab;
    if (!(A[base + 2] >= 0.0f)) throw Fail{DFC_E_INVALID_ARG, "malformed Distribution2F offset"};
    validate_distribution1(A, base + (size_t)A[base + 2]);
    const size_t marginal = base + (size_t)A[base + 2];
    if ((size_t)A[marginal + 2] != n - 1) throw Fail{DFC_E_INVALID_ARG, "Distribution2F marginal count mismatch"};
    for (size_t k = 0; k + 1 < n; ++k) {
      const float o = A[base + 3 + k];
      if (!(o >= 0.0f)) throw Fail{DFC_E_INVALID_ARG, "malformed Distribution2F offset"};
      validate_distribution1(A, base + (size_t)o);
    }
  }

  // World bounding sphere of a top-level item, used by the traversal to reject
  // candidates before the exact object-space test.  Spheres: the image of the
  // unit sphere under the object-to-world map lies within the largest singular
  // value of its 3x3 part around the translated origin.  Meshes are marked with
  // a negative radius (they are entered, not tested).  Others: the box's sphere.
  F4 bounding_sphere(const DPrim& pr, const Box& b) {
    if (pr.shape == kShapeMesh) return F4{0, 0, 0, -1};
    if (pr.shape == kShapeSphere) {
      const float* m = pr.o2w;
      double a[3][3] = {{m[0], m[1], m[2]}, {m[4], m[5], m[6]}, {m[8], m[9], m[10]}};
      double ata[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) ata[i][j] = a[0][i] * a[0][j] + a[1][i] * a[1][j] + a[2][i] * a[2][j];
      double v[3] = {1, 1, 1}, lam = 0;
      for (int it = 0; it < 64; ++it) {
        double w[3] = {ata[0][0] * v[0] + ata[0][1] * v[1] + ata[0][2] * v[2], ata[1][0] * v[0] + ata[1][1] * v[1] + ata[1][2] * v[2],
                       ata[2][0] * v[0] + ata[2][1] * v[1] + ata[2][2] * v[2]};
        double nw = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (nw == 0) break;
        lam = nw;
        for (int k = 0; k < 3; ++k) v[k] = w[k] / nw;
      }
      // the Frobenius norm bounds the largest singular value from above; take the
      // smaller of the two bounds with a relative margin
      double frob = std::sqrt(ata[0][0] + ata[1][1] + ata[2][2]);
      double r = std::fmin(std::sqrt(lam) * (1.0 + 1e-4), frob);
      return F4{m[3], m[7], m[11], (float)(r * (1.0 + 1e-5))};
    }
    float c[3], r2 = 0;
    for (int k = 0; k < 3; ++k) { c[k] = 0.5f * (b.lo[k] + b.hi[k]); float h = 0.5f * (b.hi[k] - b.lo[k]); r2 += h * h; }
    return F4{c[0], c[1], c[2], std::sqrt(r2) * 1.0001f + 1e-6f};
  }

  // Collects the triangle offsets of one mesh by walking its threaded stream.
  void mesh_triangles(int off, std::vector<int>& tris) {
    const auto& M = I("shape3FTriangleMesh3FArray");
    if (off < 0 || (size_t)off + 8 > M.size()) throw Fail{DFC_E_INVALID_ARG, "triangle mesh offset out of range"};
    const size_t limit = M.size() / 4 + 8;
    size_t steps = 0;
    int rel = 0;
    while (rel != -1) {
      if (++steps > limit) throw Fail{DFC_E_INVALID_ARG, "triangle mesh stream does not terminate"};
      size_t o = (size_t)off + (size_t)rel;
      if (rel < 0 || o + 4 > M.size()) throw Fail{DFC_E_INVALID_ARG, "triangle mesh node out of range"};
      int id = M[o], next = M[o + 2], lc = M[o + 3];
      if (id == 1) {
        if (lc < 0 || o + 4 + (size_t)lc > M.size()) throw Fail{DFC_E_INVALID_ARG, "triangle mesh leaf out of range"};
        for (int k = 0; k < lc; ++k) tris.push_back(M[o + 4 + k]);
        rel = next;
      } else if (id == 2) {
        rel = lc;
      } else {
        throw Fail{DFC_E_INVALID_ARG, "unknown triangle mesh node id"};
      }
    }
  }

  // CompiledShape3FCache.java:90-310 record lengths
  struct RecordArray { int id; const char* name; int length; size_t base; };
  // (length 0: Polygon3F, variable length 13 + 2 * point count)
  RecordArray record_arrays[8] = {
      {kShapeDisk, "shape3FDisk3FArray", 4, 0}, {kShapeCylinder, "shape3FCylinder3FArray", 4, 0},
      {kShapeCone, "shape3FCone3FArray", 4, 0}, {kShapeParaboloid, "shape3FParaboloid3FArray", 4, 0},
      {kShapeHyperboloid, "shape3FHyperboloid3FArray", 16, 0}, {kShapeCuboid, "shape3FRectangularCuboid3FArray", 8, 0},
      {kShapeTorus, "shape3FTorus3FArray", 2, 0}, {kShapePolygon, "shape3FPolygon3FArray", 0, 0}};

  void run() {
    const auto& P = I("primitiveArray");
    const auto& X = F("primitiveMatrix44FArray");
    const auto& T = F("shape3FTriangle3FArray");
    const auto& R = F("shape3FRectangle3FArray");
    const auto& AB = F("boundingVolume3FAxisAlignedBoundingBox3FArray");
    const auto& BS = F("boundingVolume3FBoundingSphere3FArray");
    const auto& C = F("cameraArray");
    if (P.size() % 8 != 0) throw Fail{DFC_E_INVALID_ARG, "primitiveArray length is not a multiple of 8"};
    const int np = (int)(P.size() / 8);
    if (X.size() < (size_t)np * 32) throw Fail{DFC_E_INVALID_ARG, "primitiveMatrix44FArray is shorter than 32 floats per primitive"};
    if (C.size() < 19) throw Fail{DFC_E_INVALID_ARG, "cameraArray needs 19 floats"};
    std::memcpy(hs.camera, C.data(), sizeof hs.camera);
    hs.rects.assign(R.begin(), R.end());
    // the record-sized shapes share one float pool on the device
    for (RecordArray& ra : record_arrays) {
      ra.base = hs.shapes.size();
      const auto& A = F(ra.name);
      hs.shapes.insert(hs.shapes.end(), A.begin(), A.end());
    }
    if (hs.shapes.empty()) hs.shapes.assign(4, 0.0f);
    hs.perez.assign(F("lightPerezLightArray").begin(), F("lightPerezLightArray").end());  // the sky pool: Perez records, then image light records
    {
      const auto& img = F("lightImageLightArray");
      hs.perez.insert(hs.perez.end(), img.begin(), img.end());
    }
    if (hs.rects.empty()) hs.rects.assign(16, 0.0f);
    if (hs.perez.empty()) hs.perez.assign(64, 0.0f);
    lights();
    std::map<int, int> blas_by_offset;  // mesh stream offset -> index in blas_info
    struct BlasInfo { int root, first, count; };
    std::vector<BlasInfo> blas_info;
    std::vector<Box> tlas_boxes;
    std::vector<int> tlas_prims;
    std::vector<F4> tlas_spheres;
    for (int p = 0; p < np; ++p) {
      const int32_t* q = P.data() + (size_t)p * 8;
      const float* m = X.data() + (size_t)p * 32;
      if (!affine(m) || !affine(m + 16)) throw Fail{DFC_E_UNSUPPORTED, "projective primitive transforms are not supported"};
      DPrim pr;
      std::memset(&pr, 0, sizeof pr);
      copy34(m, pr.o2w);
      copy34(m + 16, pr.w2o);
      pr.identity = is_identity(m) && is_identity(m + 16);
      pr.shape = q[6];
      const int soff = q[7];
      pr.light = -1;
      if (q[1] != 0) {
        uint32_t al = (uint32_t)q[1];
        auto it = light_by_key.find((int)(((al >> 16) & 0xFFFF) << 16 | (al & 0xFFFF)));
        if (it == light_by_key.end()) throw Fail{DFC_E_INVALID_ARG, "primitive area light is not in lightIDAndOffsetArray"};
        pr.light = it->second;
      }
      pr.material = material(q[4], q[5]);
      switch (pr.shape) {
        case kShapeTriangle:
          if (soff < 0 || soff % 24 != 0 || (size_t)soff + 24 > T.size()) throw Fail{DFC_E_INVALID_ARG, "triangle offset out of range"};
          pr.data = soff / 24;
          break;
        case kShapeRectangle:
          if (soff < 0 || soff % 16 != 0 || (size_t)soff + 16 > R.size()) throw Fail{DFC_E_INVALID_ARG, "rectangle offset out of range"};
          pr.data = soff / 16;
          break;
        case kShapeSphere: case kShapePlane:
          pr.data = 0;
          break;
        case kShapeDisk: case kShapeCylinder: case kShapeCone: case kShapeParaboloid: case kShapeHyperboloid:
        case kShapeCuboid: case kShapeTorus: case kShapePolygon: {
          const RecordArray* ra = nullptr;
          for (const RecordArray& x : record_arrays) if (x.id == pr.shape) ra = &x;
          const auto& A = F(ra->name);
          const size_t n = A.size();
          if (ra->length == 0) {  // Polygon3F: 13 + 2 * count floats
            if (soff < 0 || (size_t)soff + 13 > n) throw Fail{DFC_E_INVALID_ARG, "polygon offset out of range"};
            const float cnt = A[soff + 12];
            if (!(cnt >= 3.0f) || cnt != std::floor(cnt) || (size_t)soff + 13 + 2 * (size_t)cnt > n)
              throw Fail{DFC_E_INVALID_ARG, "polygon point count out of range"};
          } else if (soff < 0 || soff % ra->length != 0 || (size_t)soff + (size_t)ra->length > n) {
            throw Fail{DFC_E_INVALID_ARG, std::string(ra->name) + " offset out of range"};
          }
          pr.data = (int)(ra->base + (size_t)soff);
          hs.record_shapes = true;
          break;
        }
        case kShapeMesh: {
          auto it = blas_by_offset.find(soff);
          if (it == blas_by_offset.end()) {
            const auto t_blas = std::chrono::steady_clock::now();
            std::vector<int> offs;
            mesh_triangles(soff, offs);
            for (int to : offs)
              if (to < 0 || to % 24 != 0 || (size_t)to + 24 > T.size()) throw Fail{DFC_E_INVALID_ARG, "mesh triangle offset out of range"};
            if (offs.empty()) throw Fail{DFC_E_INVALID_ARG, "empty triangle mesh"};
            if (device_blas) {  // the device builds this hierarchy into its own node range (dfc_blas.cu)
              HostScene::BlasJob job;
              job.index_off = hs.blas_tri_index.size();
              job.count = (int)offs.size();
              job.node_base = hs.blas_nodes;
              job.node_cap = blas_node_capacity(job.count);
              job.tri_first = (int)hs.blas_tris;
              for (int to : offs) hs.blas_tri_index.push_back(to / 24);
              hs.blas_jobs.push_back(job);
              hs.blas_nodes += job.node_cap;
              hs.blas_tris += job.count;
              blas_info.push_back(BlasInfo{job.node_base, job.tri_first, job.count});
              it = blas_by_offset.emplace(soff, (int)blas_info.size() - 1).first;
              hs.triangles += (int64_t)offs.size();
              hs.blas_ms += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_blas).count();
              pr.data = job.node_base;
              pr.tri_first = job.tri_first;
              pr.tri_count = job.count;
              break;
            }
            std::vector<Box> boxes(offs.size());
            parallel_for(offs.size(), [&](size_t a, size_t b) {
              for (size_t k = a; k < b; ++k) {
                const float* t = T.data() + offs[k];
                boxes[k].grow_point(t); boxes[k].grow_point(t + 3); boxes[k].grow_point(t + 6);
              }
            });
            std::vector<int> order;
            int root = build_bvh4(boxes, 4, hs.nodes, order);
            const int first = (int)(hs.tri_pos.size() / 3);
            hs.tri_pos.resize(hs.tri_pos.size() + 3 * order.size());
            F4* tp = hs.tri_pos.data() + (size_t)first * 3;
            parallel_for(order.size(), [&](size_t a, size_t b) {
              for (size_t j = a; j < b; ++j) {
                const int off = offs[order[j]];
                const float* t = T.data() + off;
                float idx;
                int ti = off / 24;
                std::memcpy(&idx, &ti, 4);
                tp[3 * j] = F4{t[0], t[1], t[2], idx};
                tp[3 * j + 1] = F4{t[3], t[4], t[5], 0.0f};
                tp[3 * j + 2] = F4{t[6], t[7], t[8], 0.0f};
              }
            });
            // re-base the leaf ranges of this hierarchy onto the global triangle array
            for (size_t n = (size_t)root; n < hs.nodes.size(); ++n) {
              int* ch = hs.nodes[n].child;
              int* cn = hs.nodes[n].count;
              for (int s = 0; s < 4; ++s) if (ch[s] < 0 && cn[s] > 0) ch[s] = ~(~ch[s] + first);
            }
            blas_info.push_back(BlasInfo{root, first, (int)offs.size()});
            it = blas_by_offset.emplace(soff, (int)blas_info.size() - 1).first;
            hs.triangles += (int64_t)offs.size();
            hs.blas_ms += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_blas).count();
          }
          pr.data = blas_info[it->second].root;
          pr.tri_first = blas_info[it->second].first;
          pr.tri_count = blas_info[it->second].count;
          break;
        }
        default:
          throw Fail{DFC_E_UNSUPPORTED, "shape id " + std::to_string(pr.shape) + " is not supported"};
      }
      // bounding volume (CompiledBoundingVolume3FCache.java:53-78); relative offsets
      const int bvid = q[2], bvoff = q[3];
      if (bvid == kBVInfiniteId) {
        hs.unbounded.push_back(p);
      } else {
        Box b;
        if (bvid == kBVAabbId) {
          if (bvoff < 0 || (size_t)bvoff * 8 + 6 > AB.size()) throw Fail{DFC_E_INVALID_ARG, "bounding box offset out of range"};
          const float* bb = AB.data() + (size_t)bvoff * 8;
          float mx[3] = {bb[0], bb[1], bb[2]}, mn[3] = {bb[3], bb[4], bb[5]};
          b.grow_point(mx); b.grow_point(mn);
        } else if (bvid == kBVSphereId) {
          if (bvoff < 0 || (size_t)bvoff * 4 + 4 > BS.size()) throw Fail{DFC_E_INVALID_ARG, "bounding sphere offset out of range"};
          const float* s = BS.data() + (size_t)bvoff * 4;
          float lo[3] = {s[0] - s[3], s[1] - s[3], s[2] - s[3]}, hi[3] = {s[0] + s[3], s[1] + s[3], s[2] + s[3]};
          b.grow_point(lo); b.grow_point(hi);
        } else {
          throw Fail{DFC_E_UNSUPPORTED, "bounding volume id " + std::to_string(bvid) + " is not supported"};
        }
        // widen by a few ulps so that the culling stays conservative
        for (int k = 0; k < 3; ++k) {
          float e = 1e-6f * (std::fabs(b.lo[k]) + std::fabs(b.hi[k]) + 1.0f);
          b.lo[k] -= e; b.hi[k] += e;
        }
        tlas_boxes.push_back(b);
        tlas_prims.push_back(p);
        tlas_spheres.push_back(bounding_sphere(pr, b));
      }
      hs.prims.push_back(pr);
    }
    // Items whose box covers a large part of the scene (a terrain under
    // everything else, the walls of a room) can be tested before the top
    // level rather than inside it: their hit usually comes first along a ray
    // and then culls most of the top level.  At most DFC_FIRST_ITEMS of them,
    // each at least a fifth of the scene box's surface area, largest first.
#ifndef DFC_FIRST_ITEMS
#define DFC_FIRST_ITEMS 0
#endif
    constexpr size_t kFirstItems = DFC_FIRST_ITEMS;
    constexpr float kFirstArea = 0.2f;
    if (kFirstItems > 0 && tlas_boxes.size() > 1) {
      Box scene_box;
      for (const Box& b : tlas_boxes) scene_box.grow(b);
      std::vector<size_t> big;
      for (size_t k = 0; k < tlas_boxes.size(); ++k)
        if (tlas_boxes[k].area() >= kFirstArea * scene_box.area()) big.push_back(k);
      std::stable_sort(big.begin(), big.end(), [&](size_t a, size_t b) { return tlas_boxes[a].area() > tlas_boxes[b].area(); });
      if (big.size() > kFirstItems) big.resize(kFirstItems);
      if (big.size() < tlas_boxes.size()) {
        std::vector<char> out(tlas_boxes.size(), 0);
        for (size_t k : big) { hs.unbounded.push_back(tlas_prims[k]); out[k] = 1; }
        size_t w = 0;
        for (size_t k = 0; k < tlas_boxes.size(); ++k) {
          if (out[k]) continue;
          tlas_boxes[w] = tlas_boxes[k]; tlas_prims[w] = tlas_prims[k]; tlas_spheres[w] = tlas_spheres[k];
          ++w;
        }
        tlas_boxes.resize(w); tlas_prims.resize(w); tlas_spheres.resize(w);
      }
    }
    if (!tlas_boxes.empty()) {
      const auto t_tlas = std::chrono::steady_clock::now();
      std::vector<int> order;
      hs.tlas_root = build_bvh4(tlas_boxes, 4, hs.nodes, order);
      hs.tlas_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_tlas).count();
      if (hs.blas_nodes > 0) {  // host nodes follow the device-built region
        for (BVH4Node& nd : hs.nodes)
          for (int c = 0; c < 4; ++c)
            if (nd.child[c] >= 0) nd.child[c] += hs.blas_nodes;
        hs.tlas_root += hs.blas_nodes;
      }
      hs.tlas_items.resize(order.size());
      hs.tlas_bound.resize(order.size());
      for (size_t k = 0; k < order.size(); ++k) {
        hs.tlas_items[k] = tlas_prims[order[k]];
        hs.tlas_bound[k] = tlas_spheres[order[k]];
      }
    } else {
      hs.tlas_root = -1;
    }
    if (hs.tlas_items.empty()) { hs.tlas_items.push_back(0); hs.tlas_bound.push_back(F4{0, 0, 0, -1}); }
    if (hs.unbounded.empty()) hs.unbounded_storage.push_back(0);
    if (hs.tri_pos.empty() && hs.blas_tris == 0) hs.tri_pos.assign(3, F4{0, 0, 0, 0});
    if (hs.nodes.empty()) hs.nodes.push_back(BVH4Node{});
    if (hs.lights.empty()) { DLight z; std::memset(&z, 0, sizeof z); hs.lights_storage_pad = 1; hs.lights.push_back(z); }
    if (hs.materials.empty()) { DMaterial z; std::memset(&z, 0, sizeof z); hs.materials.push_back(z); }
  }
};

}  // namespace

void stage_copy(StagedF& dst, const float* src, size_t count) { stage_copy_into(dst, src, count); }
void stage_copy(StagedI& dst, const int32_t* src, size_t count) { stage_copy_into(dst, src, count); }

int ingest_scene(Staged& st, int layout, HostScene* out, std::string* err, bool device_blas) {
  try {
    if (layout != 1 && layout != 2) throw Fail{DFC_E_INVALID_ARG, "layout_version must be 1 or 2"};
    HostScene hs;
    Decoder d(st, layout, hs, device_blas);
    d.run();
    // the triangle records go to the device as they are, from the staging array
    static const float kNoTriangle[24] = {0};
    auto tri = st.f32.find("shape3FTriangle3FArray");
    if (tri != st.f32.end() && !tri->second.empty()) {
      hs.tri_attr = tri->second.data();
      hs.tri_attr_count = tri->second.size();
    } else {
      hs.tri_attr = kNoTriangle;
      hs.tri_attr_count = 24;
    }
    *out = std::move(hs);
    return DFC_OK;
  } catch (const Fail& f) {
    *err = f.msg;
    return f.code;
  } catch (const std::exception& e) {
    *err = e.what();
    return DFC_E_INVALID_ARG;
  }
}

}  // namespace dfc
