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
#include <thread>

#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <sstream>

#include "dfc_bvh.h"

namespace dfc {
namespace {

enum {
  kMatClearCoatId = 3, kMatDisneyId = 4, kMatGlassId = 7, kMatGlossyId = 8, kMatMatteId = 11, kMatMetalId = 12, kMatMirrorId = 13,
  kMatPlasticId = 14, kMatSubstrateId = 16, kMatTranslucentId = 18, kMatUberId = 19
};
enum { kTexConstantId = 4, kModNoOpId = 2 };
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

struct Fail {
  int code;
  std::string msg;
};

template <typename T>
const std::vector<T>& get(const std::map<std::string, std::vector<T>>& m, const char* name) {
  static const std::vector<T> empty;
  auto it = m.find(name);
  return it == m.end() ? empty : it->second;
}

float roughness_to_alpha(float r) {  // scene/microfacet/MicrofacetDistribution.java:convertRoughnessToAlpha
  float x = std::fmax(r, 1.0e-3f), y = std::log(x);
  return 1.62142f + 0.819955f * y + 0.1734f * y * y + 0.0171201f * y * y * y + 0.000640711f * y * y * y * y;
}

struct Decoder {
  const Staged& st;
  int layout;
  HostScene& hs;
  std::map<std::pair<int, int>, int> material_index;
  std::map<int, int> light_by_key;  // (id << 16 | rel) -> index

  Decoder(const Staged& s, int l, HostScene& h) : st(s), layout(l), hs(h) {}

  const std::vector<float>& F(const char* n) { return get(st.f32, n); }
  const std::vector<int32_t>& I(const char* n) { return get(st.i32, n); }

  void texref(const std::vector<int32_t>& arr, int base, int slot, int* ida, int* offa, int* idb, int* offb) {
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
  int plain(const std::vector<int32_t>& arr, int base, int slot) {
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
  float value(int id, int off) { float c[3]; color(id, off, c); return (c[0] + c[1] + c[2]) / 3.0f; }
  void check_modifier(int id) {
    if (id != kModNoOpId && id != 0) throw Fail{DFC_E_UNSUPPORTED, "modifier id " + std::to_string(id) + " is not supported"};
  }

  int material(int mid, int moff) {
    auto key = std::make_pair(mid, moff);
    auto it = material_index.find(key);
    if (it != material_index.end()) return it->second;
    DMaterial m;
    std::memset(&m, 0, sizeof m);
    int a, ao, b, bo;
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
    if (moff < 0) throw Fail{DFC_E_INVALID_ARG, "negative material offset"};
    texref(A, moff, 0, &a, &ao, &b, &bo);  // emission texture, modifier
    color(a, ao, m.emission);
    check_modifier(b);
    auto sat0 = [](float* c) { for (int k = 0; k < 3; ++k) c[k] = std::fmax(c[k], 0.0f); };
    auto black = [](const float* c) { return c[0] == 0.0f && c[1] == 0.0f && c[2] == 0.0f; };
    switch (mid) {
      case kMatMatteId: {  // scene/material/MatteMaterial.java:285
        texref(A, moff, 1, &a, &ao, &b, &bo);
        float ang = value(a, ao);
        color(b, bo, m.c0); sat0(m.c0);
        ang = std::fmin(std::fmax(ang, 0.0f), 90.0f) * (3.14159265358979323846f / 180.0f);
        if (ang == 0.0f) m.kind = kMatLambert;
        else { m.kind = kMatOrenNayar; float s2 = ang * ang; m.on_a = 1.0f - (s2 / (2.0f * (s2 + 0.33f))); m.on_b = 0.45f * s2 / (s2 + 0.09f); }
        break;
      }
      case kMatMirrorId: {  // MirrorMaterial.java:235
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, m.c0); sat0(m.c0);
        m.kind = black(m.c0) ? kMatNone : kMatMirror;
        break;
      }
      case kMatGlassId: {  // GlassMaterial.java:501
        texref(A, moff, 1, &a, &ao, &b, &bo);
        m.eta = value(a, ao);
        texref(A, moff, 2, &a, &ao, &b, &bo);
        color(a, ao, m.c0); sat0(m.c0); color(b, bo, m.c1); sat0(m.c1);
        texref(A, moff, 3, &a, &ao, &b, &bo);
        float ru = value(a, ao), rv = value(b, bo);
        bool remap = plain(A, moff, 4) != 0;
        m.has_kr = !black(m.c0); m.has_kt = !black(m.c1);
        if (!m.has_kr && !m.has_kt) m.kind = kMatNone;
        else if (ru == 0.0f && rv == 0.0f) m.kind = kMatGlassSpec;
        else {
          m.kind = kMatGlassRough;
          m.ax = remap ? roughness_to_alpha(ru) : ru;
          m.ay = remap ? roughness_to_alpha(rv) : rv;
        }
        break;
      }
      case kMatMetalId: {  // MetalMaterial.java:436
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, m.c1); color(b, bo, m.c2);
        texref(A, moff, 2, &a, &ao, &b, &bo);
        float ru = value(a, ao), rv = value(b, bo);
        bool remap = plain(A, moff, 3) != 0;
        m.ax = remap ? roughness_to_alpha(ru) : ru;
        m.ay = remap ? roughness_to_alpha(rv) : rv;
        m.kind = kMatMetal;
        break;
      }
      case kMatPlasticId: {  // PlasticMaterial.java:389
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, m.c0); sat0(m.c0); color(b, bo, m.c1); sat0(m.c1);
        texref(A, moff, 2, &a, &ao, &b, &bo);
        float r = value(a, ao);
        bool remap = plain(A, moff, 3) != 0;
        m.ax = m.ay = remap ? roughness_to_alpha(r) : r;
        m.has_kr = !black(m.c0); m.has_kt = !black(m.c1);
        m.kind = (m.has_kr || m.has_kt) ? kMatPlastic : kMatNone;
        break;
      }
      case kMatClearCoatId: {  // ClearCoatMaterial.java: kd, ks (the lobe is chosen per hit)
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, m.c0); color(b, bo, m.c1);
        m.kind = kMatClearCoat;
        break;
      }
      case kMatGlossyId: {  // GlossyMaterial.java: TorranceSparrowBRDF(kr, ConductorFresnel(kr, 1, 1), TR(r, r))
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, m.c0);
        const float r = value(b, bo);
        m.ax = m.ay = std::fmax(r, 0.001f);
        // ConductorFresnel with etaI = kr, etaT = k = 1: relative eta and k are 1 / kr
        for (int k = 0; k < 3; ++k) { m.c1[k] = 1.0f / m.c0[k]; m.c2[k] = 1.0f / m.c0[k]; }
        m.kind = kMatGlossy;
        break;
      }
      case kMatSubstrateId: {  // SubstrateMaterial.java: FresnelBlendBRDF(kd, ks, TR(ru, rv))
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, m.c0); sat0(m.c0); color(b, bo, m.c1); sat0(m.c1);
        texref(A, moff, 2, &a, &ao, &b, &bo);
        const float ru = value(a, ao), rv = value(b, bo);
        const bool remap = plain(A, moff, 3) != 0;
        m.ax = std::fmax(remap ? roughness_to_alpha(ru) : ru, 0.001f);
        m.ay = std::fmax(remap ? roughness_to_alpha(rv) : rv, 0.001f);
        m.kind = (black(m.c0) && black(m.c1)) ? kMatNone : kMatSubstrate;
        break;
      }
      case kMatTranslucentId: {  // TranslucentMaterial.java; flags: 1 Lambert BRDF, 2 Lambert BTDF, 4 TS BRDF, 8 TS BTDF
        float kd[3], ks[3], rf[3], tr[3];
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, kd); sat0(kd); color(b, bo, ks); sat0(ks);
        texref(A, moff, 2, &a, &ao, &b, &bo);
        color(a, ao, rf); sat0(rf); color(b, bo, tr); sat0(tr);
        texref(A, moff, 3, &a, &ao, &b, &bo);  // roughness, (isRemappingRoughness, 0)
        const float r = value(a, ao);
        const float al = std::fmax(b != 0 ? roughness_to_alpha(r) : r, 0.001f);
        m.flags = 0;
        if (!black(rf) || !black(tr)) {
          if (!black(kd)) m.flags |= (black(rf) ? 0 : 1) | (black(tr) ? 0 : 2);
          if (!black(ks)) m.flags |= (black(rf) ? 0 : 4) | (black(tr) ? 0 : 8);
        }
        for (int k = 0; k < 3; ++k) { m.c0[k] = kd[k] * rf[k]; m.c1[k] = kd[k] * tr[k]; m.c2[k] = ks[k] * rf[k]; m.c3[k] = ks[k] * tr[k]; }
        m.ax = m.ay = al;
        m.kind = m.flags ? kMatTranslucent : kMatNone;  // no lobe: no BSDF, the ray passes through
        break;
      }
      case kMatUberId: {  // UberMaterial.java; flags: 1 transparency BTDF, 2 Lambert, 4 TS BRDF, 8 specular BRDF, 16 specular BTDF
        float kd[3], kr[3], ks[3], kt[3], op[3];
        texref(A, moff, 1, &a, &ao, &b, &bo);
        color(a, ao, kd); sat0(kd); color(b, bo, kr); sat0(kr);
        texref(A, moff, 2, &a, &ao, &b, &bo);
        color(a, ao, ks); sat0(ks); color(b, bo, kt); sat0(kt);
        texref(A, moff, 3, &a, &ao, &b, &bo);
        m.eta = value(a, ao);
        color(b, bo, op); sat0(op);
        texref(A, moff, 4, &a, &ao, &b, &bo);
        const float ru = value(a, ao), rv = value(b, bo);
        const bool remap = plain(A, moff, 5) != 0;
        m.ax = std::fmax(remap ? roughness_to_alpha(ru) : ru, 0.001f);
        m.ay = std::fmax(remap ? roughness_to_alpha(rv) : rv, 0.001f);
        for (int k = 0; k < 3; ++k) {
          m.c0[k] = op[k] * kd[k]; m.c1[k] = op[k] * ks[k]; m.c2[k] = op[k] * kr[k]; m.c3[k] = op[k] * kt[k];
          m.c4[k] = std::fmax(1.0f - op[k], 0.0f);
        }
        m.flags = (black(m.c4) ? 0 : 1) | (black(m.c0) ? 0 : 2) | (black(m.c1) ? 0 : 4) | (black(m.c2) ? 0 : 8) | (black(m.c3) ? 0 : 16);
        m.kind = kMatUber;
        break;
      }
      case kMatDisneyId: {  // DisneyMaterial.java:1121-1210; record slots CompiledMaterialCache.java:2751-2759
        int ida, offa, idb, offb;
        auto f1 = [&](int slot, bool second) {
          texref(A, moff, slot, &ida, &offa, &idb, &offb);
          return second ? value(idb, offb) : value(ida, offa);
        };
        const float aniso = f1(1, false), cc = f1(2, false), ccg = f1(2, true);
        texref(A, moff, 3, &ida, &offa, &idb, &offb);
        float color[3];
        this->color(ida, offa, color);
        sat0(color);
        const float dt = value(idb, offb) / 2.0f;
        const float eta = f1(4, false), flat = f1(4, true), met = f1(5, false), rough = f1(5, true);
        texref(A, moff, 6, &ida, &offa, &idb, &offb);
        float sd[3];
        this->color(ida, offa, sd);
        const float sheen = value(idb, offb);
        const float sheen_tint = f1(7, false), spec_tint = f1(7, true);
        texref(A, moff, 8, &ida, &offa, &idb, &offb);
        const float st = value(ida, offa);
        const bool thin = idb != 0;  // second pair of slot 8: (isThin, 0)
        auto lerp = [](float a, float b, float t) { return (1.0f - t) * a + t * b; };  // utility/Floats.java:591
        const float lum = color[0] * 0.212671f + color[1] * 0.715160f + color[2] * 0.072169f;
        float tint[3];
        for (int k = 0; k < 3; ++k) tint[k] = lum > 0.0f ? color[k] / lum : 1.0f;
        m.kind = kMatDisney;
        m.flags = (thin ? kDisneyThin : 0) | (black(sd) ? 0 : kDisneyScatter) | (sheen > 0.0f ? kDisneyHasSheen : 0) |
                  (cc > 0.0f ? kDisneyHasClearCoat : 0) | (st > 0.0f ? kDisneyHasTransmission : 0);
        m.eta = eta;
        m.d_rough = rough;
        m.d_met = met;
        m.d_dw = (1.0f - met) * (1.0f - st);
        m.c2[0] = flat; m.c2[1] = dt; m.c2[2] = st;
        const float r0 = ((eta - 1.0f) * (eta - 1.0f)) / ((eta + 1.0f) * (eta + 1.0f));
        for (int k = 0; k < 3; ++k) {
          m.c0[k] = color[k];
          m.c1[k] = lerp(lerp(1.0f, tint[k], spec_tint) * r0, color[k], met);
          m.c3[k] = sheen > 0.0f ? lerp(1.0f, tint[k], sheen_tint) * (m.d_dw * sheen) : 0.0f;
          m.c4[k] = std::sqrt(color[k]) * st;
        }
        const float aspect = std::sqrt(1.0f - aniso * 0.9f);
        m.ax = std::fmax(0.001f, rough * rough / aspect);
        m.ay = std::fmax(0.001f, rough * rough * aspect);
        const float rs = (0.65f * eta - 0.35f) * rough;
        m.on_a = std::fmax(0.001f, rs * rs / aspect);
        m.on_b = std::fmax(0.001f, rs * rs * aspect);
        m.d_cc = cc;
        m.d_gloss = lerp(0.1f, 0.001f, ccg);
        break;
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
  void validate_distribution1(const std::vector<float>& A, size_t off) {
    if (off + 4 > A.size()) throw Fail{DFC_E_INVALID_ARG, "distribution out of range"};
    const float len = A[off], cdf = A[off + 1], cnt = A[off + 2];
    if (!(cnt >= 1.0f && cdf == cnt + 1.0f && len == 4.0f + cdf + cnt) || off + (size_t)len > A.size())
      throw Fail{DFC_E_INVALID_ARG, "malformed Distribution1F"};
  }
  void validate_distribution2(const std::vector<float>& A, size_t base) {
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
    hs.rects = R;
    // the record-sized shapes share one float pool on the device
    for (RecordArray& ra : record_arrays) {
      ra.base = hs.shapes.size();
      const auto& A = F(ra.name);
      hs.shapes.insert(hs.shapes.end(), A.begin(), A.end());
    }
    if (hs.shapes.empty()) hs.shapes.assign(4, 0.0f);
    hs.perez = F("lightPerezLightArray");  // the sky pool: Perez records, then image light records
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
            std::vector<int> offs;
            mesh_triangles(soff, offs);
            for (int to : offs)
              if (to < 0 || to % 24 != 0 || (size_t)to + 24 > T.size()) throw Fail{DFC_E_INVALID_ARG, "mesh triangle offset out of range"};
            if (offs.empty()) throw Fail{DFC_E_INVALID_ARG, "empty triangle mesh"};
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
    if (!tlas_boxes.empty()) {
      std::vector<int> order;
      hs.tlas_root = build_bvh4(tlas_boxes, 4, hs.nodes, order);
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
    if (hs.tri_pos.empty()) hs.tri_pos.assign(3, F4{0, 0, 0, 0});
    if (hs.nodes.empty()) hs.nodes.push_back(BVH4Node{});
    if (hs.lights.empty()) { DLight z; std::memset(&z, 0, sizeof z); hs.lights_storage_pad = 1; hs.lights.push_back(z); }
    if (hs.materials.empty()) { DMaterial z; std::memset(&z, 0, sizeof z); hs.materials.push_back(z); }
  }
};

}  // namespace

int ingest_scene(Staged& st, int layout, HostScene* out, std::string* err) {
  try {
    if (layout != 1 && layout != 2) throw Fail{DFC_E_INVALID_ARG, "layout_version must be 1 or 2"};
    HostScene hs;
    Decoder d(st, layout, hs);
    d.run();
    // the triangle records go to the device as they are: take them over
    auto tri = st.f32.find("shape3FTriangle3FArray");
    if (tri != st.f32.end()) hs.tri_attr = std::move(tri->second);
    if (hs.tri_attr.empty()) hs.tri_attr.assign(24, 0.0f);
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
