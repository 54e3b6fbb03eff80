// Material constants from texture values: the part of each reference
// material's computeScatteringFunctions that does not depend on the
// directions (scene/material/*Material.java).  Ingest runs it once for
// materials whose textures are all constant; the shading kernels run it per
// hit for materials with other textures (kMatTextured), after evaluating them.
#pragma once

#include <math.h>

#include "dfc_scene.h"

#ifdef __CUDACC__
#define DFC_HD __host__ __device__ inline
#else
#define DFC_HD inline
#endif

namespace dfc {

// Reference material ids (scene/material/*Material.java ID).
enum : int {
  kRefBullseye = 1, kRefCheckerboard = 2, kRefClearCoat = 3, kRefDisney = 4, kRefGlass = 7, kRefGlossy = 8, kRefMatte = 11,
  kRefMetal = 12, kRefMirror = 13, kRefPlastic = 14, kRefPolkaDot = 15, kRefSubstrate = 16, kRefTranslucent = 18, kRefUber = 19
};

// Where a record's textures and its plain int sit.  Texture position 2s is
// texture A of packed slot s, 2s + 1 texture B; position 1 is the modifier.
struct MatShape {
  unsigned tex_mask;  // texture positions
  int plain_slot;     // record slot holding a plain int (roughness remapping), -1 if none
  int plain_pos;      // texture position holding a plain int in its id lane (isRemappingRoughness, isThin), -1 if none
};
DFC_HD MatShape mat_shape(int ref_id) {
  switch (ref_id) {
    case kRefMatte: return {0x0Du, -1, -1};           // emission, angle, KD
    case kRefMirror: return {0x05u, -1, -1};          // emission, KR
    case kRefGlass: return {0xF5u, 4, -1};            // emission, eta, KR, KT, roughness U, V
    case kRefMetal: return {0x3Du, 3, -1};            // emission, eta, K, roughness U, V
    case kRefPlastic: return {0x1Du, 3, -1};          // emission, KD, KS, roughness
    case kRefClearCoat: return {0x0Du, -1, -1};       // emission, KD, KS
    case kRefGlossy: return {0x0Du, -1, -1};          // emission, KR, roughness
    case kRefSubstrate: return {0x3Du, 3, -1};        // emission, KD, KS, roughness U, V
    case kRefTranslucent: return {0x7Du, -1, 7};      // emission, KD, KS, reflectance, transmittance, roughness
    case kRefUber: return {0x3FDu, 5, -1};            // emission, KD, KR, KS, KT, eta, opacity, roughness U, V
    case kRefDisney: return {0x1FFF5u, -1, 17};       // emission, anisotropic, clear coat (2), colour, ..., specular transmission
    default: return {0u, -1, -1};
  }
}

struct MatInputs {
  float c[kTexPositions][3];  // texture colour per position
  int plain;
};

DFC_HD float md_avg(const float* c) { return (c[0] + c[1] + c[2]) / 3.0f; }  // Texture.getFloat: Color3F.average
DFC_HD float md_lerp(float a, float b, float t) { return (1.0f - t) * a + t * b; }  // utility/Floats.java:591
DFC_HD bool md_black(const float* c) { return c[0] == 0.0f && c[1] == 0.0f && c[2] == 0.0f; }
DFC_HD void md_sat0(float* d, const float* c) { for (int k = 0; k < 3; ++k) d[k] = fmaxf(c[k], 0.0f); }
DFC_HD float md_roughness_to_alpha(float r) {  // scene/microfacet/MicrofacetDistribution.java:convertRoughnessToAlpha
  const float x = fmaxf(r, 1.0e-3f), y = logf(x);
  return 1.62142f + 0.819955f * y + 0.1734f * y * y + 0.0171201f * y * y * y + 0.000640711f * y * y * y * y;
}

// Fills every DMaterial field the BSDF builders read.  `m` is zeroed first.
DFC_HD void derive_material(int ref_id, const MatInputs& in, DMaterial* m) {
  *m = DMaterial{};
  const float (*c)[3] = in.c;
  for (int k = 0; k < 3; ++k) m->emission[k] = c[0][k];
  switch (ref_id) {
    case kRefMatte: {  // MatteMaterial.java:285
      md_sat0(m->c0, c[3]);
      const float ang = fminf(fmaxf(md_avg(c[2]), 0.0f), 90.0f) * (3.14159265358979323846f / 180.0f);
      if (ang == 0.0f) {
        m->kind = kMatLambert;
      } else {
        m->kind = kMatOrenNayar;
        const float s2 = ang * ang;
        m->on_a = 1.0f - (s2 / (2.0f * (s2 + 0.33f)));
        m->on_b = 0.45f * s2 / (s2 + 0.09f);
      }
      break;
    }
    case kRefMirror:  // MirrorMaterial.java:235
      md_sat0(m->c0, c[2]);
      m->kind = md_black(m->c0) ? kMatNone : kMatMirror;
      break;
    case kRefGlass: {  // GlassMaterial.java:501
      m->eta = md_avg(c[2]);
      md_sat0(m->c0, c[4]);
      md_sat0(m->c1, c[5]);
      const float ru = md_avg(c[6]), rv = md_avg(c[7]);
      const bool remap = in.plain != 0;
      m->has_kr = !md_black(m->c0);
      m->has_kt = !md_black(m->c1);
      if (!m->has_kr && !m->has_kt) {
        m->kind = kMatNone;
      } else if (ru == 0.0f && rv == 0.0f) {
        m->kind = kMatGlassSpec;
      } else {
        m->kind = kMatGlassRough;
        m->ax = remap ? md_roughness_to_alpha(ru) : ru;
        m->ay = remap ? md_roughness_to_alpha(rv) : rv;
      }
      break;
    }
    case kRefMetal: {  // MetalMaterial.java:436
      for (int k = 0; k < 3; ++k) { m->c1[k] = c[2][k]; m->c2[k] = c[3][k]; }
      const float ru = md_avg(c[4]), rv = md_avg(c[5]);
      const bool remap = in.plain != 0;
      m->ax = remap ? md_roughness_to_alpha(ru) : ru;
      m->ay = remap ? md_roughness_to_alpha(rv) : rv;
      m->kind = kMatMetal;
      break;
    }
    case kRefPlastic: {  // PlasticMaterial.java:389
      md_sat0(m->c0, c[2]);
      md_sat0(m->c1, c[3]);
      const float r = md_avg(c[4]);
      m->ax = m->ay = in.plain != 0 ? md_roughness_to_alpha(r) : r;
      m->has_kr = !md_black(m->c0);
      m->has_kt = !md_black(m->c1);
      m->kind = (m->has_kr || m->has_kt) ? kMatPlastic : kMatNone;
      break;
    }
    case kRefClearCoat:  // ClearCoatMaterial.java: kd, ks (the lobe is chosen per hit)
      for (int k = 0; k < 3; ++k) { m->c0[k] = c[2][k]; m->c1[k] = c[3][k]; }
      m->kind = kMatClearCoat;
      break;
    case kRefGlossy: {  // GlossyMaterial.java: TorranceSparrowBRDF(kr, ConductorFresnel(kr, 1, 1), TR(r, r))
      for (int k = 0; k < 3; ++k) m->c0[k] = c[2][k];
      const float r = md_avg(c[3]);
      m->ax = m->ay = fmaxf(r, 0.001f);
      // ConductorFresnel with etaI = kr, etaT = k = 1: relative eta and k are 1 / kr
      for (int k = 0; k < 3; ++k) { m->c1[k] = 1.0f / m->c0[k]; m->c2[k] = 1.0f / m->c0[k]; }
      m->kind = kMatGlossy;
      break;
    }
    case kRefSubstrate: {  // SubstrateMaterial.java: FresnelBlendBRDF(kd, ks, TR(ru, rv))
      md_sat0(m->c0, c[2]);
      md_sat0(m->c1, c[3]);
      const float ru = md_avg(c[4]), rv = md_avg(c[5]);
      const bool remap = in.plain != 0;
      m->ax = fmaxf(remap ? md_roughness_to_alpha(ru) : ru, 0.001f);
      m->ay = fmaxf(remap ? md_roughness_to_alpha(rv) : rv, 0.001f);
      m->kind = (md_black(m->c0) && md_black(m->c1)) ? kMatNone : kMatSubstrate;
      break;
    }
    case kRefTranslucent: {  // TranslucentMaterial.java; flags: 1 Lambert BRDF, 2 Lambert BTDF, 4 TS BRDF, 8 TS BTDF
      float kd[3], ks[3], rf[3], tr[3];
      md_sat0(kd, c[2]);
      md_sat0(ks, c[3]);
      md_sat0(rf, c[4]);
      md_sat0(tr, c[5]);
      const float r = md_avg(c[6]);
      const float al = fmaxf(in.plain != 0 ? md_roughness_to_alpha(r) : r, 0.001f);
      m->flags = 0;
      if (!md_black(rf) || !md_black(tr)) {
        if (!md_black(kd)) m->flags |= (md_black(rf) ? 0 : 1) | (md_black(tr) ? 0 : 2);
        if (!md_black(ks)) m->flags |= (md_black(rf) ? 0 : 4) | (md_black(tr) ? 0 : 8);
      }
      for (int k = 0; k < 3; ++k) {
        m->c0[k] = kd[k] * rf[k]; m->c1[k] = kd[k] * tr[k]; m->c2[k] = ks[k] * rf[k]; m->c3[k] = ks[k] * tr[k];
      }
      m->ax = m->ay = al;
      m->kind = m->flags ? kMatTranslucent : kMatNone;  // no lobe: no BSDF, the ray passes through
      break;
    }
    case kRefUber: {  // UberMaterial.java; flags: 1 transparency BTDF, 2 Lambert, 4 TS BRDF, 8 specular BRDF, 16 specular BTDF
      float kd[3], kr[3], ks[3], kt[3], op[3];
      md_sat0(kd, c[2]);
      md_sat0(kr, c[3]);
      md_sat0(ks, c[4]);
      md_sat0(kt, c[5]);
      m->eta = md_avg(c[6]);
      md_sat0(op, c[7]);
      const float ru = md_avg(c[8]), rv = md_avg(c[9]);
      const bool remap = in.plain != 0;
      m->ax = fmaxf(remap ? md_roughness_to_alpha(ru) : ru, 0.001f);
      m->ay = fmaxf(remap ? md_roughness_to_alpha(rv) : rv, 0.001f);
      for (int k = 0; k < 3; ++k) {
        m->c0[k] = op[k] * kd[k]; m->c1[k] = op[k] * ks[k]; m->c2[k] = op[k] * kr[k]; m->c3[k] = op[k] * kt[k];
        m->c4[k] = fmaxf(1.0f - op[k], 0.0f);
      }
      m->flags = (md_black(m->c4) ? 0 : 1) | (md_black(m->c0) ? 0 : 2) | (md_black(m->c1) ? 0 : 4) | (md_black(m->c2) ? 0 : 8) |
                 (md_black(m->c3) ? 0 : 16);
      m->kind = kMatUber;
      break;
    }
    case kRefDisney: {  // DisneyMaterial.java:1121-1210; record slots CompiledMaterialCache.java:2751-2759
      const float aniso = md_avg(c[2]), cc = md_avg(c[4]), ccg = md_avg(c[5]);
      float color[3];
      md_sat0(color, c[6]);
      const float dt = md_avg(c[7]) / 2.0f;
      const float eta = md_avg(c[8]), flat = md_avg(c[9]), met = md_avg(c[10]), rough = md_avg(c[11]);
      const float* sd = c[12];
      const float sheen = md_avg(c[13]), sheen_tint = md_avg(c[14]), spec_tint = md_avg(c[15]), st = md_avg(c[16]);
      const bool thin = in.plain != 0;  // second pair of slot 8: (isThin, 0)
      const float lum = color[0] * 0.212671f + color[1] * 0.715160f + color[2] * 0.072169f;
      float tint[3];
      for (int k = 0; k < 3; ++k) tint[k] = lum > 0.0f ? color[k] / lum : 1.0f;
      m->kind = kMatDisney;
      m->flags = (thin ? kDisneyThin : 0) | (md_black(sd) ? 0 : kDisneyScatter) | (sheen > 0.0f ? kDisneyHasSheen : 0) |
                 (cc > 0.0f ? kDisneyHasClearCoat : 0) | (st > 0.0f ? kDisneyHasTransmission : 0);
      m->eta = eta;
      m->d_rough = rough;
      m->d_met = met;
      m->d_dw = (1.0f - met) * (1.0f - st);
      m->c2[0] = flat; m->c2[1] = dt; m->c2[2] = st;
      const float r0 = ((eta - 1.0f) * (eta - 1.0f)) / ((eta + 1.0f) * (eta + 1.0f));
      for (int k = 0; k < 3; ++k) {
        m->c0[k] = color[k];
        m->c1[k] = md_lerp(md_lerp(1.0f, tint[k], spec_tint) * r0, color[k], met);
        m->c3[k] = sheen > 0.0f ? md_lerp(1.0f, tint[k], sheen_tint) * (m->d_dw * sheen) : 0.0f;
        m->c4[k] = sqrtf(color[k]) * st;
      }
      const float aspect = sqrtf(1.0f - aniso * 0.9f);
      m->ax = fmaxf(0.001f, rough * rough / aspect);
      m->ay = fmaxf(0.001f, rough * rough * aspect);
      const float rs = (0.65f * eta - 0.35f) * rough;
      m->on_a = fmaxf(0.001f, rs * rs / aspect);
      m->on_b = fmaxf(0.001f, rs * rs * aspect);
      m->d_cc = cc;
      m->d_gloss = md_lerp(0.1f, 0.001f, ccg);
      break;
    }
    default:
      m->kind = kMatNone;
      break;
  }
}

}  // namespace dfc
