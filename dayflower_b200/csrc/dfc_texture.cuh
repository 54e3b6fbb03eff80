// Per-hit material evaluation for materials with non-constant textures,
// modifiers, or composite (Bullseye / Checkerboard / PolkaDot) selection.
//
// The reference evaluates every texture per hit (renderer/gpu/
// AbstractTextureKernel.java:152-435 on its GPU path, scene/texture/*.java
// getColor on the CPU path this file follows).  Here only materials that need
// it take this path: ingest resolves all-constant materials to DMaterial
// constants, so the common case costs nothing.  The evaluation runs in
// __noinline__ functions to keep the shading kernels' register allocation
// independent of it.
#pragma once

#include "dfc_device.cuh"
#include "dfc_matderive.h"

namespace dfc {

// ------------------------------------------------------------------ noise --
// noise/PerlinNoiseF.java and noise/SimplexNoiseF.java.  The permutation is
// Ken Perlin's published table as the reference holds it (entry 156 is 23,
// not 223).
__device__ const unsigned char kNoisePerm[256] = {
    151, 160, 137, 91,  90,  15,  131, 13,  201, 95,  96,  53,  194, 233, 7,   225, 140, 36,  103, 30,  69,  142, 8,   99,
    37,  240, 21,  10,  23,  190, 6,   148, 247, 120, 234, 75,  0,   26,  197, 62,  94,  252, 219, 203, 117, 35,  11,  32,
    57,  177, 33,  88,  237, 149, 56,  87,  174, 20,  125, 136, 171, 168, 68,  175, 74,  165, 71,  134, 139, 48,  27,  166,
    77,  146, 158, 231, 83,  111, 229, 122, 60,  211, 133, 230, 220, 105, 92,  41,  55,  46,  245, 40,  244, 102, 143, 54,
    65,  25,  63,  161, 1,   216, 80,  73,  209, 76,  132, 187, 208, 89,  18,  169, 200, 196, 135, 130, 116, 188, 159, 86,
    164, 100, 109, 198, 173, 186, 3,   64,  52,  217, 226, 250, 124, 123, 5,   202, 38,  147, 118, 126, 255, 82,  85,  212,
    207, 206, 59,  227, 47,  16,  58,  17,  182, 189, 28,  42,  23,  183, 170, 213, 119, 248, 152, 2,   44,  154, 163, 70,
    221, 153, 101, 155, 167, 43,  172, 9,   129, 22,  39,  253, 19,  98,  108, 110, 79,  113, 224, 232, 178, 185, 112, 104,
    218, 246, 97,  228, 251, 34,  242, 193, 238, 210, 144, 12,  191, 179, 162, 241, 81,  51,  145, 235, 249, 14,  239, 107,
    49,  192, 214, 31,  181, 199, 106, 157, 184, 84,  204, 176, 115, 121, 50,  45,  127, 4,   150, 254, 138, 236, 205, 93,
    222, 114, 67,  29,  24,  72,  243, 141, 128, 195, 78,  66,  215, 61,  156, 180};

DFC_D int nperm(int i) { return (int)kNoisePerm[i & 255]; }

DFC_D float noise_grad(int h, float x, float y, float z) {
  const float u = (h < 8 || h == 12 || h == 13) ? x : y;
  const float v = (h < 4 || h == 12 || h == 13) ? y : z;
  return ((h & 1) == 0 ? u : -u) + ((h & 2) == 0 ? v : -v);
}

// PerlinNoiseF.noiseXYZ: quintic fade, eight hashed corner gradients, trilinear blend
DFC_D float perlin3(float x, float y, float z) {
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) return 0.0f;
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
  const float x1 = x - fx, y1 = y - fy, z1 = z - fz;
  const float u = x1 * x1 * x1 * (x1 * (x1 * 6.0f - 15.0f) + 10.0f);
  const float v = y1 * y1 * y1 * (y1 * (y1 * 6.0f - 15.0f) + 10.0f);
  const float w = z1 * z1 * z1 * (z1 * (z1 * 6.0f - 15.0f) + 10.0f);
  const int a0 = nperm(X) + Y, a1 = nperm(a0) + Z, a2 = nperm(a0 + 1) + Z;
  const int b0 = nperm(X + 1) + Y, b1 = nperm(b0) + Z, b2 = nperm(b0 + 1) + Z;
  const float g0 = noise_grad(nperm(a1) & 15, x1, y1, z1), g1 = noise_grad(nperm(b1) & 15, x1 - 1.0f, y1, z1);
  const float g2 = noise_grad(nperm(a2) & 15, x1, y1 - 1.0f, z1), g3 = noise_grad(nperm(b2) & 15, x1 - 1.0f, y1 - 1.0f, z1);
  const float g4 = noise_grad(nperm(a1 + 1) & 15, x1, y1, z1 - 1.0f), g5 = noise_grad(nperm(b1 + 1) & 15, x1 - 1.0f, y1, z1 - 1.0f);
  const float g6 = noise_grad(nperm(a2 + 1) & 15, x1, y1 - 1.0f, z1 - 1.0f);
  const float g7 = noise_grad(nperm(b2 + 1) & 15, x1 - 1.0f, y1 - 1.0f, z1 - 1.0f);
  const float l0 = g0 + u * (g1 - g0), l1 = g2 + u * (g3 - g2), l2 = g4 + u * (g5 - g4), l3 = g6 + u * (g7 - g6);
  const float l4 = l0 + v * (l1 - l0), l5 = l2 + v * (l3 - l2);
  return fminf(fmaxf(l4 + w * (l5 - l4), -1.0f), 1.0f);
}

// PerlinNoiseF.turbulenceXYZ(x, y, z, octaves)
DFC_D float perlin_turbulence(float x, float y, float z, int octaves) {
  float n = fabsf(perlin3(x, y, z)), wgt = 1.0f;
  for (int i = 1; i < octaves; ++i) {
    wgt *= 2.0f;
    n += fabsf(perlin3(x * wgt, y * wgt, z * wgt)) / wgt;
  }
  return n;
}

// SimplexNoiseF.noiseXYZ (Gustavson's 3D simplex noise)
DFC_D float simplex3(float x, float y, float z) {
  if (!isfinite(x) || !isfinite(y) || !isfinite(z)) return 0.0f;
  const float F3 = 1.0f / 3.0f, G3 = 1.0f / 6.0f;
  const float s = (x + y + z) * F3;
  auto ffloor = [](float f) { const int i = (int)f; return f < (float)i ? i - 1 : i; };
  const int i = ffloor(x + s), j = ffloor(y + s), k = ffloor(z + s);
  const float t = (float)(i + j + k) * G3;
  const float x0 = x - ((float)i - t), y0 = y - ((float)j - t), z0 = z - ((float)k - t);
  int i1, j1, k1, i2, j2, k2;
  if (x0 >= y0) {
    if (y0 >= z0) { i1 = 1; j1 = 0; k1 = 0; i2 = 1; j2 = 1; k2 = 0; }
    else if (x0 >= z0) { i1 = 1; j1 = 0; k1 = 0; i2 = 1; j2 = 0; k2 = 1; }
    else { i1 = 0; j1 = 0; k1 = 1; i2 = 1; j2 = 0; k2 = 1; }
  } else {
    if (y0 < z0) { i1 = 0; j1 = 0; k1 = 1; i2 = 0; j2 = 1; k2 = 1; }
    else if (x0 < z0) { i1 = 0; j1 = 1; k1 = 0; i2 = 0; j2 = 1; k2 = 1; }
    else { i1 = 0; j1 = 1; k1 = 0; i2 = 1; j2 = 1; k2 = 0; }
  }
  const int ii = i & 255, jj = j & 255, kk = k & 255;
  float n = 0.0f;
  for (int q = 0; q < 4; ++q) {
    const int di = q == 0 ? 0 : (q == 1 ? i1 : (q == 2 ? i2 : 1));
    const int dj = q == 0 ? 0 : (q == 1 ? j1 : (q == 2 ? j2 : 1));
    const int dk = q == 0 ? 0 : (q == 1 ? k1 : (q == 2 ? k2 : 1));
    const float cx = q == 0 ? x0 : (q == 3 ? x0 - 1.0f + 3.0f * G3 : x0 - di + (float)q * G3);
    const float cy = q == 0 ? y0 : (q == 3 ? y0 - 1.0f + 3.0f * G3 : y0 - dj + (float)q * G3);
    const float cz = q == 0 ? z0 : (q == 3 ? z0 - 1.0f + 3.0f * G3 : z0 - dk + (float)q * G3);
    const float tq = 0.6f - cx * cx - cy * cy - cz * cz;
    if (tq < 0.0f) continue;
    const int g = nperm(ii + di + nperm(jj + dj + nperm(kk + dk))) % 12;
    // the twelve edge directions of SimplexNoiseF's gradient table
    const float gx = g < 4 ? ((g & 1) ? -1.0f : 1.0f) : (g < 8 ? ((g & 1) ? -1.0f : 1.0f) : 0.0f);
    const float gy = g < 4 ? ((g & 2) ? -1.0f : 1.0f) : (g < 8 ? 0.0f : ((g & 1) ? -1.0f : 1.0f));
    const float gz = g < 4 ? 0.0f : (g < 8 ? ((g & 2) ? -1.0f : 1.0f) : ((g & 2) ? -1.0f : 1.0f));
    n += (tq * tq) * (tq * tq) * (gx * cx + gy * cy + gz * cz);
  }
  return fminf(fmaxf(32.0f * n, -1.0f), 1.0f);
}

// SimplexNoiseF.fractionalBrownianMotionXYZ
DFC_D float simplex_fbm(float x, float y, float z, float frequency, float gain, float minimum, float maximum, int octaves) {
  float amp = 1.0f, amp_sum = 0.0f, f = frequency, n = 0.0f;
  for (int i = 0; i < octaves; ++i) {
    n += simplex3(x * f, y * f, z * f) * amp;
    amp_sum += amp;
    amp *= gain;
    f *= 2.0f;
  }
  n /= amp_sum;
  return n * (maximum - minimum) / 2.0f + (maximum + minimum) / 2.0f;
}

// --------------------------------------------------------------- textures --
// What a texture sees of the hit: world point, object-space point, shading
// normal (after the material's modifier), ray direction, texture coordinates.
struct TexCtx { V3 p, p_obj, ns, d; float u, v; };

DFC_D float tx_frac(float x) { return x - floorf(x); }  // Floats.fractionalPart(x, false)
DFC_D float tx_posmod(float x, float y) { return x < 0.0f ? fmodf(fmodf(x, y) + y, y) : fmodf(x, y); }  // Floats.positiveModulo
DFC_D int tx_posmod_i(int x, int y) { return x < 0 ? (x % y + y) % y : x % y; }
DFC_D V3 tx_argb(unsigned c) {
  return {(float)((c >> 16) & 0xFFu) / 255.0f, (float)((c >> 8) & 0xFFu) / 255.0f, (float)(c & 0xFFu) / 255.0f};
}
DFC_D V3 tx_lerp(V3 a, V3 b, V3 t) {
  return {(1.0f - t.x) * a.x + t.x * b.x, (1.0f - t.y) * a.y + t.y * b.y, (1.0f - t.z) * a.z + t.z * b.z};
}
// Point2F.rotateCounterclockwise, Point2F.scale, Point2F.toImage
DFC_D void tx_image_point(float cs, float sn, float su, float sv, int rx, int ry, float u, float v, float* x, float* y) {
  const float ru = u * cs - v * sn, rv = v * cs + u * sn;
  *x = tx_posmod(ru * su * (float)rx - 0.5f, (float)rx);
  *y = tx_posmod(rv * sv * (float)ry - 0.5f, (float)ry);
}
DFC_D V3 tx_texel(const unsigned* px, int rx, int ry, int x, int y) {
  return tx_argb(__ldg(px + tx_posmod_i(y, ry) * rx + tx_posmod_i(x, rx)));
}

// Texture.getColor for one node; pattern textures walk to the chosen child,
// BlendTexture evaluates both children (nesting bounded by D).
template <int D>
static __device__ __noinline__ V3 tex_eval(const SceneView& S, int node, const TexCtx& c) {
  for (int guard = 0; guard < 64 && node >= 0; ++guard) {
    const DTexture& t = S.textures[node];
    switch (t.kind) {
      case kTexConstant: return {t.p[0], t.p[1], t.p[2]};
      case kTexBlend:
        if constexpr (D > 0) return tx_lerp(tex_eval<D - 1>(S, t.a, c), tex_eval<D - 1>(S, t.b, c), V3{t.p[0], t.p[1], t.p[2]});
        else return {0.5f, 0.5f, 0.5f};
      case kTexBullseye: {  // object-space distance to the origin, fractional part above 0.5 picks A
        const V3 dv = c.p_obj - V3{t.p[0], t.p[1], t.p[2]};
        node = fmodf(len(dv) * t.p[3], 1.0f) > 0.5f ? t.a : t.b;
        continue;
      }
      case kTexCheckerboard: {
        const bool iu = tx_frac((c.u * t.p[0] - c.v * t.p[1]) * t.p[2]) > 0.5f;
        const bool iv = tx_frac((c.v * t.p[0] + c.u * t.p[1]) * t.p[3]) > 0.5f;
        node = (iu ^ iv) ? t.a : t.b;
        continue;
      }
      case kTexPolkaDot: {
        const float x = tx_frac((c.u * t.p[0] - c.v * t.p[1]) * t.p[2]) - 0.5f;
        const float y = tx_frac((c.v * t.p[0] + c.u * t.p[1]) * t.p[2]) - 0.5f;
        node = x * x + y * y < t.p[3] * t.p[3] ? t.a : t.b;
        continue;
      }
      case kTexDotProduct: {
        const float d = fabsf(dot(c.ns, c.d));
        return {d, d, d};
      }
      case kTexLDRImage: {  // LDRImageTexture: bilinear over wrapped texels (one texel when x, y are integral)
        float x, y;
        tx_image_point(t.p[0], t.p[1], t.p[2], t.p[3], t.a, t.b, c.u, c.v, &x, &y);
        const unsigned* px = S.texels + t.c;
        const int x0 = (int)floorf(x), x1 = (int)ceilf(x), y0 = (int)floorf(y), y1 = (int)ceilf(y);
        if (x0 == x1 && y0 == y1) return tx_texel(px, t.a, t.b, x0, y0);
        const float tx = x - (float)x0, ty = y - (float)y0;
        const V3 t3{tx, tx, tx}, s3{ty, ty, ty};
        return tx_lerp(tx_lerp(tx_texel(px, t.a, t.b, x0, y0), tx_texel(px, t.a, t.b, x1, y0), t3),
                       tx_lerp(tx_texel(px, t.a, t.b, x0, y1), tx_texel(px, t.a, t.b, x1, y1), t3), s3);
      }
      case kTexMarble: {  // MarbleTexture.getColor
        const float x = c.p.x * t.p[9], y = c.p.y * t.p[9], z = c.p.z * t.p[9];
        const float r = t.p[10] * perlin_turbulence(x, y, z, t.a);
        const float s = 2.0f * fabsf((float)sin((double)(x + r)));
        const float tt = s < 1.0f ? s : s - 1.0f;
        const V3 ca{t.p[0], t.p[1], t.p[2]}, cb{t.p[3], t.p[4], t.p[5]}, cc{t.p[6], t.p[7], t.p[8]};
        return tx_lerp(s < 1.0f ? cc : cb, s < 1.0f ? cb : ca, V3{tt, tt, tt});
      }
      case kTexSimplexFBM: {
        const float n = simplex_fbm(c.p.x, c.p.y, c.p.z, t.p[3], t.p[4], 0.0f, 1.0f, t.a);
        return V3{t.p[0], t.p[1], t.p[2]} * n;
      }
      case kTexSurfaceNormal: {
        const V3 n = dot(c.ns, c.d) > 0.0f ? -c.ns : c.ns;
        return {(n.x + 1.0f) / 2.0f, (n.y + 1.0f) / 2.0f, (n.z + 1.0f) / 2.0f};
      }
      case kTexUV: return {c.u, c.v, 0.0f};
      default: return {0.5f, 0.5f, 0.5f};
    }
  }
  return {0.5f, 0.5f, 0.5f};
}

// Intersection.setSurfaceNormalS: OrthonormalBasis33F(w = n, v = the old v)
DFC_D void set_normal_s(Surface* sf, V3 n) {
  const V3 w = normalize(n);
  const V3 u = normalize(cross(normalize(sf->s.v), w));
  sf->s.w = w;
  sf->s.u = u;
  sf->s.v = cross(w, u);
}

// Modifier.modify (scene/modifier/NormalMapLDRImageModifier.java, SimplexNoiseNormalMapModifier.java)
DFC_D void apply_modifier(const SceneView& S, int mi, Surface* sf) {
  const DModifier& m = S.modifiers[mi];
  if (m.kind == kModNormalMapLDRImage) {  // nearest texel, mapped through the geometric frame
    float x, y;
    tx_image_point(m.p[0], m.p[1], m.p[2], m.p[3], m.rx, m.ry, sf->tu, sf->tv, &x, &y);
    const V3 c = tx_texel(S.texels + m.texel, m.rx, m.ry, (int)x, (int)y);
    const V3 l{c.x * 2.0f - 1.0f, c.y * 2.0f - 1.0f, c.z * 2.0f - 1.0f};
    const ONB& g = sf->g;
    const V3 n{l.x * g.u.x + l.y * g.v.x + l.z * g.w.x, l.x * g.u.y + l.y * g.v.y + l.z * g.w.y, l.x * g.u.z + l.y * g.v.z + l.z * g.w.z};
    set_normal_s(sf, normalize(n));
  } else if (m.kind == kModSimplexNoiseNormalMap) {
    const float freq = m.p[0], scale = m.p[1], rf = 1.0f / freq;
    const V3 p = sf->p, n = sf->s.w;
    const float x0 = p.x * rf, y0 = p.y * rf, z0 = p.z * rf;
    const float x1 = n.x + simplex_fbm(x0, y0, z0, freq, 0.5f, -0.25f, 0.25f, 16) * scale;
    const float y1 = n.y + simplex_fbm(y0, z0, x0, freq, 0.5f, -0.25f, 0.25f, 16) * scale;
    const float z1 = n.z + simplex_fbm(z0, x0, y0, freq, 0.5f, -0.25f, 0.25f, 16) * scale;
    set_normal_s(sf, normalize(V3{x1, y1, z1}));
  }
}

// The material a composite picks at this hit (BullseyeMaterial / CheckerboardMaterial /
// PolkaDotMaterial.doGetMaterial, repeated while the pick is composite).
DFC_D int resolve_composite(const SceneView& S, int mat, V3 p_obj, float u, float v) {
  for (int guard = 0; guard < 64 && S.materials[mat].kind == kMatComposite; ++guard) {
    const DComposite& c = S.composites[S.materials[mat].flags];
    bool a;
    if (c.kind == kCompBullseye) {
      a = fmodf(len(p_obj - V3{c.p[0], c.p[1], c.p[2]}) * c.p[3], 1.0f) > 0.5f;
    } else if (c.kind == kCompCheckerboard) {
      a = (tx_frac((u * c.p[0] - v * c.p[1]) * c.p[2]) > 0.5f) ^ (tx_frac((v * c.p[0] + u * c.p[1]) * c.p[3]) > 0.5f);
    } else {
      const float x = tx_frac((u * c.p[0] - v * c.p[1]) * c.p[2]) - 0.5f, y = tx_frac((v * c.p[0] + u * c.p[1]) * c.p[2]) - 0.5f;
      a = x * x + y * y < c.p[3] * c.p[3];
    }
    mat = a ? c.a : c.b;
  }
  return mat;
}

DFC_D V3 object_point(const DPrim& pr, const Surface& sf) { return pr.identity ? sf.p : xf_point(pr.w2o, sf.p); }

// Material.computeScatteringFunctions up to the BSDF build for a kMatTextured
// material: modifier (changes the hit's shading frame for the rest of the
// bounce), texture evaluation at the modified hit, derivation of the constants.
static __device__ __noinline__ void eval_textured(const SceneView& S, int tm_index, V3 p_obj, V3 ray_d, Surface* sf, DMaterial* out) {
  const DTexMaterial& tm = S.texmats[tm_index];
  if (tm.modifier >= 0) apply_modifier(S, tm.modifier, sf);
  const TexCtx c{sf->p, p_obj, sf->s.w, ray_d, sf->tu, sf->tv};
  MatInputs in;
  for (int k = 0; k < kTexPositions; ++k) {
    const int n = tm.tex[k];
    const V3 col = n >= 0 ? tex_eval<kMaxBlendDepth>(S, n, c) : V3{0, 0, 0};
    in.c[k][0] = col.x; in.c[k][1] = col.y; in.c[k][2] = col.z;
  }
  in.plain = tm.plain;
  derive_material(tm.ref_id, in, out);
}

// build_bsdf for a kMatTextured or kMatComposite material: the composite
// picks its material, a textured material is evaluated (its modifier may
// change sf's shading frame, which the caller keeps for the rest of the
// bounce).  Out of line, so that the shading kernels' common path (constant
// materials, build_bsdf inline) keeps its register allocation.
static __device__ __noinline__ bool textured_bsdf(const SceneView& S, const DPrim& pr, V3 ray_d, float u_material, bool multi, Surface* sf,
                                           Bsdf* B) {
  int mat = pr.material;
  const V3 p_obj = object_point(pr, *sf);
  if (S.materials[mat].kind == kMatComposite) mat = resolve_composite(S, mat, p_obj, sf->tu, sf->tv);
  if (S.materials[mat].kind != kMatTextured) return build_bsdf(S.materials[mat], *sf, ray_d, u_material, B, multi);
  DMaterial m;
  eval_textured(S, S.materials[mat].flags, p_obj, ray_d, sf, &m);
  return build_bsdf(m, *sf, ray_d, u_material, B, multi);
}

// Material.emittance at this hit: the (picked) material's emission texture, on the unmodified hit.
static __device__ __noinline__ V3 hit_material_emission(const SceneView& S, const DPrim& pr, V3 ray_d, const Surface& sf) {
  int mat = pr.material;
  const V3 p_obj = object_point(pr, sf);
  if (S.materials[mat].kind == kMatComposite) mat = resolve_composite(S, mat, p_obj, sf.tu, sf.tv);
  const DMaterial& m = S.materials[mat];
  if (m.kind != kMatTextured) return ld3(m.emission);
  const DTexMaterial& tm = S.texmats[m.flags];
  if (tm.tex[0] < 0) return {0, 0, 0};
  const TexCtx c{sf.p, p_obj, sf.s.w, ray_d, sf.tu, sf.tv};
  return tex_eval<kMaxBlendDepth>(S, tm.tex[0], c);
}

// Material.emittance: constant materials from the table, others evaluated.
DFC_D V3 material_Le(const SceneView& S, const DPrim& pr, V3 ray_d, const Surface& sf) {
  const DMaterial& m = S.materials[pr.material];
  return m.kind < kMatTextured ? ld3(m.emission) : hit_material_emission(S, pr, ray_d, sf);
}

}  // namespace dfc
