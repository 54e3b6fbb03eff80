// Device math, sampling, intersection and shading routines of the render path.
// Each routine names the reference code whose semantics it implements (paths
// relative to src/main/java/org/dayflower/); the CPU renderer (CPURenderer)
// is the behaviour followed where it differs from the Aparapi kernel.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dfc_scene.h"

namespace dfc {

#define DFC_D __device__ __forceinline__

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTMin = 0.001f;  // scene/Scene.java:70
constexpr float kFltMax = 3.402823466e+38f;

// ---------------------------------------------------------------- vectors --
struct V3 { float x, y, z; };
DFC_D V3 v3(float x, float y, float z) { return V3{x, y, z}; }
DFC_D V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
DFC_D V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
DFC_D V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
DFC_D V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
DFC_D V3 mul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
DFC_D float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DFC_D V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
DFC_D float len(V3 a) { return sqrtf(dot(a, a)); }
DFC_D bool is_black(V3 c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
DFC_D V3 ld3(const float* p) { return {p[0], p[1], p[2]}; }
// geometry/Vector3F.java:1000: lengths within [nextDown^3(1), nextUp(1)] are kept.
DFC_D V3 normalize(V3 v) {
  const float l = len(v);
  if (l >= 0.99999982f && l <= 1.00000012f) return v;
  return V3{v.x / l, v.y / l, v.z / l};
}
DFC_D float clampf(float v, float a, float b) { return v < a ? a : (v > b ? b : v); }
DFC_D float luminance(V3 c) { return c.x * 0.212671f + c.y * 0.715160f + c.z * 0.072169f; }

// 3x4 row-major affine transforms (the top three rows of Matrix44F).
DFC_D V3 xf_point(const float* m, V3 p) {
  return {m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7], m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
}
DFC_D V3 xf_vec(const float* m, V3 v) {
  return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z, m[8] * v.x + m[9] * v.y + m[10] * v.z};
}
DFC_D V3 xf_vec_t(const float* m, V3 v) {  // transpose of the 3x3 part
  return {m[0] * v.x + m[4] * v.y + m[8] * v.z, m[1] * v.x + m[5] * v.y + m[9] * v.z, m[2] * v.x + m[6] * v.y + m[10] * v.z};
}

struct ONB { V3 u, v, w; };
DFC_D V3 compute_v(V3 w) {  // geometry/Vector3F.java:527
  V3 n = normalize(w);
  float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
  if (ax < ay && ax < az) return normalize(V3{0.0f, n.z, -n.y});
  if (ay < az) return normalize(V3{n.z, 0.0f, -n.x});
  return normalize(V3{n.y, -n.x, 0.0f});
}
DFC_D ONB onb_w(V3 w) { ONB o; o.w = normalize(w); o.v = compute_v(w); o.u = cross(o.v, o.w); return o; }  // OrthonormalBasis33F.java:88
DFC_D ONB onb_wv(V3 w, V3 v) {  // OrthonormalBasis33F.java:110
  ONB o; o.w = normalize(w); o.u = normalize(cross(normalize(v), o.w)); o.v = cross(o.w, o.u); return o;
}
DFC_D V3 to_local(V3 a, const ONB& b) { return {dot(a, b.u), dot(a, b.v), dot(a, b.w)}; }
DFC_D V3 to_world(V3 a, const ONB& b) { return b.u * a.x + b.v * a.y + b.w * a.z; }

// ------------------------------------------------------------ random numbers
// Counter-based: every draw is keyed by (seed, pixel, sample, dimension), so a
// sample gets the same numbers alone or batched with other work.
DFC_D uint32_t rng_hash(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16; return x;
}
DFC_D uint32_t rng_path_key(uint32_t seed, uint32_t pixel, uint32_t sample) {
  return rng_hash(seed ^ rng_hash(pixel ^ rng_hash(sample + 0x632be5abu)));
}
DFC_D float rng_uniform(uint32_t key, uint32_t dim) {
  return (float)(rng_hash(key + dim * 0x9e3779b9u) >> 8) * (1.0f / 16777216.0f);
}
enum : uint32_t {
  kDimPixelX = 0, kDimPixelY = 1, kDimLensU = 2, kDimLensV = 3, kDimBounceBase = 8, kDimBounceStride = 16,
  kDimLightPick = 0, kDimLightSampleU = 1, kDimLightSampleV = 2, kDimMisSampleU = 3, kDimMisSampleV = 4,
  kDimSunPick = 5, kDimBsdfU = 6, kDimBsdfV = 7, kDimRoulette = 8, kDimMaterial = 9,
};
DFC_D uint32_t bounce_dim(int b, uint32_t w) { return kDimBounceBase + (uint32_t)b * kDimBounceStride + w; }

// -------------------------------------------------------------- sampling --
DFC_D void concentric(float u, float v, float* x, float* y) {  // geometry/SampleGeneratorF.java:129
  if (u == 0.0f && v == 0.0f) { *x = 0.0f; *y = 0.0f; return; }
  float a = u * 2.0f - 1.0f, b = v * 2.0f - 1.0f;
  float r, phi;
  if (a * a > b * b) { r = a; phi = (kPi / 4.0f) * (b / a); }
  else { r = b; phi = (kPi / 2.0f) - (kPi / 4.0f) * (a / b); }
  float s, c;
  sincosf(phi, &s, &c);
  *x = r * c; *y = r * s;
}
DFC_D V3 cosine_hemisphere(float u, float v) {
  float x, y;
  concentric(u, v, &x, &y);
  return {x, y, sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y))};
}
DFC_D V3 uniform_hemisphere(float u, float v) {
  float st = sqrtf(fmaxf(0.0f, 1.0f - u * u)), s, c;
  sincosf(2.0f * kPi * v, &s, &c);
  return {st * c, st * s, u};
}

// ------------------------------------------------------------------ camera
// scene/Camera.java:243 createPrimaryRay over the 19-float compiled camera.
DFC_D bool camera_ray(const float* c, float ix, float iy, float px, float py, float lu, float lv, V3* o, V3* d) {
  const float cx = 2.0f * ((ix + px) / (c[17] - 1.0f)) - 1.0f;
  const float cy = 2.0f * ((iy + py) / (c[18] - 1.0f)) - 1.0f;
  float wf = 1.0f;
  if ((int)c[2] == 0) {  // Lens.FISHEYE
    float dp = cx * cx + cy * cy;
    if (dp > 1.0f) return false;
    wf = sqrtf(1.0f - dp);
  }
  V3 U = ld3(c + 3), Vv = ld3(c + 6), W = ld3(c + 9), eye = ld3(c + 12);
  V3 pp = (U * (c[0] * cx) + Vv * (c[1] * cy)) + (eye + W * wf);
  V3 pip = eye + normalize(pp - eye) * c[16];
  V3 org = eye;
  if (c[15] > 0.00001f) {
    float dx, dy;
    concentric(lu, lv, &dx, &dy);
    org = eye + (U * (dx * c[15]) + Vv * (dy * c[15]));
  }
  *o = org;
  *d = normalize(normalize(pip - org));
  return true;
}

// ---------------------------------------------------------- intersection --
DFC_D float gamma_n(int n) { const float e = 5.9604645e-8f; return (n * e) / (1.0f - n * e); }

// Double-precision edge functions (Triangle3F.java:537-546), taken only when a
// float edge function is exactly zero; kept out of line to keep the hot loop
// small, and returned by value so that the caller's edge values stay in
// registers (an address taken for an out-of-line call puts them in local memory).
struct Edges { float e0, e1, e2; };
static __device__ __noinline__ Edges tri_edges_fp64(float x0, float y0, float x1, float y1, float x2, float y2) {
  return Edges{(float)((double)y2 * (double)x1 - (double)x2 * (double)y1), (float)((double)y0 * (double)x2 - (double)x0 * (double)y2),
               (float)((double)y1 * (double)x0 - (double)x1 * (double)y0)};
}

// geometry/shape/Triangle3F.java:505 watertight test; returns -1 on a miss.
DFC_D float tri_t(V3 a, V3 b, V3 c, V3 o, V3 d, float tmin, float tmax) {
  V3 p0 = a - o, p1 = b - o, p2 = c - o;
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  // permutation (kx, ky, kz) = (kz+1, kz+2, kz) mod 3
  float dX, dY, dZ, x0, y0, z0, x1, y1, z1, x2, y2, z2;
  if (kz == 0) { dX = d.y; dY = d.z; dZ = d.x; x0 = p0.y; y0 = p0.z; z0 = p0.x; x1 = p1.y; y1 = p1.z; z1 = p1.x; x2 = p2.y; y2 = p2.z; z2 = p2.x; }
  else if (kz == 1) { dX = d.z; dY = d.x; dZ = d.y; x0 = p0.z; y0 = p0.x; z0 = p0.y; x1 = p1.z; y1 = p1.x; z1 = p1.y; x2 = p2.z; y2 = p2.x; z2 = p2.y; }
  else { dX = d.x; dY = d.y; dZ = d.z; x0 = p0.x; y0 = p0.y; z0 = p0.z; x1 = p1.x; y1 = p1.y; z1 = p1.z; x2 = p2.x; y2 = p2.y; z2 = p2.z; }
  const float sx = -dX / dZ, sy = -dY / dZ, sz = 1.0f / dZ;
  x0 = x0 + sx * z0; y0 = y0 + sy * z0;
  x1 = x1 + sx * z1; y1 = y1 + sy * z1;
  x2 = x2 + sx * z2; y2 = y2 + sy * z2;
  float e0 = x1 * y2 - y1 * x2;
  float e1 = x2 * y0 - y2 * x0;
  float e2 = x0 * y1 - y0 * x1;
  if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) { const Edges E = tri_edges_fp64(x0, y0, x1, y1, x2, y2); e0 = E.e0; e1 = E.e1; e2 = E.e2; }
  if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return -1.0f;
  const float det = e0 + e1 + e2;
  if (det == 0.0f) return -1.0f;
  z0 *= sz; z1 *= sz; z2 *= sz;
  const float ts = e0 * z0 + e1 * z1 + e2 * z2;
  if (det < 0.0f && (ts >= tmin || ts < tmax * det)) return -1.0f;
  if (det > 0.0f && (ts <= tmin || ts > tmax * det)) return -1.0f;
  const float inv = 1.0f / det;
  const float t = ts * inv;
  const float mz = fmaxf(fabsf(z0), fmaxf(fabsf(z1), fabsf(z2)));
  const float mx = fmaxf(fabsf(x0), fmaxf(fabsf(x1), fabsf(x2)));
  const float my = fmaxf(fabsf(y0), fmaxf(fabsf(y1), fabsf(y2)));
  const float dz = gamma_n(3) * mz;
  const float ddx = gamma_n(5) * (mx + mz);
  const float ddy = gamma_n(5) * (my + mz);
  const float de = 2.0f * (gamma_n(2) * mx * my + ddy * mx + ddx * my);
  const float me = fmaxf(fabsf(e0), fmaxf(fabsf(e1), fabsf(e2)));
  const float dt = 3.0f * (gamma_n(3) * me * mz + de * mz + dz * me) * fabsf(inv);
  if (t <= dt) return -1.0f;
  return t;
}

// The ray-only part of tri_t, computed once per ray and space: the dominant
// axis kz and the shear (sx, sy, sz).
struct Shear { int kz; float sx, sy, sz; };
DFC_D Shear make_shear(V3 d) {
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  Shear s;
  s.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  const float dX = s.kz == 0 ? d.y : (s.kz == 1 ? d.z : d.x);
  const float dY = s.kz == 0 ? d.z : (s.kz == 1 ? d.x : d.y);
  const float dZ = s.kz == 0 ? d.x : (s.kz == 1 ? d.y : d.z);
  s.sx = -dX / dZ; s.sy = -dY / dZ; s.sz = 1.0f / dZ;
  return s;
}

// tri_t with the shear precomputed; the same arithmetic step for step, so the
// result is bit-identical.  Vertex components are permuted by selects, not
// branches, so lanes with different dominant axes do not diverge.
DFC_D float tri_t_sheared(float4 A, float4 B, float4 C, V3 o, const Shear& sh, float tmin, float tmax) {
  const V3 p0 = {A.x - o.x, A.y - o.y, A.z - o.z}, p1 = {B.x - o.x, B.y - o.y, B.z - o.z}, p2 = {C.x - o.x, C.y - o.y, C.z - o.z};
  const bool k0 = sh.kz == 0, k1 = sh.kz == 1;
  float x0 = k0 ? p0.y : (k1 ? p0.z : p0.x), y0 = k0 ? p0.z : (k1 ? p0.x : p0.y), z0 = k0 ? p0.x : (k1 ? p0.y : p0.z);
  float x1 = k0 ? p1.y : (k1 ? p1.z : p1.x), y1 = k0 ? p1.z : (k1 ? p1.x : p1.y), z1 = k0 ? p1.x : (k1 ? p1.y : p1.z);
  float x2 = k0 ? p2.y : (k1 ? p2.z : p2.x), y2 = k0 ? p2.z : (k1 ? p2.x : p2.y), z2 = k0 ? p2.x : (k1 ? p2.y : p2.z);
  x0 = x0 + sh.sx * z0; y0 = y0 + sh.sy * z0;
  x1 = x1 + sh.sx * z1; y1 = y1 + sh.sy * z1;
  x2 = x2 + sh.sx * z2; y2 = y2 + sh.sy * z2;
  float e0 = x1 * y2 - y1 * x2;
  float e1 = x2 * y0 - y2 * x0;
  float e2 = x0 * y1 - y0 * x1;
  if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) { const Edges E = tri_edges_fp64(x0, y0, x1, y1, x2, y2); e0 = E.e0; e1 = E.e1; e2 = E.e2; }
  if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return -1.0f;
  const float det = e0 + e1 + e2;
  if (det == 0.0f) return -1.0f;
  z0 *= sh.sz; z1 *= sh.sz; z2 *= sh.sz;
  const float ts = e0 * z0 + e1 * z1 + e2 * z2;
  if (det < 0.0f && (ts >= tmin || ts < tmax * det)) return -1.0f;
  if (det > 0.0f && (ts <= tmin || ts > tmax * det)) return -1.0f;
  const float inv = 1.0f / det;
  const float t = ts * inv;
  const float mz = fmaxf(fabsf(z0), fmaxf(fabsf(z1), fabsf(z2)));
  const float mx = fmaxf(fabsf(x0), fmaxf(fabsf(x1), fabsf(x2)));
  const float my = fmaxf(fabsf(y0), fmaxf(fabsf(y1), fabsf(y2)));
  const float dz = gamma_n(3) * mz;
  const float ddx = gamma_n(5) * (mx + mz);
  const float ddy = gamma_n(5) * (my + mz);
  const float de = 2.0f * (gamma_n(2) * mx * my + ddy * mx + ddx * my);
  const float me = fmaxf(fabsf(e0), fmaxf(fabsf(e1), fabsf(e2)));
  const float dt = 3.0f * (gamma_n(3) * me * mz + de * mz + dz * me) * fabsf(inv);
  if (t <= dt) return -1.0f;
  return t;
}

// utility/EFloat.java: running float interval for the sphere test.
struct EF { float v, lo, hi; };
DFC_D EF ef(float v) { return {v, v, v}; }
DFC_D float nup(float v) { return nextafterf(v, __int_as_float(0x7f800000)); }
DFC_D float ndn(float v) { return nextafterf(v, -__int_as_float(0x7f800000)); }
DFC_D EF ef_add(EF a, EF b) { return {a.v + b.v, ndn(a.lo + b.lo), nup(a.hi + b.hi)}; }
DFC_D EF ef_sub(EF a, EF b) { return {a.v - b.v, ndn(a.lo - b.hi), nup(a.hi - b.lo)}; }
DFC_D EF ef_mul(EF a, EF b) {
  float p0 = a.lo * b.lo, p1 = a.hi * b.lo, p2 = a.lo * b.hi, p3 = a.hi * b.hi;
  return {a.v * b.v, ndn(fminf(fminf(p0, p1), fminf(p2, p3))), nup(fmaxf(fmaxf(p0, p1), fmaxf(p2, p3)))};
}
DFC_D EF ef_div(EF a, EF b) {
  float v = a.v / b.v;
  if (b.lo < 0.0f && b.hi > 0.0f) return {v, -__int_as_float(0x7f800000), __int_as_float(0x7f800000)};
  float d0 = a.lo / b.lo, d1 = a.hi / b.lo, d2 = a.lo / b.hi, d3 = a.hi / b.hi;
  return {v, ndn(fminf(fminf(d0, d1), fminf(d2, d3))), nup(fmaxf(fmaxf(d0, d1), fmaxf(d2, d3)))};
}
// geometry/shape/Sphere3F.java:507, unit sphere; returns -1 on a miss.
static __device__ __noinline__ float sphere_t_exact(V3 o, V3 d, float tmin, float tmax);
// A float pre-test that only rejects rays that clearly miss (the closest
// approach of the line is outside the sphere by a margin far above rounding),
// so that most candidate spheres never reach the interval-arithmetic test.
DFC_D float sphere_t(V3 o, V3 d, float tmin, float tmax) {
  const float b = o.x * d.x + o.y * d.y + o.z * d.z;
  const float oo = o.x * o.x + o.y * o.y + o.z * o.z;
  const float disc = b * b - (oo - 1.0f);
  // float rounding of b*b and oo is below 1e-6 (1 + oo); reject only beyond 1e-5 (1 + oo)
  if (disc < -1.0e-5f * (1.0f + oo)) return -1.0f;
  return sphere_t_exact(o, d, tmin, tmax);
}
static __device__ __noinline__ float sphere_t_exact(V3 o, V3 d, float tmin, float tmax) {
  EF ox = ef(o.x), oy = ef(o.y), oz = ef(o.z), dx = ef(d.x), dy = ef(d.y), dz = ef(d.z);
  EF a = ef_add(ef_add(ef_mul(dx, dx), ef_mul(dy, dy)), ef_mul(dz, dz));
  EF b = ef_mul(ef(2.0f), ef_add(ef_add(ef_mul(dx, ox), ef_mul(dy, oy)), ef_mul(dz, oz)));
  EF c = ef_sub(ef_add(ef_add(ef_mul(ox, ox), ef_mul(oy, oy)), ef_mul(oz, oz)), ef(1.0f));
  double disc = (double)b.v * (double)b.v - 4.0 * (double)a.v * (double)c.v;
  if (disc < 0.0) return -1.0f;
  double root = sqrt(disc);
  float fr = (float)root;
  EF r = {fr, ndn(fr - 5.9604645e-8f * fr), nup(fr + 5.9604645e-8f * fr)};
  if (fr == 0.0f) r = ef(0.0f);
  EF q = b.v < 0.0f ? ef_mul(ef(-0.5f), ef_sub(b, r)) : ef_mul(ef(-0.5f), ef_add(b, r));
  EF t0 = ef_div(q, a), t1 = ef_div(c, q);
  if (t0.v > t1.v) { EF s = t0; t0 = t1; t1 = s; }
  if (t0.hi > tmax || t1.lo <= tmin) return -1.0f;
  EF th = t0;
  if (th.lo <= 0.0f) { th = t1; if (th.hi > tmax) return -1.0f; }
  return th.v;
}

// geometry/shape/Rectangle3F.java:368 over the compiled record (position, side A, side B, normal).
DFC_D float rect_t(const float* q, V3 o, V3 d, float tmin, float tmax) {
  V3 n = ld3(q + 9);
  float dp = dot(n, d);
  if (dp == 0.0f) return -1.0f;
  V3 a = ld3(q), sa = ld3(q + 3), sb = ld3(q + 6);
  float t = dot(a - o, n) / dp;
  if (t <= tmin || t >= tmax) return -1.0f;
  V3 ap = (o + d * t) - a;
  float x = dot(ap, normalize(sa)), y = dot(ap, normalize(sb));
  if (x >= 0.0f && x <= len(sa) && y >= 0.0f && y <= len(sb)) return t;
  return -1.0f;
}

// geometry/shape/Plane3F.java (z = 0 in object space)
DFC_D float plane_t(V3 o, V3 d, float tmin, float tmax) {
  if (d.z == 0.0f) return -1.0f;
  float t = -o.z / d.z;
  return (t > tmin && t < tmax) ? t : -1.0f;
}

// ------------------------------------------------------------- surfaces --
struct Surface { ONB g, s; V3 p; float tu, tv; };

// geometry/shape/Triangle3F.java:1070-1160 surface at object-space distance t.
DFC_D Surface triangle_surface(const float* q, V3 o, V3 d, float t) {
  V3 A = ld3(q), B = ld3(q + 3), C = ld3(q + 6);
  V3 eab = B - A, eca = A - C;
  V3 d1 = cross(eab, eca);
  float inv = 1.0f / dot(d, d1);
  V3 d3 = cross(A - o, d);
  float bu = dot(d3, eca) * inv, bv = dot(d3, eab) * inv, bw = 1.0f - bu - bv;
  Surface s;
  s.p = o + d * t;
  s.tu = q[9] * bw + q[11] * bu + q[13] * bv;
  s.tv = q[10] * bw + q[12] * bu + q[14] * bv;
  s.g = onb_w(normalize(cross(normalize(B - A), normalize(C - A))));
  V3 w = normalize(ld3(q + 15) * bw + ld3(q + 18) * bu + ld3(q + 21) * bv);
  float ca0 = q[9] - q[13], ca1 = q[10] - q[14], cb0 = q[11] - q[13], cb1 = q[12] - q[14];
  float det = ca0 * cb1 - ca1 * cb0;
  if (det == 0.0f) {
    s.s = onb_w(w);
  } else {
    float rd = 1.0f / det;
    V3 ec = A - C, eb = B - C;
    s.s = onb_wv(w, V3{(-cb0 * ec.x + ca0 * eb.x) * rd, (-cb0 * ec.y + ca0 * eb.y) * rd, (-cb0 * ec.z + ca0 * eb.z) * rd});
  }
  return s;
}

// geometry/shape/Sphere3F.java:243 surface (unit sphere, full).
DFC_D Surface sphere_surface(V3 o, V3 d, float t) {
  V3 p = o + d * t;
  float sc = 1.0f / len(p);
  p = p * sc;
  if (p.x == 0.0f && p.y == 0.0f) p.x = 1.0e-5f;
  float phi = atan2f(p.y, p.x);
  if (phi < 0.0f) phi += 2.0f * kPi;
  const float phiMax = 2.0f * kPi;
  float theta = acosf(clampf(p.z, -1.0f, 1.0f));
  float zr = sqrtf(p.x * p.x + p.y * p.y), zri = 1.0f / zr;
  float cphi = p.x * zri, sphi = p.y * zri;
  V3 dpdu = {-phiMax * p.y, phiMax * p.x, 0.0f};
  V3 dpdv = V3{p.z * cphi, p.z * sphi, -sinf(theta)} * (-kPi);
  Surface s;
  s.g.w = normalize(cross(dpdu, dpdv)); s.g.v = dpdv; s.g.u = dpdu;  // stored unnormalized as the reference does
  s.s = s.g;
  s.p = p; s.tu = phi / phiMax; s.tv = (theta - kPi) / (0.0f - kPi);
  return s;
}

DFC_D Surface rect_surface(const float* q, V3 o, V3 d, float t) {
  Surface s;
  V3 n = ld3(q + 9), a = ld3(q), b = a + ld3(q + 3), dd = a + ld3(q + 6);
  s.p = o + d * t;
  s.g = onb_w(n); s.s = s.g;
  V3 na = {fabsf(n.x), fabsf(n.y), fabsf(n.z)};
  bool isX = na.x > na.y && na.x > na.z, isY = na.y > na.z;
  auto pr0 = [&](V3 p) { return isX ? p.y : (isY ? p.z : p.x); };
  auto pr1 = [&](V3 p) { return isX ? p.z : (isY ? p.x : p.y); };
  float vA0 = pr0(a), vA1 = pr1(a), vB0 = pr0(dd), vB1 = pr1(dd), vC0 = pr0(b), vC1 = pr1(b);
  float ab0 = vB0 - vA0, ab1 = vB1 - vA1, ac0 = vC0 - vA0, ac1 = vC1 - vA1;
  float di = 1.0f / (ab0 * ac1 - ab1 * ac0);
  float h0 = pr0(s.p), h1 = pr1(s.p);
  s.tu = h0 * (-ab1 * di) + h1 * (ab0 * di) + (vA0 * ab1 - vA1 * ab0) * di;
  s.tv = h0 * (ac1 * di) + h1 * (-ac0 * di) + (ac0 * vA1 - ac1 * vA0) * di;
  return s;
}

DFC_D Surface plane_surface(V3 o, V3 d, float t) {
  Surface s;
  s.p = o + d * t;
  s.g.w = {0, 0, 1}; s.g.v = {0, 1, 0}; s.g.u = {1, 0, 0};
  s.s = s.g;
  s.tu = s.p.x; s.tv = s.p.y;
  return s;
}

// geometry/SurfaceIntersection3F.java:372 object -> world for one primitive.
DFC_D void surface_to_world(const DPrim& pr, Surface& s) {
  if (pr.identity) {
    s.g.u = normalize(s.g.u); s.g.v = normalize(s.g.v); s.g.w = normalize(s.g.w);
    s.s.u = normalize(s.s.u); s.s.v = normalize(s.s.v); s.s.w = normalize(s.s.w);
  } else {
    s.g.u = normalize(xf_vec_t(pr.w2o, s.g.u)); s.g.v = normalize(xf_vec_t(pr.w2o, s.g.v)); s.g.w = normalize(xf_vec_t(pr.w2o, s.g.w));
    s.s.u = normalize(xf_vec_t(pr.w2o, s.s.u)); s.s.v = normalize(xf_vec_t(pr.w2o, s.s.v)); s.s.w = normalize(xf_vec_t(pr.w2o, s.s.w));
    s.p = xf_point(pr.o2w, s.p);
  }
  if (dot(s.s.w, s.g.w) < 0.0f) s.s.w = -s.s.w;  // OrthonormalBasis33F.flipW
}

// ---------------------------------------------------------------- BSDFs --
enum { kRefl = 1, kTrans = 2, kDiffuse = 4, kGlossy = 8, kSpecular = 16, kAll = 31, kAllButSpecular = 15 };
enum : int {
  kLambert = 0, kOrenNayar = 1, kSpecBRDF = 2, kFresnelSpec = 3, kSpecBTDF = 4, kTSBRDF = 5, kTSBTDF = 6,
  kLambertBTDF = 7,                                                                   // scene/bxdf/LambertianBTDF.java
  kFresnelBlend = 13,                                                                 // scene/bxdf/FresnelBlendBRDF.java
  kDisneyDiffuse = 8, kDisneyFakeSS = 9, kDisneyRetro = 10, kDisneySheen = 11, kDisneyClearCoat = 12  // scene/bxdf/Disney*.java
};
enum : int { kFresConst = 0, kFresDielectric = 1, kFresConductor = 2, kFresDisney = 3 };
constexpr int kMaxLobes = 8;  // DisneyMaterial, thin: diffuse, fake subsurface, retro, sheen, specular, clear coat, two transmissions

// One BxDF of a BSDF: 24 bytes.  Parameters every lobe of one material shares
// (Fresnel and refraction indices, conductor or Disney colours) live in the Bsdf.
struct Lobe {
  unsigned char kind, type, fresnel, separable;  // separable: G = G1(wo) G1(wi) (MicrofacetDistribution.isSeparableModel)
  V3 scale;
  float p0, p1;  // Oren-Nayar A, B | microfacet alpha x, y | Disney roughness | clear coat alpha, weight | specular BTDF etaA, etaB
};
// A BSDF of at most N lobes.  The matte, mirror, glass, metal and plastic
// materials need at most two (kSimpleLobes): their shading kernel holds the
// lobes in registers and compiles none of the other materials' lobe code.
template <int N>
struct BsdfN {
  static constexpr int kN = N;
  int n;
  Lobe l[N];
  float eta;            // BSDF.getEta
  float fr_i, fr_t;     // dielectric Fresnel of reflection lobes (Disney: etaT)
  float bt_a, bt_b;     // etaA, etaB of transmission lobes
  float metallic;       // DisneyFresnel blend
  V3 ca, cb;            // conductor eta and k | Disney R0 | FresnelSpecular transmittance (ca) | FresnelBlend specular (ca)
  ONB s;
  V3 ng, wo_w, wo;
};
using Bsdf = BsdfN<kMaxLobes>;
constexpr int kSimpleLobes = 2;
using SimpleBsdf = BsdfN<kSimpleLobes>;
// Every lobe kind and Fresnel term (false: only those of the matte, mirror, glass, metal and plastic materials).
template <class BT> constexpr bool kAllLobes = BT::kN >= kMaxLobes;

DFC_D float fr_dielectric(float cosi, float etaI, float etaT) {  // scene/fresnel/DielectricFresnel.java
  float c = clampf(cosi, -1.0f, 1.0f);
  bool ent = c > 0.0f;
  float ci = ent ? c : fabsf(c);
  float ei = ent ? etaI : etaT, et = ent ? etaT : etaI;
  float si = sqrtf(fmaxf(0.0f, 1.0f - ci * ci));
  float st = ei / et * si;
  if (st >= 1.0f) return 1.0f;
  float ct = sqrtf(fmaxf(0.0f, 1.0f - st * st));
  float rpa = ((et * ci) - (ei * ct)) / ((et * ci) + (ei * ct));
  float rpe = ((ei * ci) - (et * ct)) / ((ei * ci) + (et * ct));
  return (rpa * rpa + rpe * rpe) / 2.0f;
}
DFC_D float fr_conductor1(float c, float eta, float k) {  // scene/fresnel/ConductorFresnel.java, etaI = 1
  c = clampf(c, -1.0f, 1.0f);
  float c2 = c * c, s2 = 1.0f - c2, s4 = s2 * s2, eta2 = eta * eta, k2 = k * k;
  float t0 = eta2 - k2 - s2;
  float ab = sqrtf(t0 * t0 + eta2 * k2 * 4.0f);
  float t1 = ab + c2, t2 = sqrtf((ab + t0) * 0.5f) * (c * 2.0f), t3 = ab * c2 + s4, t4 = t2 * s2;
  float rs = (t1 - t2) / (t1 + t2);
  float rp = rs * (t3 - t4) / (t3 + t4);
  return (rp + rs) * 0.5f;
}
DFC_D float schlick_w(float c) { float m = clampf(1.0f - c, 0.0f, 1.0f); return (m * m) * (m * m) * m; }  // Schlick.java:104
DFC_D float lerpf(float a, float b, float t) { return (1.0f - t) * a + t * b; }  // utility/Floats.java:591
template <class BT>
DFC_D V3 fresnel(const BT& B, const Lobe& L, float cosi) {
  if (L.fresnel == kFresDielectric) { float f = fr_dielectric(cosi, B.fr_i, B.fr_t); return {f, f, f}; }
  if (L.fresnel == kFresConductor) {
    float c = fabsf(cosi);
    return {fr_conductor1(c, B.ca.x, B.cb.x), fr_conductor1(c, B.ca.y, B.cb.y), fr_conductor1(c, B.ca.z, B.cb.z)};
  }
  if constexpr (kAllLobes<BT>) {
    if (L.fresnel == kFresDisney) {  // scene/fresnel/DisneyFresnel.java
      const float d = fr_dielectric(cosi, 1.0f, B.fr_t), w = schlick_w(cosi);
      return {lerpf(d, lerpf(B.ca.x, 1.0f, w), B.metallic), lerpf(d, lerpf(B.ca.y, 1.0f, w), B.metallic),
              lerpf(d, lerpf(B.ca.z, 1.0f, w), B.metallic)};
    }
  }
  return {1, 1, 1};
}

DFC_D float sin2t(V3 v) { return fmaxf(0.0f, 1.0f - v.z * v.z); }
DFC_D float sint(V3 v) { return sqrtf(sin2t(v)); }
DFC_D float cosphi(V3 v) { float s = sint(v); return s == 0.0f ? 1.0f : clampf(v.x / s, -1.0f, 1.0f); }
DFC_D float sinphi(V3 v) { float s = sint(v); return s == 0.0f ? 0.0f : clampf(v.y / s, -1.0f, 1.0f); }
DFC_D bool same_hemi(V3 a, V3 b) { return a.z * b.z > 0.0f; }

// scene/microfacet/TrowbridgeReitzMicrofacetDistribution.java (alphas in p0, p1)
DFC_D float tr_D(const Lobe& L, V3 h) {
  float t2 = sin2t(h) / (h.z * h.z);
  if (isinf(t2)) return 0.0f;
  float cp = cosphi(h), sp = sinphi(h);
  float c4 = (h.z * h.z) * (h.z * h.z);
  float e = (cp * cp / (L.p0 * L.p0) + sp * sp / (L.p1 * L.p1)) * t2;
  return 1.0f / (kPi * L.p0 * L.p1 * c4 * (1.0f + e) * (1.0f + e));
}
DFC_D float tr_lambda(const Lobe& L, V3 w) {
  float ta = fabsf(sint(w) / w.z);
  if (isinf(ta)) return 0.0f;
  float cp = cosphi(w), sp = sinphi(w);
  float al = sqrtf(cp * cp * L.p0 * L.p0 + sp * sp * L.p1 * L.p1);
  float x = (al * ta) * (al * ta);
  return (-1.0f + sqrtf(1.0f + x)) / 2.0f;
}
DFC_D float tr_G(const Lobe& L, V3 wo, V3 wi) {
  return L.separable ? (1.0f / (1.0f + tr_lambda(L, wo))) * (1.0f / (1.0f + tr_lambda(L, wi)))
                     : 1.0f / (1.0f + tr_lambda(L, wo) + tr_lambda(L, wi));
}
DFC_D float tr_pdf(const Lobe& L, V3 wo, V3 h) {
  return tr_D(L, h) * (1.0f / (1.0f + tr_lambda(L, wo))) * fabsf(dot(wo, h)) / fabsf(wo.z);
}
DFC_D V3 tr_visible(V3 w, float ax, float ay, float u, float v) {
  V3 ws = normalize(V3{w.x * ax, w.y * ay, w.z});
  float ct = ws.z, sx, sy;
  if (ct > 0.9999f) {
    float r = sqrtf(u / (1.0f - u)), s, c;
    sincosf(2.0f * kPi * v, &s, &c);
    sx = r * c; sy = r * s;
  } else {
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct)), tt = st / ct;
    float a = 2.0f / (1.0f + sqrtf(1.0f + 1.0f / ((1.0f / tt) * (1.0f / tt))));
    float b = 2.0f * u / a - 1.0f;
    float c = fminf(1.0f / (b * b - 1.0f), 1.0e10f);
    float e = sqrtf(fmaxf(tt * tt * c * c - (b * b - tt * tt) * c, 0.0f));
    float f = tt * c - e, g = tt * c + e;
    float hs = v > 0.5f ? 1.0f : -1.0f;
    float i = v > 0.5f ? 2.0f * (v - 0.5f) : 2.0f * (0.5f - v);
    float j = (i * (i * (i * 0.27385f - 0.73369f) + 0.46341f)) / (i * (i * (i * 0.093073f + 0.309420f) - 1.0f) + 0.597999f);
    sx = (b < 0.0f || g > 1.0f / tt) ? f : g;
    sy = hs * j * sqrtf(1.0f + sx * sx);
  }
  float cp = cosphi(ws), sp = sinphi(ws);
  return normalize(V3{-((cp * sx - sp * sy) * ax), -((sp * sx + cp * sy) * ay), 1.0f});
}
DFC_D V3 tr_sample_h(const Lobe& L, V3 wo, float u, float v) {
  return wo.z >= 0.0f ? tr_visible(wo, L.p0, L.p1, u, v) : -tr_visible(-wo, L.p0, L.p1, u, v);
}
DFC_D bool refract(V3 d, V3 n, float eta, V3* out) {  // geometry/Vector3F.java:454
  float ci = dot(d, n);
  float st2 = eta * eta * fmaxf(0.0f, 1.0f - ci * ci);
  if (st2 >= 1.0f) return false;
  *out = (-d) * eta + n * (eta * ci - sqrtf(1.0f - st2));
  return true;
}
// DisneyClearCoatBRDF.java:330 doGTR1, :337 doSmithGGGX
DFC_D float gtr1(float ct, float alpha) {
  const float a = alpha * alpha;
  return (a - 1.0f) / (kPi * logf(a) * (1.0f + (a - 1.0f) * ct * ct));
}
DFC_D float smith_ggx(float ct, float alpha) {
  const float a = alpha * alpha, b = ct * ct;
  return 1.0f / (ct + sqrtf(a + b - a * b));
}

template <class BT>
DFC_D V3 lobe_f(const BT& B, const Lobe& L, V3 wo, V3 wi) {
  switch (L.kind) {
    case kLambert: case kLambertBTDF: return L.scale * (1.0f / kPi);
    case kOrenNayar: {
      float ci = fabsf(wi.z), co = fabsf(wo.z), si = sint(wi), so = sint(wo);
      float mc = (si > 1.0e-4f && so > 1.0e-4f) ? fmaxf(0.0f, cosphi(wi) * cosphi(wo) + sinphi(wi) * sinphi(wo)) : 0.0f;
      float sa = ci > co ? so : si, tb = ci > co ? si / ci : so / co;
      return L.scale * (1.0f / kPi) * (L.p0 + L.p1 * mc * sa * tb);
    }
    case kTSBRDF: {
      float co = fabsf(wo.z), ci = fabsf(wi.z);
      if (co == 0.0f || ci == 0.0f) return {0, 0, 0};
      V3 h = wi + wo;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return {0, 0, 0};
      h = normalize(h);
      V3 hf = h.z < 0.0f ? -h : h;
      V3 F = fresnel(B, L, dot(wi, hf));
      return mul(L.scale * (tr_D(L, h) * tr_G(L, wo, wi)), F) * (1.0f / (4.0f * ci * co));
    }
    case kTSBTDF: {
      if (same_hemi(wo, wi)) return {0, 0, 0};
      if (wi.z == 0.0f || wo.z == 0.0f) return {0, 0, 0};
      float eta = wo.z > 0.0f ? B.bt_b / B.bt_a : B.bt_a / B.bt_b;
      V3 h = normalize(wi * eta + wo);
      if (h.z < 0.0f) h = -h;
      float oh = dot(wo, h), ih = dot(wi, h);
      if (oh * ih > 0.0f) return {0, 0, 0};
      float F = fr_dielectric(oh, B.bt_a, B.bt_b);
      float a = oh + eta * ih, b = 1.0f / eta;
      float k = fabsf(tr_D(L, h) * tr_G(L, wo, wi) * eta * eta * fabsf(ih) * fabsf(oh) * b * b / (wi.z * wo.z * a * a));
      return L.scale * ((1.0f - F) * k);
    }
    default: break;
  }
  if constexpr (kAllLobes<BT>) switch (L.kind) {
    case kFresnelBlend: {  // FresnelBlendBRDF.java (scale: diffuse, Bsdf.ca: specular)
      V3 h = wo + wi;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return {0, 0, 0};
      h = normalize(h);
      auto pow5 = [](float x) { return x * x * x * x * x; };
      const float a = 28.0f / (23.0f * kPi);
      const float b = 1.0f - pow5(1.0f - 0.5f * fabsf(wi.z));
      const float c = 1.0f - pow5(1.0f - 0.5f * fabsf(wo.z));
      const float f = tr_D(L, h) / (4.0f * fabsf(dot(wi, h)) * fmaxf(fabsf(wi.z), fabsf(wo.z)));
      const float w = pow5(1.0f - dot(wi, h));
      const V3 ks = B.ca;
      const V3 fr = {ks.x + (1.0f - ks.x) * w, ks.y + (1.0f - ks.y) * w, ks.z + (1.0f - ks.z) * w};
      return mul(L.scale * a, V3{1.0f - ks.x, 1.0f - ks.y, 1.0f - ks.z}) * b * c + fr * f;
    }
    case kDisneyDiffuse: {  // DisneyDiffuseBRDF.java
      const float a = 1.0f - schlick_w(fabsf(wo.z)) / 2.0f, b = 1.0f - schlick_w(fabsf(wi.z)) / 2.0f;
      return V3{L.scale.x * (1.0f / kPi) * a * b, L.scale.y * (1.0f / kPi) * a * b, L.scale.z * (1.0f / kPi) * a * b};
    }
    case kDisneyFakeSS: case kDisneyRetro: case kDisneySheen: case kDisneyClearCoat: {
      V3 h = wi + wo;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return {0, 0, 0};
      h = normalize(h);
      if (L.kind == kDisneyClearCoat) {  // DisneyClearCoatBRDF.java
        const float d = gtr1(fabsf(h.z), L.p0);
        const float f = lerpf(0.04f, 1.0f, schlick_w(dot(wo, h)));
        const float g = smith_ggx(fabsf(wo.z), 0.25f) * smith_ggx(fabsf(wi.z), 0.25f);
        const float c = L.p1 * g * f * d / 4.0f;
        return {c, c, c};
      }
      const float cd = dot(wi, h);
      if (L.kind == kDisneySheen) return L.scale * schlick_w(cd);  // DisneySheenBRDF.java
      const float co = fabsf(wo.z), ci = fabsf(wi.z), fo = schlick_w(co), fi = schlick_w(ci);
      if (L.kind == kDisneyRetro) {  // DisneyRetroBRDF.java
        const float a = 2.0f * L.p0 * cd * cd;
        const float b = fo + fi + fo * fi * (a - 1.0f);
        return V3{L.scale.x * (1.0f / kPi) * a * b, L.scale.y * (1.0f / kPi) * a * b, L.scale.z * (1.0f / kPi) * a * b};
      }
      const float f90 = cd * cd * L.p0;  // DisneyFakeSSBRDF.java
      const float fss = lerpf(1.0f, f90, fo) * lerpf(1.0f, f90, fi);
      const float ss = 1.25f * (fss * (1.0f / (co + ci) - 0.5f) + 0.5f);
      return V3{L.scale.x * (1.0f / kPi) * ss, L.scale.y * (1.0f / kPi) * ss, L.scale.z * (1.0f / kPi) * ss};
    }
    default: break;
  }
  return {0, 0, 0};
}
template <class BT>
DFC_D float lobe_pdf(const BT& B, const Lobe& L, V3 wo, V3 wi) {
  if constexpr (kAllLobes<BT>) switch (L.kind) {
    case kDisneyDiffuse: case kDisneyFakeSS: case kDisneyRetro: case kDisneySheen:
      return same_hemi(wo, wi) ? fabsf(wi.z) * (1.0f / kPi) : 0.0f;
    case kLambertBTDF: return same_hemi(wo, wi) ? 0.0f : fabsf(wi.z) * (1.0f / kPi);
    case kFresnelBlend: {
      if (!same_hemi(wo, wi)) return 0.0f;
      const V3 h = normalize(wo + wi);
      return 0.5f * (fabsf(wi.z) * (1.0f / kPi) + tr_pdf(L, wo, h) / (4.0f * dot(wo, h)));
    }
    case kDisneyClearCoat: {
      if (!same_hemi(wo, wi)) return 0.0f;
      V3 h = wi + wo;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return 0.0f;
      h = normalize(h);
      const float ch = fabsf(h.z);
      return gtr1(ch, L.p0) * ch / (4.0f * dot(wo, h));
    }
    default: break;
  }
  switch (L.kind) {
    case kLambert: case kOrenNayar:
      return same_hemi(wo, wi) ? fabsf(wi.z) * (1.0f / kPi) : 0.0f;
    case kTSBRDF: {
      if (!same_hemi(wo, wi)) return 0.0f;
      V3 h = normalize(wo + wi);
      return tr_pdf(L, wo, h) / (4.0f * dot(wo, h));
    }
    case kTSBTDF: {
      if (same_hemi(wo, wi)) return 0.0f;
      float eta = wo.z > 0.0f ? B.bt_b / B.bt_a : B.bt_a / B.bt_b;
      V3 h = normalize(wi * eta + wo);
      float oh = dot(wo, h), ih = dot(wi, h);
      if (oh * ih > 0.0f) return 0.0f;
      float a = oh + eta * ih;
      return tr_pdf(L, wo, h) * fabsf((eta * eta * ih) / (a * a));
    }
    default: return 0.0f;
  }
}
struct LSample { V3 f, wi; float pdf; int type; };
template <class BT>
DFC_D bool lobe_sample(const BT& B, const Lobe& L, V3 wo, float u, float v, LSample* s) {
  s->type = L.type;
  if constexpr (kAllLobes<BT>) switch (L.kind) {
    case kFresnelBlend: {  // FresnelBlendBRDF.java:sampleDistributionFunction
      V3 wi;
      if (u < 0.5f) {
        wi = cosine_hemisphere(fminf(2.0f * u, 0.99999994f), v);
        if (wo.z < 0.0f) wi.z = -wi.z;
      } else {
        const V3 h = tr_sample_h(L, wo, fminf(2.0f * (u - 0.5f), 0.99999994f), v);
        wi = h * (dot(wo, h) * 2.0f) - wo;
        if (!same_hemi(wo, wi)) return false;
      }
      s->wi = wi; s->f = lobe_f(B, L, wo, wi); s->pdf = lobe_pdf(B, L, wo, wi); return true;
    }
    case kDisneyClearCoat: {  // DisneyClearCoatBRDF.java:sampleDistributionFunction
      if (wo.z == 0.0f) return false;
      const float a2 = L.p0 * L.p0;
      const float ct = sqrtf(fmaxf(0.0f, (1.0f - powf(a2, 1.0f - u)) / (1.0f - a2)));
      const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
      float sp, cp;
      sincosf(2.0f * kPi * v, &sp, &cp);
      V3 h = {st * cp, st * sp, ct};
      if (!same_hemi(wo, h)) h = -h;
      const V3 wi = h * (dot(wo, h) * 2.0f) - wo;
      if (!same_hemi(wo, wi)) return false;
      s->wi = wi; s->f = lobe_f(B, L, wo, wi); s->pdf = lobe_pdf(B, L, wo, wi); return true;
    }
    default: break;
  }
  switch (L.kind) {
    case kLambert: case kOrenNayar: case kDisneyDiffuse: case kDisneyFakeSS: case kDisneyRetro: case kDisneySheen:
    case kLambertBTDF: {
      V3 wi = cosine_hemisphere(u, v);
      // faceForwardZ for reflection, faceForwardZNegated for LambertianBTDF
      if (L.kind == kLambertBTDF ? wo.z > 0.0f : wo.z < 0.0f) wi.z = -wi.z;
      s->wi = wi; s->f = lobe_f(B, L, wo, wi); s->pdf = lobe_pdf(B, L, wo, wi); return true;
    }
    case kSpecBRDF: {
      V3 wi = {-wo.x, -wo.y, wo.z};
      s->wi = wi; s->f = mul(fresnel(B, L, wi.z), L.scale) * (1.0f / fabsf(wi.z)); s->pdf = 1.0f; return true;
    }
    case kSpecBTDF: case kFresnelSpec: {
      // SpecularBTDF carries its own etas (UberMaterial has two with different ones)
      const float ea = L.kind == kSpecBTDF ? L.p0 : B.bt_a, eb = L.kind == kSpecBTDF ? L.p1 : B.bt_b;
      float F = L.kind == kFresnelSpec ? fr_dielectric(wo.z, ea, eb) : 0.0f;
      if (L.kind == kFresnelSpec && u < F) {
        V3 wi = {-wo.x, -wo.y, wo.z};
        s->type = kSpecular | kRefl; s->wi = wi; s->f = L.scale * (F / fabsf(wi.z)); s->pdf = F; return true;
      }
      bool ent = wo.z > 0.0f;
      float ei = ent ? ea : eb, et = ent ? eb : ea;
      V3 n = wo.z < 0.0f ? V3{0, 0, -1} : V3{0, 0, 1};
      V3 wi;
      if (!refract(wo, n, ei / et, &wi)) return false;
      if (L.kind == kSpecBTDF) {
        float Ft = fr_dielectric(wi.z, ea, eb);
        s->wi = wi; s->f = L.scale * ((1.0f - Ft) * ((ei * ei) / (et * et)) / fabsf(wi.z)); s->pdf = 1.0f; return true;
      }
      s->type = kSpecular | kTrans; s->wi = wi;
      s->f = B.ca * ((1.0f - F) * ((ei * ei) / (et * et)) / fabsf(wi.z)); s->pdf = 1.0f - F; return true;
    }
    case kTSBRDF: {
      if (wo.z == 0.0f) return false;
      V3 h = tr_sample_h(L, wo, u, v);
      if (dot(wo, h) < 0.0f) return false;
      V3 wi = h * (dot(wo, h) * 2.0f) - wo;
      if (!same_hemi(wo, wi)) return false;
      s->wi = wi; s->f = lobe_f(B, L, wo, wi); s->pdf = tr_pdf(L, wo, h) / (4.0f * dot(wo, h)); return true;
    }
    case kTSBTDF: {
      if (wo.z == 0.0f) return false;
      V3 h = tr_sample_h(L, wo, u, v);
      if (dot(wo, h) < 0.0f) return false;
      float eta = wo.z > 0.0f ? B.bt_a / B.bt_b : B.bt_b / B.bt_a;
      V3 wi;
      if (!refract(wo, h, eta, &wi)) return false;
      s->wi = wi; s->f = lobe_f(B, L, wo, wi); s->pdf = lobe_pdf(B, L, wo, wi); return true;
    }
    default: break;
  }
  return false;
}
DFC_D bool type_match(int t, int flags) { return (t & flags) == t; }
DFC_D bool is_spec(int t) { return (t & kSpecular) != 0; }

DFC_D Lobe make_lobe(int kind, int type, V3 scale, float p0 = 0.0f, float p1 = 0.0f) {
  Lobe L;
  L.kind = (unsigned char)kind; L.type = (unsigned char)type; L.fresnel = kFresConst; L.separable = 0;
  L.scale = scale; L.p0 = p0; L.p1 = p1;
  return L;
}
DFC_D Lobe tr_lobe(int kind, int type, V3 scale, float ax, float ay) { return make_lobe(kind, type, scale, fmaxf(ax, 0.001f), fmaxf(ay, 0.001f)); }

// Appends a lobe.  The two-lobe form writes its slots by selects, so that no
// indexed store moves its lobes to local memory.
template <int N>
DFC_D void push_lobe(BsdfN<N>* B, const Lobe& L) {
  if constexpr (N <= kSimpleLobes) {
#pragma unroll
    for (int k = 0; k < N; ++k)
      if (B->n == k) B->l[k] = L;
  } else {
    B->l[B->n] = L;
  }
  ++B->n;
}

// DisneyMaterial.computeScatteringFunctions (scene/material/DisneyMaterial.java:1121-1210)
// from the per-material quantities ingest computed (DMaterial comments).
DFC_D void build_disney(const DMaterial& m, Bsdf* B) {
  const V3 color = ld3(m.c0);
  const bool thin = (m.flags & kDisneyThin) != 0;
  const float dw = m.d_dw;
  if (dw > 0.0f) {
    if (thin) {
      const float flat = m.c2[0], dt = m.c2[1];
      B->l[B->n++] = make_lobe(kDisneyDiffuse, kRefl | kDiffuse, color * (dw * (1.0f - flat) * (1.0f - dt)));
      B->l[B->n++] = make_lobe(kDisneyFakeSS, kRefl | kDiffuse, color * (dw * (0.0f + flat) * (1.0f - dt)), m.d_rough);
    } else if (!(m.flags & kDisneyScatter)) {
      B->l[B->n++] = make_lobe(kDisneyDiffuse, kRefl | kDiffuse, color * dw);
    } else {
      B->l[B->n++] = make_lobe(kSpecBTDF, kTrans | kSpecular, V3{1, 1, 1}, 1.0f, m.eta);
    }
    B->l[B->n++] = make_lobe(kDisneyRetro, kRefl | kDiffuse, color * dw, m.d_rough);
    if (m.flags & kDisneyHasSheen) B->l[B->n++] = make_lobe(kDisneySheen, kRefl | kDiffuse, ld3(m.c3));
  }
  Lobe spec = tr_lobe(kTSBRDF, kRefl | kGlossy, V3{1, 1, 1}, m.ax, m.ay);
  spec.fresnel = kFresDisney;
  spec.separable = 1;
  B->l[B->n++] = spec;
  if (m.flags & kDisneyHasClearCoat) B->l[B->n++] = make_lobe(kDisneyClearCoat, kRefl | kGlossy, V3{0, 0, 0}, m.d_gloss, m.d_cc);
  if (m.flags & kDisneyHasTransmission) {
    Lobe t = thin ? tr_lobe(kTSBTDF, kTrans | kGlossy, ld3(m.c4), m.on_a, m.on_b) : tr_lobe(kTSBTDF, kTrans | kGlossy, ld3(m.c4), m.ax, m.ay);
    t.separable = thin ? 0 : 1;
    B->l[B->n++] = t;
  }
  if (thin) B->l[B->n++] = make_lobe(kLambertBTDF, kTrans | kDiffuse, color * m.c2[1]);
  B->fr_t = m.eta;
  B->bt_a = 1.0f; B->bt_b = m.eta;
  B->metallic = m.d_met;
  B->ca = ld3(m.c1);
}

// Material.computeScatteringFunctions(intersection, RADIANCE, isAllowingMultipleLobes = true)
// for the resolved kinds (scene/material/*Material.java).  u_material is the
// random number ClearCoatMaterial draws per hit (ClearCoatMaterial.java:323).
// Returns false when the material gives no BSDF (the ray passes through).
// multi = isAllowingMultipleLobes: false (the ray tracer) builds smooth glass
// as separate specular reflection and transmission lobes (GlassMaterial.java:520).
// With fewer than kMaxLobes lobes (SimpleBsdf) only the matte, mirror, glass,
// metal and plastic kinds are built; the shading kernels route the others to
// the full Bsdf by the material sort.
template <int N>
DFC_D bool build_bsdf(const DMaterial& m, const Surface& sf, V3 ray_d, float u_material, BsdfN<N>* B, bool multi = true) {
  B->n = 0; B->eta = 1.0f;
  B->fr_i = 1.0f; B->fr_t = 1.0f; B->bt_a = 1.0f; B->bt_b = 1.0f; B->metallic = 0.0f;
  B->ca = V3{0, 0, 0}; B->cb = V3{0, 0, 0};
  switch (m.kind) {
    case kMatLambert: case kMatOrenNayar:
      push_lobe(B, make_lobe(m.kind == kMatLambert ? kLambert : kOrenNayar, kRefl | kDiffuse, ld3(m.c0), m.on_a, m.on_b));
      break;
    case kMatMirror:
      push_lobe(B, make_lobe(kSpecBRDF, kRefl | kSpecular, ld3(m.c0)));
      break;
    case kMatGlassSpec:
      if (multi) {
        push_lobe(B, make_lobe(kFresnelSpec, kRefl | kTrans | kSpecular, ld3(m.c0)));
        B->ca = ld3(m.c1);
      } else {
        if (m.has_kr) { Lobe L = make_lobe(kSpecBRDF, kRefl | kSpecular, ld3(m.c0)); L.fresnel = kFresDielectric; push_lobe(B, L); }
        if (m.has_kt) push_lobe(B, make_lobe(kSpecBTDF, kTrans | kSpecular, ld3(m.c1), 1.0f, m.eta));
        B->fr_i = 1.0f; B->fr_t = m.eta;
      }
      B->bt_a = 1.0f; B->bt_b = m.eta; B->eta = m.eta;
      break;
    case kMatGlassRough: {
      if (m.has_kr) { Lobe L = tr_lobe(kTSBRDF, kRefl | kGlossy, ld3(m.c0), m.ax, m.ay); L.fresnel = kFresDielectric; push_lobe(B, L); }
      if (m.has_kt) push_lobe(B, tr_lobe(kTSBTDF, kTrans | kGlossy, ld3(m.c1), m.ax, m.ay));
      B->fr_i = 1.0f; B->fr_t = m.eta; B->bt_a = 1.0f; B->bt_b = m.eta; B->eta = m.eta;
      break;
    }
    case kMatMetal: {
      Lobe L = tr_lobe(kTSBRDF, kRefl | kGlossy, V3{1, 1, 1}, m.ax, m.ay);
      L.fresnel = kFresConductor;
      push_lobe(B, L);
      B->ca = ld3(m.c1); B->cb = ld3(m.c2);
      break;
    }
    case kMatPlastic: {
      if (m.has_kr) push_lobe(B, make_lobe(kLambert, kRefl | kDiffuse, ld3(m.c0)));
      if (m.has_kt) { Lobe L = tr_lobe(kTSBRDF, kRefl | kGlossy, ld3(m.c1), m.ax, m.ay); L.fresnel = kFresDielectric; push_lobe(B, L); }
      B->fr_i = 1.5f; B->fr_t = 1.0f;
      break;
    }
    default:
      if constexpr (N >= kMaxLobes) {
        switch (m.kind) {
        case kMatDisney: build_disney(m, B); break;
        case kMatClearCoat: {  // ClearCoatMaterial.java:computeScatteringFunctions
          const V3 n = sf.s.w;
          const V3 nco = dot(n, ray_d) > 0.0f ? -n : n;  // Intersection.getSurfaceNormalSCorrectlyOriented
          const bool entering = dot(n, nco) > 0.0f;
          const float etaI = entering ? 1.0f : 1.5f, etaT = entering ? 1.5f : 1.0f;
          V3 refr;
          if (refract(ray_d, nco, etaI / etaT, &refr)) {  // Vector3F.refraction(direction, normal, eta)
            const float cosi = dot(ray_d, nco);
            const float R = fr_dielectric(entering ? -cosi : dot(refr, n), 1.0f, 1.5f), T = 1.0f - R;
            const float p = 0.25f + 0.5f * R;
            if (u_material < p) push_lobe(B, make_lobe(kSpecBRDF, kRefl | kSpecular, ld3(m.c1) * (R / p)));
            else push_lobe(B, make_lobe(kLambert, kRefl | kDiffuse, ld3(m.c0) * (T / (1.0f - p))));
          } else {
            push_lobe(B, make_lobe(kSpecBRDF, kRefl | kSpecular, ld3(m.c1)));
          }
          break;
        }
        case kMatGlossy: {
          Lobe L = tr_lobe(kTSBRDF, kRefl | kGlossy, ld3(m.c0), m.ax, m.ay);
          L.fresnel = kFresConductor;
          push_lobe(B, L);
          B->ca = ld3(m.c1); B->cb = ld3(m.c2);
          break;
        }
        case kMatSubstrate:
          push_lobe(B, tr_lobe(kFresnelBlend, kRefl | kGlossy, ld3(m.c0), m.ax, m.ay));
          B->ca = ld3(m.c1);
          break;
        case kMatTranslucent: {
          if (m.flags & 1) push_lobe(B, make_lobe(kLambert, kRefl | kDiffuse, ld3(m.c0)));
          if (m.flags & 2) push_lobe(B, make_lobe(kLambertBTDF, kTrans | kDiffuse, ld3(m.c1)));
          if (m.flags & 4) { Lobe L = tr_lobe(kTSBRDF, kRefl | kGlossy, ld3(m.c2), m.ax, m.ay); L.fresnel = kFresDielectric; push_lobe(B, L); }
          if (m.flags & 8) push_lobe(B, tr_lobe(kTSBTDF, kTrans | kGlossy, ld3(m.c3), m.ax, m.ay));
          B->fr_i = 1.0f; B->fr_t = 1.5f; B->bt_a = 1.0f; B->bt_b = 1.5f;
          break;
        }
        case kMatUber: {
          if (m.flags & 1) push_lobe(B, make_lobe(kSpecBTDF, kTrans | kSpecular, ld3(m.c4), 1.0f, 1.0f));
          if (m.flags & 2) push_lobe(B, make_lobe(kLambert, kRefl | kDiffuse, ld3(m.c0)));
          if (m.flags & 4) { Lobe L = tr_lobe(kTSBRDF, kRefl | kGlossy, ld3(m.c1), m.ax, m.ay); L.fresnel = kFresDielectric; push_lobe(B, L); }
          if (m.flags & 8) { Lobe L = make_lobe(kSpecBRDF, kRefl | kSpecular, ld3(m.c2)); L.fresnel = kFresDielectric; push_lobe(B, L); }
          if (m.flags & 16) push_lobe(B, make_lobe(kSpecBTDF, kTrans | kSpecular, ld3(m.c3), 1.0f, m.eta));
          B->fr_i = 1.0f; B->fr_t = m.eta;
          B->eta = (m.flags & 1) ? 1.0f : m.eta;
          break;
        }
        default: return false;
        }
        break;
      } else {
        return false;
      }
  }
  B->s = sf.s;
  B->ng = sf.g.w;
  B->wo_w = -ray_d;
  B->wo = normalize(to_local(B->wo_w, B->s));
  return B->n > 0 || m.kind == kMatUber;  // UberMaterial gives a BSDF even without lobes: the path ends there
}
// The lobe loops run over the N slots of the BSDF, unrolled for the two-lobe
// form so that its lobes stay in registers.
template <int N>
DFC_D V3 bsdf_f(const BsdfN<N>& B, int flags, V3 wi_w) {
  V3 wi = normalize(to_local(wi_w, B.s));
  bool refl = dot(wi_w, B.ng) * dot(B.wo_w, B.ng) > 0.0f;
  V3 r = {0, 0, 0};
#pragma unroll(N <= kSimpleLobes ? N : 1)
  for (int k = 0; k < N; ++k) {
    if (k >= B.n) break;
    const Lobe& L = B.l[k];
    if (type_match(L.type, flags) && ((refl && (L.type & kRefl)) || (!refl && (L.type & kTrans)))) r = r + lobe_f(B, L, B.wo, wi);
  }
  return r;
}
template <int N>
DFC_D float bsdf_pdf(const BsdfN<N>& B, int flags, V3 wi_w) {
  if (B.n == 0 || B.wo.z == 0.0f) return 0.0f;
  V3 wi = normalize(to_local(wi_w, B.s));
  float p = 0.0f;
  int m = 0;
#pragma unroll(N <= kSimpleLobes ? N : 1)
  for (int k = 0; k < N; ++k) {
    if (k >= B.n) break;
    if (type_match(B.l[k].type, flags)) { ++m; p += lobe_pdf(B, B.l[k], B.wo, wi); }
  }
  return m > 1 ? p / m : p;
}
struct BSample { V3 f, wi; float pdf; int type; };
// scene/BSDF.java:323 sampleDistributionFunction
template <int N>
DFC_D bool bsdf_sample(const BsdfN<N>& B, int flags, float u, float v, BSample* out) {
  if (B.wo.z == 0.0f) return false;
  int m = 0, match_k = -1;
#pragma unroll(N <= kSimpleLobes ? N : 1)
  for (int k = 0; k < N; ++k) {
    if (k >= B.n) break;
    if (type_match(B.l[k].type, flags)) ++m;
  }
  if (m == 0) return false;
  const int match = min((int)floorf(u * m), m - 1);
#pragma unroll(N <= kSimpleLobes ? N : 1)
  for (int k = 0, j = 0; k < N; ++k) {
    if (k >= B.n) break;
    if (!type_match(B.l[k].type, flags)) continue;
    if (j++ == match) { match_k = k; break; }
  }
  Lobe L;
  if constexpr (N <= kSimpleLobes) {  // a select, not an indexed (local-memory) read
    L = B.l[0];
#pragma unroll
    for (int k = 1; k < N; ++k)
      if (match_k == k) L = B.l[k];
  } else {
    L = B.l[match_k];
  }
  LSample s;
  if (!lobe_sample(B, L, B.wo, fminf(u * m - match, 0.99999994f), v, &s)) return false;
  V3 wiw = normalize(to_world(s.wi, B.s));
  V3 f = s.f;
  float pdf = s.pdf;
  if (!is_spec(L.type)) {
    bool refl = dot(wiw, B.ng) * dot(B.wo_w, B.ng) > 0.0f;
    f = {0, 0, 0};
#pragma unroll(N <= kSimpleLobes ? N : 1)
    for (int k = 0; k < N; ++k) {
      if (k >= B.n) break;
      const Lobe& O = B.l[k];
      if (!type_match(O.type, flags)) continue;
      if (k != match_k) pdf += lobe_pdf(B, O, B.wo, s.wi);
      if ((refl && (O.type & kRefl)) || (!refl && (O.type & kTrans))) f = f + lobe_f(B, O, B.wo, s.wi);
    }
  }
  if (m > 1) pdf /= m;
  out->f = f; out->wi = wiw; out->pdf = pdf; out->type = s.type;
  return true;
}
template <int N>
DFC_D int bsdf_nonspec(const BsdfN<N>& B) {
  int c = 0;
#pragma unroll(N <= kSimpleLobes ? N : 1)
  for (int k = 0; k < N; ++k) {
    if (k >= B.n) break;
    c += is_spec(B.l[k].type) ? 0 : 1;
  }
  return c;
}

// ---------------------------------------------------------------- lights --
// sampler/Distribution1F.java + Distribution2F.java over the packed array form.
DFC_D int d1_index(const float* a, int off, float value) {
  int lenc = (int)a[off + 1], mn = 0, cl = lenc;
  while (cl > 0) {
    int half = cl >> 1, mid = mn + half;
    if (a[off + 4 + mid] <= value) { mn = mid + 1; cl -= half + 1; } else { cl = half; }
  }
  int r = mn - 1;
  return r < 0 ? 0 : (r > lenc - 2 ? lenc - 2 : r);
}
DFC_D float d1_remap(const float* a, int off, float value, int i) {
  float n = a[off + 2], c0 = a[off + 4 + i], c1 = a[off + 4 + i + 1];
  if (c1 - c0 > 0.0f) return (i + ((value - c0) / (c1 - c0))) / n;
  return (i + (value - c0)) / n;
}
DFC_D void d2_remap(const float* a, float su, float sv, float* ou, float* ov) {
  bool uv = (int)a[0] != 0;
  float m = uv ? su : sv, c = uv ? sv : su;
  int offM = (int)a[2];
  int iM = d1_index(a, offM, m);
  int offC = (int)a[3 + iM];
  int iC = d1_index(a, offC, c);
  float mr = d1_remap(a, offM, m, iM), cr = d1_remap(a, offC, c, iC);
  *ou = uv ? mr : cr; *ov = uv ? cr : mr;
}
DFC_D float d2_pdf(const float* a, float su, float sv) {
  bool uv = (int)a[0] != 0;
  float m = uv ? su : sv, c = uv ? sv : su;
  int offM = (int)a[2];
  int nM = (int)a[offM + 2];
  int iM = max(0, min((int)(m * nM), nM - 1));
  int offC = (int)a[3 + iM];
  int nC = (int)a[offC + 2];
  int iC = max(0, min((int)(c * nC), nC - 1));
  return a[offC + 4 + iC + (int)a[offC + 1]] / a[offM + 3];
}

// The sky models and the light sampling and pdf routines below are large
// (perez_sky alone evaluates 15 exponentials) and are reached from several
// places of a shading kernel; compiled out of line they are held once in the
// instruction cache instead of once per call site.
#ifndef DFC_LIGHT_NOINLINE
#define DFC_LIGHT_NOINLINE 1
#endif
#if DFC_LIGHT_NOINLINE
#define DFC_LIGHT_FN static __device__ __noinline__
#else
#define DFC_LIGHT_FN DFC_D
#endif

// scene/light/PerezLight.java doRadianceSky (renderer/gpu/AbstractLightKernel.java:1615 form).
DFC_LIGHT_FN V3 perez_sky(const float* q, V3 dir) {
  if (dir.z < 0.0f) return {0, 0, 0};
  V3 ds = normalize(V3{dir.x, dir.y, fmaxf(dir.z, 0.001f)});
  const float T = q[41];
  const float theta = acosf(clampf(ds.z, -1.0f, 1.0f));
  const float gamma = acosf(clampf(dot(ds, ld3(q + 35)), -1.0f, 1.0f));
  const float thS = q[46], cs = cosf(thS), cs2 = cs * cs, cg = cosf(gamma), cg2 = cg * cg, ict = 1.0f / cosf(theta);
  auto perez = [&](float l0, float l1, float l2, float l3, float l4, float z) {
    return z * ((1.0f + l0 * expf(l1 * ict)) * (1.0f + l2 * expf(l3 * gamma) + l4 * cg2)) / ((1.0f + l0 * expf(l1)) * (1.0f + l2 * expf(l3 * thS) + l4 * cs2));
  };
  float Y = perez(0.17872f * T - 1.46303f, -0.35540f * T + 0.42749f, -0.02266f * T + 5.32505f, 0.12064f * T - 2.57705f, -0.06696f * T + 0.37027f, q[42]) * 0.0001f;
  float x = perez(-0.01925f * T - 0.25922f, -0.06651f * T + 0.00081f, -0.00041f * T + 0.21247f, -0.06409f * T - 0.89887f, -0.00325f * T + 0.04517f, q[43]);
  float y = perez(-0.01669f * T - 0.26078f, -0.09495f * T + 0.00921f, -0.00792f * T + 0.21023f, -0.04405f * T - 1.65369f, -0.01092f * T + 0.05291f, q[44]);
  float den = 0.0241f + 0.2562f * x - 0.7341f * y;
  float m1 = (-1.3515f - 1.7703f * x + 5.9114f * y) / den;
  float m2 = (0.03f - 31.4424f * x + 30.0717f * y) / den;
  float X = 95.6824722290f + m1 * 1.7548348904f + m2 * 1.9917192459f;
  float Yc = 99.7036819458f + m1 * 1.8025954962f + m2 * 0.7136800885f;
  float Z = 115.5248031616f + m1 * 32.5218048096f + m2 * -2.1984319687f;
  float cx = X * Y / Yc, cy = Y, cz = Z * Y / Yc;
  // sRGB XYZ -> RGB (color/ColorSpaceF.java:85), matrix derived from the sRGB primaries
  return {3.2404542f * cx - 1.5371385f * cy - 0.4985314f * cz, -0.9692660f * cx + 1.8760108f * cy + 0.0415560f * cz,
          0.0556434f * cx - 0.2040259f * cy + 1.0572252f * cz};
}
DFC_D V3 sat0(V3 c) { return {fmaxf(c.x, 0.0f), fmaxf(c.y, 0.0f), fmaxf(c.z, 0.0f)}; }

// scene/light/ImageLight.java:544 doRadianceSky over the compiled record
// (CompiledLightCache.java:1393-1460: angle +32, scale +33, resolution +36,
// distribution +40, RGB image +2352): spherical texture coordinates, rotated
// counterclockwise, scaled, mapped to pixels (Point2F.toImage) and read with
// bilinear interpolation and wrap-around (ImageF.getColorRGB).
DFC_LIGHT_FN V3 image_sky(const float* q, V3 d) {
  float phi = atan2f(d.y, d.x);
  if (phi < 0.0f) phi += 2.0f * kPi;
  const float theta = acosf(clampf(d.z, -1.0f, 1.0f));
  const float u = phi * (1.0f / (2.0f * kPi)), v = theta * (1.0f / kPi);
  float s, c;
  sincosf(q[32], &s, &c);
  const float us = (u * c - v * s) * q[33], vs = (v * c + u * s) * q[34];
  const float rx = q[36], ry = q[37];
  auto posmod = [](float x, float y) { return x < 0.0f ? fmodf(fmodf(x, y) + y, y) : fmodf(x, y); };
  const float x = posmod(us * rx - 0.5f, rx), y = posmod(vs * ry - 0.5f, ry);
  const int w = (int)rx, h = (int)ry;
  const int x0 = (int)floorf(x), x1 = (int)ceilf(x), y0 = (int)floorf(y), y1 = (int)ceilf(y);
  auto px = [&](int ix, int iy) {
    ix = ((ix % w) + w) % w;
    iy = ((iy % h) + h) % h;
    const float* p = q + 2352 + ((size_t)iy * (size_t)w + (size_t)ix) * 3;
    return V3{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
  };
  if (x0 == x1 && y0 == y1) return px(x0, y0);
  const float xf = x - (float)x0, yf = y - (float)y0;
  auto lerp3 = [](V3 a, V3 b, float t) { return V3{lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t)}; };
  return lerp3(lerp3(px(x0, y0), px(x1, y0), xf), lerp3(px(x0, y1), px(x1, y1), xf), yf);
}

// A light sample; the out-of-line samplers return pdf 0 for no sample (every
// caller skips a sample whose pdf is not positive).
struct LightS { V3 L, p, wi; float pdf; };

// DiffuseAreaLight.sampleRadianceIncoming for a triangle or sphere shape.
DFC_LIGHT_FN LightS area_light_sample(const float* tri_attr, const DLight& lt, V3 p, float u, float v) {
  V3 ref = xf_point(lt.w2o, p);
  V3 sp, sn;
  float pdf;
  if (lt.shape == kShapeTriangle) {
    // Triangle3F.sample(Point2F) + Shape3F.sample(sample, ref): the solid-angle
    // pdf there is dist^2/|cos| (the area density of the point is not applied).
    const float* q = tri_attr + (size_t)lt.shape_data * 24;
    float su = sqrtf(u), b0 = 1.0f - su, b1 = v * su, b2 = 1.0f - b0 - b1;
    V3 A = ld3(q), B = ld3(q + 3), C = ld3(q + 6);
    sp = {A.x * b0 + B.x * b1 + C.x * b2, A.y * b0 + B.y * b1 + C.y * b2, A.z * b0 + B.z * b1 + C.z * b2};
    sn = normalize(ld3(q + 15) * b0 + ld3(q + 18) * b1 + ld3(q + 21) * b2);
    V3 inc = sp - ref;
    if (dot(inc, inc) == 0.0f) return LightS{};
    V3 incn = normalize(inc);
    pdf = dot(inc, inc) / fabsf(dot(sn, -incn));
    if (isinf(pdf) || isnan(pdf)) return LightS{};
  } else if (lt.shape == kShapeSphere) {
    if (dot(ref, ref) <= 1.0f) {
      float ct = 1.0f - 2.0f * u, st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct)), s, c;
      sincosf(v * 2.0f * kPi, &s, &c);
      sp = {st * c, st * s, ct};
      sn = normalize(sp);
      V3 inc = sp - ref;
      if (dot(inc, inc) == 0.0f) return LightS{};
      pdf = dot(inc, inc) / fabsf(dot(sn, -normalize(inc)));
      if (isinf(pdf) || isnan(pdf)) return LightS{};
    } else {
      float dist = len(ref), dr = 1.0f / dist;
      V3 dc = (-ref) * dr;
      ONB b = onb_w(dc);
      float stm2 = dr * dr, stmr = dist;
      float ctm = sqrtf(fmaxf(0.0f, 1.0f - stm2));
      float ct = stm2 < 0.00068523f ? sqrtf(1.0f - stm2 * u) : (ctm - 1.0f) * u + 1.0f;
      float st2 = stm2 < 0.00068523f ? stm2 * u : 1.0f - ct * ct;
      float ca = st2 * stmr + ct * sqrtf(fmaxf(0.0f, 1.0f - st2 * stmr * stmr));
      float sa = sqrtf(fmaxf(0.0f, 1.0f - ca * ca)), s, c;
      sincosf(v * 2.0f * kPi, &s, &c);
      V3 sd = (-b.u) * (sa * c) + (-b.v) * (sa * s) + (-b.w) * ca;
      sp = sd; sn = normalize(sd); pdf = 1.0f / (2.0f * kPi * (1.0f - ctm));
    }
  } else {
    return LightS{};  // Shape3F.sample default: no sample for other shapes
  }
  V3 pw = xf_point(lt.o2w, sp);
  V3 nw = normalize(xf_vec_t(lt.w2o, sn));
  V3 wi = normalize(pw - p);
  if (pdf > 0.0f && (lt.two_sided || dot(nw, -wi) > 0.0f)) return LightS{ld3(lt.radiance), pw, wi, pdf};
  return LightS{};
}

// PerezLight and ImageLight (scene/light/ImageLight.java:207) sampleRadianceIncoming;
// q is the light's record in the sky pool, gw and sw the surface's geometric and
// shading normals.
DFC_LIGHT_FN LightS sky_light_sample(const float* q, int type, V3 p, V3 gw, V3 sw, float u, float v, float sun_pick) {
  if (type == kLightPerez) {
    const float* dist = q + 48;
    V3 sunW = ld3(q + 38), sunO = ld3(q + 35);
    if (dot(sunW, gw) > sun_pick && dot(sunW, sw) > sun_pick) {
      float st = sint(sunO);
      if (st != 0.0f) {
        float phi = atan2f(sunO.y, sunO.x);
        if (phi < 0.0f) phi += 2.0f * kPi;
        float pdf = d2_pdf(dist, phi * (1.0f / (2.0f * kPi)), acosf(clampf(sunO.z, -1.0f, 1.0f)) * (1.0f / kPi)) / (2.0f * kPi * kPi * st);
        if (pdf != 0.0f) return LightS{ld3(q + 32), p + sunW * (2.0f * q[45]), sunW, pdf};
      }
    }
    float ru, rv;
    d2_remap(dist, u, v, &ru, &rv);
    float pr = d2_pdf(dist, ru, rv);
    if (pr == 0.0f) return LightS{};
    float sth, cth, sph, cph;
    sincosf(rv * kPi, &sth, &cth);
    sincosf(ru * 2.0f * kPi, &sph, &cph);
    V3 dobj = {sth * cph, sth * sph, cth};
    V3 dw = normalize(xf_vec(q, dobj));
    float st = sint(dobj);
    if (st == 0.0f) return LightS{};
    return LightS{sat0(perez_sky(q, dobj)), p + dw * (2.0f * q[45]), dw, pr / (2.0f * kPi * kPi * st)};
  }
  float ru, rv;
  d2_remap(q + 40, u, v, &ru, &rv);
  const float pr = d2_pdf(q + 40, ru, rv);
  if (pr == 0.0f) return LightS{};
  float sth, cth, sph, cph;
  sincosf(rv * kPi, &sth, &cth);
  sincosf(ru * 2.0f * kPi, &sph, &cph);
  const V3 dobj = {sth * cph, sth * sph, cth};
  const V3 dw = normalize(xf_vec(q, dobj));
  const float st = sint(dobj);
  if (st == 0.0f) return LightS{};
  return LightS{image_sky(q, dobj), p + dw * (2.0f * q[35]), dw, pr / (2.0f * kPi * kPi * st)};
}

// Light.sampleRadianceIncoming for each supported light type.
DFC_D bool light_sample(const SceneView& S, const DLight& lt, const Surface& sf, float u, float v, float sun_pick, LightS* o) {
  const V3 p = sf.p;
  switch (lt.type) {
    case kLightDiffuseArea: *o = area_light_sample(S.tri_attr, lt, p, u, v); return o->pdf > 0.0f;
    case kLightPoint: {
      V3 pos = ld3(lt.pos);
      V3 d = pos - p;
      *o = LightS{ld3(lt.radiance) * (1.0f / dot(d, d)), pos, normalize(d), 1.0f};
      return true;
    }
    case kLightSpot: {
      V3 pos = ld3(lt.pos);
      V3 d = pos - p;
      V3 wi = normalize(d);
      V3 dobj = normalize(xf_vec(lt.w2o, -wi));
      float ct = dobj.z, fall;
      if (ct < lt.cos_cone) fall = 0.0f;
      else if (ct >= lt.cos_cone_delta) fall = 1.0f;
      else { float t = (ct - lt.cos_cone) / (lt.cos_cone_delta - lt.cos_cone); fall = (t * t) * (t * t); }
      *o = LightS{ld3(lt.radiance) * (fall / dot(d, d)), pos, wi, 1.0f};
      return true;
    }
    case kLightDirectional: {
      V3 d = ld3(lt.dir);
      *o = LightS{ld3(lt.radiance), p + d * (2.0f * lt.radius), d, 1.0f};
      return true;
    }
    case kLightPerez:
    case kLightImage: *o = sky_light_sample(S.perez + lt.perez, lt.type, p, sf.g.w, sf.s.w, u, v, sun_pick); return o->pdf > 0.0f;
  }
  return false;
}

DFC_D bool light_is_delta(int type) { return type == kLightPoint || type == kLightSpot || type == kLightDirectional; }

// Light.evaluateRadianceEmitted(Ray3F): only the sky lights (Perez, image) emit along a missed ray.
DFC_D V3 light_Le_miss(const SceneView& S, const DLight& lt, V3 d) {
  if (lt.type != kLightPerez && lt.type != kLightImage) return {0, 0, 0};
  const float* q = S.perez + lt.perez;
  const V3 dobj = normalize(xf_vec(q + 16, d));
  return lt.type == kLightPerez ? sat0(perez_sky(q, dobj)) : image_sky(q, dobj);
}

// Light.evaluateProbabilityDensityFunctionRadianceIncoming of the sky lights
// (PerezLight, ImageLight.java:348); their distribution starts at +48 and +40.
DFC_LIGHT_FN float sky_pdf_q(const float* q, int type, V3 wi) {
  V3 d = normalize(xf_vec(q + 16, wi));
  float th = acosf(clampf(d.z, -1.0f, 1.0f));
  float st = sinf(th);
  if (st == 0.0f) return 0.0f;
  float phi = atan2f(d.y, d.x);
  if (phi < 0.0f) phi += 2.0f * kPi;
  return d2_pdf(q + (type == kLightPerez ? 48 : 40), phi * (1.0f / (2.0f * kPi)), th * (1.0f / kPi)) / (2.0f * kPi * kPi * st);
}
DFC_D float sky_pdf(const SceneView& S, const DLight& lt, V3 wi) { return sky_pdf_q(S.perez + lt.perez, lt.type, wi); }

}  // namespace dfc
