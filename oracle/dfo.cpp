// dfo: a CPU restatement of Dayflower's CPURenderer over the scene compiler's
// flattened arrays.  TEST INFRASTRUCTURE ONLY: tests/, the smoke check and the
// benchmark's CPU-baseline leg use it as the checker; the renderer product
// never links, loads or calls it.
//
// What it restates (paths relative to src/main/java/org/dayflower/):
//   scene/Scene.java:272-345 (ambient occlusion, depth camera), :451-619 (path
//   tracer), :675-701 (ray caster), :797-813 (one-light sampling), :874-894
//   (linear primitive loop), :1066-1090 (light visibility), :1530-1640 (direct
//   lighting with MIS); scene/Intersector.java; geometry/SurfaceIntersector3F.java;
//   geometry/SurfaceIntersection3F.java:372 (object->world); the shapes under
//   geometry/shape/ (Sphere3F, Triangle3F, TriangleMesh3F, Rectangle3F, Plane3F);
//   scene/BSDF.java; scene/bxdf/*; scene/microfacet/TrowbridgeReitzMicrofacetDistribution.java;
//   scene/fresnel/*; scene/light/{DiffuseAreaLight,PointLight,SpotLight,
//   DirectionalLight,PerezLight}.java; sampler/Distribution{1,2}F.java;
//   renderer/cpu/AbstractCPURenderer.java:215-246 (pixel loop + film guard).
//
// The input format is the one renderer/gpu/AbstractSceneKernel.java:1777-1852
// uploads (CompiledScene arrays, same names), decoded here independently of
// the device renderer's ingest.
#include "dfo_math.h"
#include "dfo_noise.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace dfo {

// ---- type ids (scene classes' public static final int ID) -------------------
enum { kBVAabb = 1, kBVSphere = 2, kBVInfinite = 3 };
enum { kShapeCone = 2, kShapeCylinder = 5, kShapeDisk = 6, kShapeHyperboloid = 7, kShapeParaboloid = 9, kShapePlane = 10,
       kShapePolygon = 11, kShapeRectangle = 13, kShapeCuboid = 14, kShapeSphere = 15, kShapeTorus = 16, kShapeTriangle = 17,
       kShapeMesh = 18 };
enum {
  kMatClearCoat = 3, kMatDisney = 4, kMatGlass = 7, kMatGlossy = 8, kMatMatte = 11, kMatMetal = 12, kMatMirror = 13, kMatPlastic = 14,
  kMatSubstrate = 16, kMatTranslucent = 18, kMatUber = 19,
  kMatBullseye = 1, kMatCheckerboard = 2, kMatPolkaDot = 15  // composite: pick material A or B per hit
};
enum {  // scene/texture/*Texture.java ID
  kTexBlend = 1, kTexBullseye = 2, kTexCheckerboard = 3, kTexConstant = 4, kTexDotProduct = 5, kTexLDRImage = 7, kTexMarble = 8,
  kTexPolkaDot = 9, kTexSimplexFBM = 10, kTexSurfaceNormal = 11, kTexUV = 12
};
enum { kModNoOp = 2, kModNormalMapLDRImage = 3, kModSimplexNoiseNormalMap = 4 };  // scene/modifier/*Modifier.java ID
enum { kLightDiffuseArea = 1, kLightDirectional = 2, kLightImage = 3, kLightPerez = 4, kLightPoint = 5, kLightSpot = 7 };
enum { kAlgoAO = 0, kAlgoDepth = 1, kAlgoPath = 2, kAlgoRayCast = 3, kAlgoRayTrace = 4 };

struct Scene {
  std::map<std::string, std::vector<float>> f;
  std::map<std::string, std::vector<int32_t>> i;
  int layout = 1;
  int prim_count = 0;
  std::vector<int32_t> prims;  // 8 ints per primitive
  std::vector<M44> o2w, w2o;
  std::vector<int32_t> lights;  // lightIDAndOffsetArray
  float cam[19];
  std::string err;

  const std::vector<float>& F(const char* n) const { static const std::vector<float> e; auto it = f.find(n); return it == f.end() ? e : it->second; }
  const std::vector<int32_t>& I(const char* n) const { static const std::vector<int32_t> e; auto it = i.find(n); return it == i.end() ? e : it->second; }
};

// ---- EFloat (utility/EFloat.java) ------------------------------------------
struct EF { float v, lo, hi; };
inline EF ef(float v) { return EF{v, v, v}; }
inline EF ef(float v, float err) { return err == 0.0f ? ef(v) : EF{v, next_down(v - err), next_up(v + err)}; }
inline EF ef_add(EF a, EF b) { return EF{a.v + b.v, next_down(a.lo + b.lo), next_up(a.hi + b.hi)}; }
inline EF ef_sub(EF a, EF b) { return EF{a.v - b.v, next_down(a.lo - b.hi), next_up(a.hi - b.lo)}; }
inline EF ef_mul(EF a, EF b) {
  float p0 = a.lo * b.lo, p1 = a.hi * b.lo, p2 = a.lo * b.hi, p3 = a.hi * b.hi;
  return EF{a.v * b.v, next_down(std::fmin(std::fmin(p0, p1), std::fmin(p2, p3))), next_up(std::fmax(std::fmax(p0, p1), std::fmax(p2, p3)))};
}
inline EF ef_div(EF a, EF b) {
  float v = a.v / b.v;
  if (b.lo < 0.0f && b.hi > 0.0f) return EF{v, -INFINITY, INFINITY};
  float d0 = a.lo / b.lo, d1 = a.hi / b.lo, d2 = a.lo / b.hi, d3 = a.hi / b.hi;
  return EF{v, next_down(std::fmin(std::fmin(d0, d1), std::fmin(d2, d3))), next_up(std::fmax(std::fmax(d0, d1), std::fmax(d2, d3)))};
}
// utility/EFloat.java:165
inline bool ef_quadratic(EF a, EF b, EF c, EF* t0, EF* t1) {
  double discrim = (double)b.v * (double)b.v - 4.0 * a.v * c.v;
  if (discrim < 0.0) return false;
  double root = std::sqrt(discrim);
  EF fr = ef((float)root, kMachineEpsilon() * (float)root);
  EF q = b.v < 0.0f ? ef_mul(ef(-0.5f), ef_sub(b, fr)) : ef_mul(ef(-0.5f), ef_add(b, fr));
  *t0 = ef_div(q, a);
  *t1 = ef_div(c, q);
  if (t0->v > t1->v) std::swap(*t0, *t1);
  return true;
}

// ---- surface intersection records ------------------------------------------
struct Surface {  // geometry/SurfaceIntersection3F.java
  ONB g, s;
  float tu, tv;
  V3 p;
  Ray ray;
  float t;
};

struct Tri { V3 a, b, c; float uva[2], uvb[2], uvc[2]; V3 na, nb, nc; };
inline Tri load_tri(const std::vector<float>& T, int off) {
  Tri t;
  const float* q = T.data() + off;
  t.a = {q[0], q[1], q[2]}; t.b = {q[3], q[4], q[5]}; t.c = {q[6], q[7], q[8]};
  t.uva[0] = q[9]; t.uva[1] = q[10]; t.uvb[0] = q[11]; t.uvb[1] = q[12]; t.uvc[0] = q[13]; t.uvc[1] = q[14];
  t.na = {q[15], q[16], q[17]}; t.nb = {q[18], q[19], q[20]}; t.nc = {q[21], q[22], q[23]};
  return t;
}

// geometry/shape/Triangle3F.java:505-596 (watertight test with its tScaled/tMinimum comparison)
inline float triangle_t(const Tri& tr, const Ray& r, float tmin, float tmax) {
  V3 p0 = tr.a - r.o, p1 = tr.b - r.o, p2 = tr.c - r.o;
  V3 ad = {std::fabs(r.d.x), std::fabs(r.d.y), std::fabs(r.d.z)};
  int kz = (ad.x > ad.y) ? (ad.x > ad.z ? 0 : 2) : (ad.y > ad.z ? 1 : 2);  // Vector3F.getMaxDimension
  int kx = kz + 1; if (kx == 3) kx = 0;
  int ky = kx + 1; if (ky == 3) ky = 0;
  auto perm = [&](V3 v) { float c[3] = {v.x, v.y, v.z}; return V3{c[kx], c[ky], c[kz]}; };
  V3 d = perm(r.d);
  p0 = perm(p0); p1 = perm(p1); p2 = perm(p2);
  float sx = -d.x / d.z, sy = -d.y / d.z, sz = 1.0f / d.z;
  p0 = {p0.x + sx * p0.z, p0.y + sy * p0.z, p0.z};
  p1 = {p1.x + sx * p1.z, p1.y + sy * p1.z, p1.z};
  p2 = {p2.x + sx * p2.z, p2.y + sy * p2.z, p2.z};
  float e0 = p1.x * p2.y - p1.y * p2.x;
  float e1 = p2.x * p0.y - p2.y * p0.x;
  float e2 = p0.x * p1.y - p0.y * p1.x;
  if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
    e0 = (float)((double)p2.y * (double)p1.x - (double)p2.x * (double)p1.y);
    e1 = (float)((double)p0.y * (double)p2.x - (double)p0.x * (double)p2.y);
    e2 = (float)((double)p1.y * (double)p0.x - (double)p1.x * (double)p0.y);
  }
  if ((e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) && (e0 > 0.0f || e1 > 0.0f || e2 > 0.0f)) return NAN;
  float det = e0 + e1 + e2;
  if (det == 0.0f) return NAN;
  p0.z *= sz; p1.z *= sz; p2.z *= sz;
  float ts = e0 * p0.z + e1 * p1.z + e2 * p2.z;
  if (det < 0.0f && (ts >= tmin || ts < tmax * det)) return NAN;
  if (det > 0.0f && (ts <= tmin || ts > tmax * det)) return NAN;
  float inv = 1.0f / det;
  float t = ts * inv;
  float mz = max_component(V3{std::fabs(p0.z), std::fabs(p1.z), std::fabs(p2.z)});
  float mx = max_component(V3{std::fabs(p0.x), std::fabs(p1.x), std::fabs(p2.x)});
  float my = max_component(V3{std::fabs(p0.y), std::fabs(p1.y), std::fabs(p2.y)});
  float dz = gamma_n(3) * mz;
  float dx = gamma_n(5) * (mx + mz);
  float dy = gamma_n(5) * (my + mz);
  float de = 2.0f * (gamma_n(2) * mx * my + dy * mx + dx * my);
  float me = max_component(V3{std::fabs(e0), std::fabs(e1), std::fabs(e2)});
  float dt = 3.0f * (gamma_n(3) * me * mz + de * mz + dz * me) * std::fabs(inv);
  if (t <= dt) return NAN;
  return t;
}

// geometry/shape/Triangle3F.java:1070-1160
inline Surface triangle_surface(const Tri& tr, const Ray& r, float t) {
  Surface s;
  V3 eab = tr.b - tr.a, eca = tr.a - tr.c;
  V3 d1 = cross(eab, eca);
  float det = dot(r.d, d1);
  float inv = 1.0f / det;
  V3 d2 = tr.a - r.o;
  V3 d3 = cross(d2, r.d);
  float bu = dot(d3, eca) * inv;
  float bv = dot(d3, eab) * inv;
  float bw = 1.0f - bu - bv;  // barycentric (w, u, v) weights A, B, C
  s.p = r.o + r.d * t;
  s.tu = tr.uva[0] * bw + tr.uvb[0] * bu + tr.uvc[0] * bv;
  s.tv = tr.uva[1] * bw + tr.uvb[1] * bu + tr.uvc[1] * bv;
  V3 ng = normalize(cross(normalize(tr.b - tr.a), normalize(tr.c - tr.a)));
  s.g = onb_from_w(ng);
  V3 w = normalize(tr.na * bw + tr.nb * bu + tr.nc * bv);
  float tca0 = tr.uva[0] - tr.uvc[0], tca1 = tr.uva[1] - tr.uvc[1];
  float tcb0 = tr.uvb[0] - tr.uvc[0], tcb1 = tr.uvb[1] - tr.uvc[1];
  float d = tca0 * tcb1 - tca1 * tcb0;  // Vector2F.crossProduct
  if (d == 0.0f) {
    s.s = onb_from_w(w);
  } else {
    float rd = 1.0f / d;
    V3 ec = tr.a - tr.c, eb = tr.b - tr.c;
    V3 v = {(-tcb0 * ec.x + tca0 * eb.x) * rd, (-tcb0 * ec.y + tca0 * eb.y) * rd, (-tcb0 * ec.z + tca0 * eb.z) * rd};
    s.s = onb_from_wv(w, v);
  }
  s.ray = r; s.t = t;
  return s;
}

inline float triangle_area(const Tri& tr) { return length(cross(tr.b - tr.a, tr.c - tr.a)) * 0.5f; }

// geometry/boundingvolume/AxisAlignedBoundingBox3F.java:238, :309
inline bool aabb_contains_or_intersects(const float* bb, const Ray& r, float tmin, float tmax) {
  V3 mx = {bb[0], bb[1], bb[2]}, mn = {bb[3], bb[4], bb[5]};
  if (r.o.x >= mn.x && r.o.x <= mx.x && r.o.y >= mn.y && r.o.y <= mx.y && r.o.z >= mn.z && r.o.z <= mx.z) return true;
  V3 rc = {1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z};
  V3 a = {(mx.x - r.o.x) * rc.x, (mx.y - r.o.y) * rc.y, (mx.z - r.o.z) * rc.z};
  V3 b = {(mn.x - r.o.x) * rc.x, (mn.y - r.o.y) * rc.y, (mn.z - r.o.z) * rc.z};
  float t0 = std::fmax(std::fmax(std::fmin(a.x, b.x), std::fmin(a.y, b.y)), std::fmin(a.z, b.z));
  float t1 = std::fmin(std::fmin(std::fmax(a.x, b.x), std::fmax(a.y, b.y)), std::fmax(a.z, b.z));
  if (t0 > t1) return false;
  if (t0 > tmin && t0 < tmax) return true;
  if (t1 > tmin && t1 < tmax) return true;
  return false;
}

// geometry/boundingvolume/BoundingSphere3F.java:238, :317 (Floats.solveQuadraticSystem)
inline bool bsphere_contains_or_intersects(const float* bs, const Ray& r, float tmin, float tmax) {
  V3 c = {bs[0], bs[1], bs[2]};
  float r2 = bs[3] * bs[3];
  if (distance_squared(c, r.o) <= r2) return true;
  V3 co = r.o - c;
  float a = dot(r.d, r.d), b = 2.0f * dot(co, r.d), cc = dot(co, co) - r2;
  float disc = b * b - 4.0f * a * cc;
  if (disc < 0.0f) return false;
  float sq = std::sqrt(disc);
  float q = b < 0.0f ? -0.5f * (b - sq) : -0.5f * (b + sq);
  float t0 = q / a, t1 = cc / q;
  if (t0 > t1) std::swap(t0, t1);
  if (t0 > tmin && t0 < tmax) return true;
  if (t1 > tmin && t1 < tmax) return true;
  return false;
}

// geometry/shape/Sphere3F.java:507 (unit sphere; the compiled scene has no sphere data)
struct SphereHit { float t; V3 p; };
inline bool sphere_hit(const Ray& r, float tmin, float tmax, SphereHit* out) {
  EF ox = ef(r.o.x), oy = ef(r.o.y), oz = ef(r.o.z), dx = ef(r.d.x), dy = ef(r.d.y), dz = ef(r.d.z);
  EF a = ef_add(ef_add(ef_mul(dx, dx), ef_mul(dy, dy)), ef_mul(dz, dz));
  EF b = ef_mul(ef(2.0f), ef_add(ef_add(ef_mul(dx, ox), ef_mul(dy, oy)), ef_mul(dz, oz)));
  EF c = ef_sub(ef_add(ef_add(ef_mul(ox, ox), ef_mul(oy, oy)), ef_mul(oz, oz)), ef_mul(ef(1.0f), ef(1.0f)));
  EF t0, t1;
  if (!ef_quadratic(a, b, c, &t0, &t1)) return false;
  if (t0.hi > tmax || t1.lo <= tmin) return false;
  EF th = t0;
  bool second = false;
  if (th.lo <= 0.0f) { th = t1; second = true; if (th.hi > tmax) return false; }
  V3 p = r.o + r.d * th.v;
  float s = 1.0f / distance(V3{0, 0, 0}, p);
  p = p * s;
  if (p.x == 0.0f && p.y == 0.0f) p.x = 1.0e-5f;
  (void)second;
  // A full sphere (zMin = -r, zMax = r, phiMax = 2 pi) never clips.
  out->t = th.v; out->p = p;
  return true;
}

inline Surface sphere_surface(const Ray& r, const SphereHit& h) {
  Surface s;
  V3 p = h.p;
  float phi = std::atan2(p.y, p.x);
  if (phi < 0.0f) phi += 2.0f * kPi;
  const float phiMax = 2.0f * kPi, thetaMin = kPi, thetaMax = 0.0f;  // acos(-1), acos(1)
  float u = phi / phiMax;
  float theta = std::acos(saturate(p.z, -1.0f, 1.0f));
  float v = (theta - thetaMin) / (thetaMax - thetaMin);
  float zr = std::sqrt(p.x * p.x + p.y * p.y);
  float zri = 1.0f / zr;
  float cphi = p.x * zri, sphi = p.y * zri;
  V3 dpdu = {-phiMax * p.y, phiMax * p.x, 0.0f};
  V3 dpdv = V3{p.z * cphi, p.z * sphi, -1.0f * std::sin(theta)} * (thetaMax - thetaMin);
  V3 n = normalize(cross(dpdu, dpdv));
  s.g = ONB{n, dpdv, dpdu};  // OrthonormalBasis33F(w, v, u) stores the vectors as given
  s.s = s.g;
  s.tu = u; s.tv = v; s.p = p; s.ray = r; s.t = h.t;
  return s;
}

// geometry/shape/Rectangle3F.java:368 (compiled: position a, sideA = b - a, sideB = c - b)
struct Rect { V3 a, b, c, d, n; };
inline Rect load_rect(const std::vector<float>& R, int off) {
  const float* q = R.data() + off;
  Rect r;
  r.a = {q[0], q[1], q[2]};
  V3 sa = {q[3], q[4], q[5]}, sb = {q[6], q[7], q[8]};
  r.b = r.a + sa; r.c = r.b + sb; r.d = r.a + sb;
  r.n = {q[9], q[10], q[11]};
  return r;
}
inline float rect_t(const Rect& q, const Ray& r, float tmin, float tmax) {
  float dp = dot(q.n, r.d);
  if (dp == 0.0f) return NAN;
  float t = dot(q.a - r.o, q.n) / dp;
  if (t <= tmin || t >= tmax) return NAN;
  V3 ab = q.b - q.a, bc = q.c - q.b, ap = (r.o + r.d * t) - q.a;
  float x = dot(ap, normalize(ab)), y = dot(ap, normalize(bc));
  if (x >= 0.0f && x <= length(ab) && y >= 0.0f && y <= length(bc)) return t;
  return NAN;
}
inline Surface rect_surface(const Rect& q, const Ray& r, float t) {
  Surface s;
  s.p = r.o + r.d * t;
  s.g = onb_from_w(q.n); s.s = s.g;
  V3 na = {std::fabs(q.n.x), std::fabs(q.n.y), std::fabs(q.n.z)};
  bool isX = na.x > na.y && na.x > na.z, isY = na.y > na.z;
  auto proj = [&](V3 p, float* o) {
    if (isX) { o[0] = p.y; o[1] = p.z; } else if (isY) { o[0] = p.z; o[1] = p.x; } else { o[0] = p.x; o[1] = p.y; }
  };
  float vA[2], vB[2], vC[2];
  proj(q.a, vA); proj(q.d, vB); proj(q.b, vC);
  float vAB[2] = {vB[0] - vA[0], vB[1] - vA[1]}, vAC[2] = {vC[0] - vA[0], vC[1] - vA[1]};
  float det = vAB[0] * vAC[1] - vAB[1] * vAC[0];
  float di = 1.0f / det;
  float h[2]; proj(s.p, h);
  s.tu = h[0] * (-vAB[1] * di) + h[1] * (vAB[0] * di) + (vA[0] * vAB[1] - vA[1] * vAB[0]) * di;
  s.tv = h[0] * (vAC[1] * di) + h[1] * (-vAC[0] * di) + (vAC[0] * vA[1] - vAC[1] * vA[0]) * di;
  s.ray = r; s.t = t;
  return s;
}

// geometry/shape/Plane3F.java (unit plane z = 0 in object space)
inline float plane_t(const Ray& r, float tmin, float tmax) {
  float dp = r.d.z;
  if (dp == 0.0f) return NAN;
  float t = -r.o.z / dp;  // dot(direction(origin, 0), z) / dp
  if (t > tmin && t < tmax) return t;
  return NAN;
}
inline Surface plane_surface(const Ray& r, float t) {
  Surface s;
  s.p = r.o + r.d * t;
  s.g = ONB{V3{0, 0, 1}, V3{0, 1, 0}, V3{1, 0, 0}}; s.s = s.g;
  s.tu = s.p.x; s.tv = s.p.y; s.ray = r; s.t = t;
  return s;
}

// ---- quadric, disk, box and torus shapes -----------------------------------
// The CPU shapes call org.macroing.java.lang.Floats, which is not vendored; its
// routines are restated from the same author's utility/Floats.java.

// java.lang.Math.min/max on floats: NaN propagates, -0 < +0.
inline float jmin(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == 0.0f && b == 0.0f) return std::signbit(a) ? a : b;
  return a <= b ? a : b;
}
inline float jmax(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == 0.0f && b == 0.0f) return std::signbit(a) ? b : a;
  return a >= b ? a : b;
}

// geometry/Point3F.java:223 sphericalPhi (Floats.atan2 is Math.atan2 in double)
inline float spherical_phi(float x, float y) {
  float phi = (float)std::atan2((double)y, (double)x);
  return phi < 0.0f ? phi + 2.0f * kPi : phi;
}

// utility/Floats.java:1227 solveQuadraticSystem: {NaN, NaN} without real roots.
inline void solve_quadratic(float a, float b, float c, float* r0, float* r1) {
  const float disc2 = b * b - 4.0f * a * c;
  *r0 = NAN; *r1 = NAN;
  if (disc2 == 0.0f) {
    const float q = -0.5f * b / a;
    *r0 = q; *r1 = q;
  } else if (disc2 > 0.0f) {
    const float disc = std::sqrt(disc2);
    const float q = -0.5f * (b > 0.0f ? b + disc : b - disc);
    const float x0 = q / a, x1 = c / q;
    *r0 = jmin(x0, x1); *r1 = jmax(x0, x1);
  }
}

inline V3 point_at(const Ray& r, float t) { return V3{r.o.x + r.d.x * t, r.o.y + r.d.y * t, r.o.z + r.d.z * t}; }
inline float len2d(V3 p) { return std::sqrt(p.x * p.x + p.y * p.y); }

// The quadrics share one loop: the first root in (tmin, tmax) whose point
// passes `inside` wins; a NaN root ends the search (Cylinder3F.java:342 and
// the same method of Cone3F, Paraboloid3F, Hyperboloid3F).
template <typename PointF, typename InsideF>
inline float quadric_t(float a, float b, float c, const Ray& r, float tmin, float tmax, PointF point, InsideF inside) {
  float ts[2];
  solve_quadratic(a, b, c, &ts[0], &ts[1]);
  for (int i = 0; i < 2; ++i) {
    const float t = ts[i];
    if (t != t) return NAN;
    if (t > tmin && t < tmax && inside(point(r, t))) return t;
  }
  return NAN;
}

inline ONB uv_frame(V3 u, V3 v) {
  u = normalize(u);
  v = normalize(v);
  return ONB{cross(u, v), v, u};
}

inline Surface simple_surface(const Ray& r, float t, V3 p, ONB g, float tu, float tv) {
  Surface s;
  s.g = g; s.s = g; s.tu = tu; s.tv = tv; s.p = p; s.ray = r; s.t = t;
  return s;
}

// geometry/shape/Disk3F.java:342 (record: phiMax, radiusInner, radiusOuter, zMax)
inline float disk_t(const float* q, const Ray& r, float tmin, float tmax) {
  if (r.d.z == 0.0f) return NAN;
  const float t = (q[3] - r.o.z) / r.d.z;
  if (t <= tmin || t >= tmax) return NAN;
  V3 p = point_at(r, t);
  p.z = q[3];
  const float l2 = p.x * p.x + p.y * p.y;
  if (l2 > q[2] * q[2] || l2 < q[1] * q[1] || spherical_phi(p.x, p.y) > q[0]) return NAN;
  return t;
}
inline Surface disk_surface(const float* q, const Ray& r, float t) {
  V3 p = point_at(r, t);
  p.z = q[3];
  const float l = len2d(p);
  const ONB g = uv_frame(V3{-q[0] * p.y, q[0] * p.x, 0.0f}, V3{p.x * (q[1] - q[2]) / l, p.y * (q[1] - q[2]) / l, 0.0f});
  return simple_surface(r, t, p, g, spherical_phi(p.x, p.y) / q[0], (q[2] - l) / (q[2] - q[1]));
}

// geometry/shape/Cylinder3F.java:342 (record: phiMax, radius, zMax, zMin)
inline V3 cylinder_point(const float* q, const Ray& r, float t) {
  const V3 p = point_at(r, t);
  const float s = q[1] / len2d(p);
  return V3{p.x * s, p.y * s, p.z};
}
inline float cylinder_t(const float* q, const Ray& r, float tmin, float tmax) {
  const V3 o = r.o, d = r.d;
  const float a = d.x * d.x + d.y * d.y;
  const float b = 2.0f * (d.x * o.x + d.y * o.y);
  const float c = o.x * o.x + o.y * o.y - q[1] * q[1];
  return quadric_t(a, b, c, r, tmin, tmax, [&](const Ray& rr, float t) { return cylinder_point(q, rr, t); },
                   [&](V3 p) { return p.z >= q[3] && p.z <= q[2] && spherical_phi(p.x, p.y) <= q[0]; });
}
inline Surface cylinder_surface(const float* q, const Ray& r, float t) {
  const V3 p = cylinder_point(q, r, t);
  const ONB g = uv_frame(V3{-q[0] * p.y, q[0] * p.x, 0.0f}, V3{0.0f, 0.0f, q[2] - q[3]});
  return simple_surface(r, t, p, g, spherical_phi(p.x, p.y) / q[0], (p.z - q[3]) / (q[2] - q[3]));
}

// geometry/shape/Cone3F.java (record: phiMax, radius, zMax, 0)
inline float cone_t(const float* q, const Ray& r, float tmin, float tmax) {
  const V3 o = r.o, d = r.d;
  const float k = (q[1] / q[2]) * (q[1] / q[2]);
  const float a = d.x * d.x + d.y * d.y - k * d.z * d.z;
  const float b = 2.0f * (d.x * o.x + d.y * o.y - k * d.z * (o.z - q[2]));
  const float c = o.x * o.x + o.y * o.y - k * (o.z - q[2]) * (o.z - q[2]);
  return quadric_t(a, b, c, r, tmin, tmax, [](const Ray& rr, float t) { return point_at(rr, t); },
                   [&](V3 p) { return p.z >= 0.0f && p.z <= q[2] && spherical_phi(p.x, p.y) <= q[0]; });
}
inline Surface cone_surface(const float* q, const Ray& r, float t) {
  const V3 p = point_at(r, t);
  const float value = 1.0f - (p.z / q[2]);
  const ONB g = uv_frame(V3{-q[0] * p.y, q[0] * p.x, 0.0f}, V3{-p.x / value, -p.y / value, q[2]});
  return simple_surface(r, t, p, g, spherical_phi(p.x, p.y) / q[0], p.z / q[2]);
}

// geometry/shape/Paraboloid3F.java (record: phiMax, radius, zMax, zMin)
inline float paraboloid_t(const float* q, const Ray& r, float tmin, float tmax) {
  const V3 o = r.o, d = r.d;
  const float k = q[2] / (q[1] * q[1]);
  const float a = k * (d.x * d.x + d.y * d.y);
  const float b = 2.0f * k * (d.x * o.x + d.y * o.y) - d.z;
  const float c = k * (o.x * o.x + o.y * o.y) - o.z;
  return quadric_t(a, b, c, r, tmin, tmax, [](const Ray& rr, float t) { return point_at(rr, t); },
                   [&](V3 p) { return p.z >= q[3] && p.z <= q[2] && spherical_phi(p.x, p.y) <= q[0]; });
}
inline Surface paraboloid_surface(const float* q, const Ray& r, float t) {
  const V3 p = point_at(r, t);
  const float dz = q[2] - q[3];
  const ONB g = uv_frame(V3{-q[0] * p.y, q[0] * p.x, 0.0f}, V3{dz * (p.x / (2.0f * p.z)), dz * (p.y / (2.0f * p.z)), dz});
  return simple_surface(r, t, p, g, spherical_phi(p.x, p.y) / q[0], (p.z - q[3]) / dz);
}

// geometry/shape/Hyperboloid3F.java (record: phiMax, A xyz, B xyz, aH, cH, rMax, zMax, zMin)
inline float hyperboloid_phi(const float* q, V3 p, float v) {
  // Point3F.lerp with Floats.lerp: (1 - t) * a + t * b
  const float ax = (1.0f - v) * q[1] + v * q[4], ay = (1.0f - v) * q[2] + v * q[5];
  return spherical_phi(p.x * ax + p.y * ay, p.y * ax - p.x * ay);
}
inline float hyperboloid_phi(const float* q, V3 p) { return hyperboloid_phi(q, p, (p.z - q[3]) / (q[6] - q[3])); }
inline float hyperboloid_t(const float* q, const Ray& r, float tmin, float tmax) {
  const V3 o = r.o, d = r.d;
  const float aH = q[7], cH = q[8];
  const float a = aH * d.x * d.x + aH * d.y * d.y - cH * d.z * d.z;
  const float b = 2.0f * (aH * d.x * o.x + aH * d.y * o.y - cH * d.z * o.z);
  const float c = aH * o.x * o.x + aH * o.y * o.y - cH * o.z * o.z - 1.0f;
  return quadric_t(a, b, c, r, tmin, tmax, [](const Ray& rr, float t) { return point_at(rr, t); },
                   [&](V3 p) { return p.z >= q[11] && p.z <= q[10] && hyperboloid_phi(q, p) <= q[0]; });
}
inline Surface hyperboloid_surface(const float* q, const Ray& r, float t) {
  const V3 p = point_at(r, t);
  const float phi = hyperboloid_phi(q, p);
  const float c = (float)std::cos((double)phi), sn = (float)std::sin((double)phi);
  const V3 v = {(q[4] - q[1]) * c - (q[5] - q[2]) * sn, (q[4] - q[1]) * sn + (q[5] - q[2]) * c, q[6] - q[3]};
  const ONB g = uv_frame(V3{-q[0] * p.y, q[0] * p.x, 0.0f}, v);
  const float tv = (p.z - q[3]) / (q[6] - q[3]);
  return simple_surface(r, t, p, g, hyperboloid_phi(q, p, tv) / q[0], tv);
}

// geometry/shape/RectangularCuboid3F.java (record: maximum xyz, minimum xyz, 0, 0)
inline float cuboid_t(const float* q, const Ray& r, float tmin, float tmax) {
  const V3 rd = {1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z};
  const V3 da = {(q[3] - r.o.x) * rd.x, (q[4] - r.o.y) * rd.y, (q[5] - r.o.z) * rd.z};
  const V3 db = {(q[0] - r.o.x) * rd.x, (q[1] - r.o.y) * rd.y, (q[2] - r.o.z) * rd.z};
  const float t0 = jmax(jmax(jmin(da.x, db.x), jmin(da.y, db.y)), jmin(da.z, db.z));
  const float t1 = jmin(jmin(jmax(da.x, db.x), jmax(da.y, db.y)), jmax(da.z, db.z));
  if (t0 > t1) return NAN;
  if (t0 > tmin && t0 < tmax) return t0;
  if (t1 > tmin && t1 < tmax) return t1;
  return NAN;
}
inline Surface cuboid_surface(const float* q, const Ray& r, float t) {
  const V3 p = point_at(r, t);
  const V3 mid = {(q[0] + q[3]) * 0.5f, (q[1] + q[4]) * 0.5f, (q[2] + q[5]) * 0.5f};
  const V3 half = {(q[0] - q[3]) * 0.5f, (q[1] - q[4]) * 0.5f, (q[2] - q[5]) * 0.5f};
  const bool x0 = p.x + half.x - 0.0001f < mid.x, x1 = p.x - half.x + 0.0001f > mid.x;
  const bool y0 = p.y + half.y - 0.0001f < mid.y, y1 = p.y - half.y + 0.0001f > mid.y;
  const bool z0 = p.z + half.z - 0.0001f < mid.z, z1 = p.z - half.z + 0.0001f > mid.z;
  ONB g = ONB{V3{0, 0, 1}, V3{0, 1, 0}, V3{1, 0, 0}};
  if (x0) g = onb_from_w(V3{-1, 0, 0});
  else if (x1) g = onb_from_w(V3{1, 0, 0});
  else if (y0) g = onb_from_w(V3{0, -1, 0});
  else if (y1) g = onb_from_w(V3{0, 1, 0});
  else if (z0) g = onb_from_w(V3{0, 0, -1});
  else if (z1) g = onb_from_w(V3{0, 0, 1});
  auto nrm = [](float v, float a, float b) { const float mx = jmax(a, b), mn = jmin(a, b); return (v - mn) / (mx - mn); };
  float tu = 0.0f, tv = 0.0f;
  if (x0 || x1) { tu = nrm(p.z, q[5], q[2]); tv = nrm(p.y, q[4], q[1]); }
  else if (y0 || y1) { tu = nrm(p.x, q[3], q[0]); tv = nrm(p.z, q[5], q[2]); }
  else if (z0 || z1) { tu = nrm(p.x, q[3], q[0]); tv = nrm(p.y, q[4], q[1]); }
  return simple_surface(r, t, p, g, tu, tv);
}

// geometry/shape/Torus3F.java (record: radiusInner, radiusOuter): a quartic in
// double precision, solved by the reference's own resolvent-cubic method.
inline double torus_cubic(double p, double q, double r) {
  const double p2 = p * p;
  const double q0 = (p2 - 3.0 * q) / 9.0;
  const double q0c = q0 * q0 * q0;
  const double r0 = (p * (p2 - 4.5 * q) + 13.5 * r) / 27.0;
  const double r02 = r0 * r0;
  const double d = q0c - r02;
  const double e = p / 3.0;
  if (d >= 0.0) {
    const double d0 = r0 / std::sqrt(q0c);
    const double theta = std::acos(d0) / 3.0;
    const double q1 = -2.0 * std::sqrt(q0);
    return q1 * std::cos(theta) - e;
  }
  const double q1 = std::pow(std::sqrt(r02 - q0c) + std::fabs(r0), 1.0 / 3.0);
  return r0 < 0.0 ? (q1 + q0 / q1) - e : -(q1 + q0 / q1) - e;
}
inline int torus_quartic(double a, double b, double c, double d, double e, double* out) {
  const double ar = 1.0 / a;
  const double bA = b * ar, bA2 = bA * bA, cA = c * ar, dA = d * ar, eA = e * ar;
  const double p = -0.375 * bA2 + cA;
  const double q = 0.125 * bA2 * bA - 0.5 * bA * cA + dA;
  const double r = -0.01171875 * bA2 * bA2 + 0.0625 * bA2 * cA - 0.25 * bA * dA + eA;
  const double z = torus_cubic(-0.5 * p, -r, 0.5 * r * p - 0.125 * q * q);
  double d1 = 2.0 * z - p, d2;
  if (d1 < 0.0) return 0;
  if (d1 < 1.0e-10) {
    d2 = z * z - r;
    if (d2 < 0.0) return 0;
    d2 = std::sqrt(d2);
  } else {
    d1 = std::sqrt(d1);
    d2 = 0.5 * q / d1;
  }
  const double q1 = d1 * d1, q2 = -0.25 * bA;
  const double pm = q1 - 4.0 * (z - d2), pp = q1 - 4.0 * (z + d2);
  if (pm >= 0.0 && pp >= 0.0) {
    const double pms = std::sqrt(pm), pps = std::sqrt(pp);
    out[0] = -0.5 * (d1 + pms) + q2;
    out[1] = -0.5 * (d1 - pms) + q2;
    out[2] = 0.5 * (d1 + pps) + q2;
    out[3] = 0.5 * (d1 - pps) + q2;
    for (int i = 1; i < 4; ++i)
      for (int j = i; j > 0 && out[j - 1] > out[j]; --j) std::swap(out[j], out[j - 1]);
    return 4;
  }
  if (pm >= 0.0) {
    const double pms = std::sqrt(pm);
    out[0] = -0.5 * (d1 + pms) + q2;
    out[1] = -0.5 * (d1 - pms) + q2;
    return 2;
  }
  if (pp >= 0.0) {
    const double pps = std::sqrt(pp);
    out[0] = 0.5 * (d1 - pps) + q2;
    out[1] = 0.5 * (d1 + pps) + q2;
    return 2;
  }
  return 0;
}
inline float torus_t(const float* q, const Ray& r, float tmin, float tmax) {
  const float ri2 = q[0] * q[0], ro2 = q[1] * q[1];
  const double f0 = (double)dot(r.d, r.d);
  const double f1 = (double)dot(r.o, r.d) * 2.0;
  const double f2 = ri2, f3 = ro2;
  const double f4 = (double)dot(r.o, r.o) - f2 - f3;
  const double f5 = r.d.z, f6 = r.o.z;
  const double a = f0 * f0;
  const double b = f0 * 2.0 * f1;
  const double c = f1 * f1 + 2.0 * f0 * f4 + 4.0 * f3 * f5 * f5;
  const double d = f1 * 2.0 * f4 + 8.0 * f3 * f6 * f5;
  const double e = f4 * f4 + 4.0 * f3 * f6 * f6 - 4.0 * f3 * f2;
  double ts[4];
  const int n = torus_quartic(a, b, c, d, e, ts);
  if (n == 0) return NAN;
  if (ts[0] >= tmax || ts[n - 1] <= tmin) return NAN;
  for (int i = 0; i < n; ++i)
    if (ts[i] > tmin) return (float)ts[i];
  return NAN;
}
inline Surface torus_surface(const float* q, const Ray& r, float t) {
  const V3 p = point_at(r, t);
  const float ri2 = q[0] * q[0], ro2 = q[1] * q[1];
  const float der = dot(p, p) - ri2 - ro2;
  const ONB g = onb_from_w(normalize(V3{p.x * der, p.y * der, p.z * der + 2.0f * ro2 * p.z}));
  const float phi = (float)std::asin((double)saturate(p.z / q[0], -1.0f, 1.0f));
  const float theta = spherical_phi(p.x, p.y);
  return simple_surface(r, t, p, g, theta * (1.0f / (2.0f * kPi)), (phi + kPi / 2.0f) * (1.0f / kPi));
}

// renderer/gpu/AbstractShape3FKernel.java:3735 threaded mesh BVH stream, walked
// with TriangleMesh3F's closest-hit rule (geometry/boundingvolume/hierarchy/*BVHNode3F.java).
inline float mesh_t(const Scene& sc, int mesh_off, const Ray& r, float tmin, float tmax, int* tri_out) {
  const auto& M = sc.I("shape3FTriangleMesh3FArray");
  const auto& A = sc.F("boundingVolume3FAxisAlignedBoundingBox3FArray");
  const auto& T = sc.F("shape3FTriangle3FArray");
  float best = NAN;
  int rel = 0;
  long guard = 0;
  while (rel != -1 && guard++ < (1L << 31)) {
    const int o = mesh_off + rel;
    const int id = M[o], bv = M[o + 1], next = M[o + 2], lc = M[o + 3];
    bool hitbv = aabb_contains_or_intersects(A.data() + (size_t)bv * 8, r, tmin, tmax);
    if (hitbv && id == 1) {
      for (int k = 0; k < lc; ++k) {
        int toff = M[o + 4 + k];
        float t = triangle_t(load_tri(T, toff), r, tmin, tmax);
        if (!std::isnan(t) && (std::isnan(best) || t < best) && t > tmin && t < tmax) { best = t; tmax = t; *tri_out = toff; }
      }
      rel = next;
    } else if (hitbv && id == 2) {
      rel = lc;
    } else {
      rel = next;
    }
  }
  return best;
}

// geometry/shape/Polygon3F.java over the compiled record (CompiledShape3FCache:
// points 0, 1 and n-1 at +0, +3, +6, surface normal +9, point count +12, the
// polygon projected on its plane at +13, two floats per point).
inline bool polygon_contains(const float* q, V3 p) {  // Polygon3F.doContains + Polygon2F.contains
  const V3 a = {q[0], q[1], q[2]}, b = {q[3], q[4], q[5]}, w = {q[9], q[10], q[11]};
  const V3 u = normalize(b - a), v = cross(w, u);
  const V3 ap = p - a;
  const float px = dot(ap, u), py = dot(ap, v);
  const int n = (int)q[12];
  const float* P = q + 13;
  for (int i = 0, j = 1; i < n; ++i, j = (j + 1) % n) {  // LineSegment2F.contains on every edge
    const float ax = P[2 * i], ay = P[2 * i + 1], bx = P[2 * j], by = P[2 * j + 1];
    const float dx = px - ax, dy = py - ay, ex = bx - ax, ey = by - ay;
    if (dx * ey - dy * ex != 0.0f) continue;
    if (std::fabs(ex) >= std::fabs(ey) ? (ex > 0.0f ? ax <= px && px <= bx : bx <= px && px <= ax)
                                       : (ey > 0.0f ? ay <= py && py <= by : by <= py && py <= ay))
      return true;
  }
  bool inside = false;  // Polygon2F.doContains (crossing test)
  for (int i = 0, j = n - 1; i < n; j = i++) {
    const float ix = P[2 * i], iy = P[2 * i + 1], jx = P[2 * j], jy = P[2 * j + 1];
    if ((iy > py) != (jy > py) && px < (jx - ix) * (py - iy) / (jy - iy) + ix) inside = !inside;
  }
  return inside;
}
inline float polygon_t(const float* q, const Ray& r, float tmin, float tmax) {  // Polygon3F.java:321
  const V3 n = {q[9], q[10], q[11]}, a = {q[0], q[1], q[2]};
  const float dp = dot(n, r.d);
  if (dp == 0.0f) return NAN;
  const float t = dot(a - r.o, n) / dp;
  if (t > tmin && t < tmax && polygon_contains(q, point_at(r, t))) return t;
  return NAN;
}
inline Surface polygon_surface(const float* q, const Ray& r, float t) {  // Polygon3F.doCreateSurfaceIntersection
  const V3 p = point_at(r, t);
  const V3 n = {q[9], q[10], q[11]};
  const V3 na = {std::fabs(n.x), std::fabs(n.y), std::fabs(n.z)};
  const bool isx = na.x > na.y && na.x > na.z, isy = na.y > na.z;
  auto proj = [&](const float* c) { return isx ? std::make_pair(c[1], c[2]) : isy ? std::make_pair(c[2], c[0]) : std::make_pair(c[0], c[1]); };
  const auto A = proj(q), B = proj(q + 6), C = proj(q + 3);  // vB from the last point, vC from the second (doCreateTextureCoordinates)
  const float abx = B.first - A.first, aby = B.second - A.second, acx = C.first - A.first, acy = C.second - A.second;
  const float dr = 1.0f / (abx * acy - aby * acx);
  const float hu = isx ? p.y : isy ? p.z : p.x, hv = isx ? p.z : isy ? p.x : p.y;
  const float tu = hu * (-aby * dr) + hv * (abx * dr) + (A.first * aby - A.second * abx) * dr;
  const float tv = hu * (acy * dr) + hv * (-acx * dr) + (acx * A.second - acy * A.first) * dr;
  return simple_surface(r, t, p, onb_from_w(n), tu, tv);
}

// Shape3F.intersectionT dispatch (object space).  aux receives the mesh's
// winning triangle offset.
inline float shape_t(const Scene& sc, int sid, int soff, const Ray& r, float tmin, float tmax, int* aux) {
  switch (sid) {
    case kShapeTriangle: return triangle_t(load_tri(sc.F("shape3FTriangle3FArray"), soff), r, tmin, tmax);
    case kShapeMesh: return mesh_t(sc, soff, r, tmin, tmax, aux);
    case kShapeSphere: { SphereHit h; return sphere_hit(r, tmin, tmax, &h) ? h.t : NAN; }
    case kShapeRectangle: return rect_t(load_rect(sc.F("shape3FRectangle3FArray"), soff), r, tmin, tmax);
    case kShapePlane: return plane_t(r, tmin, tmax);
    case kShapeDisk: return disk_t(sc.F("shape3FDisk3FArray").data() + soff, r, tmin, tmax);
    case kShapeCylinder: return cylinder_t(sc.F("shape3FCylinder3FArray").data() + soff, r, tmin, tmax);
    case kShapeCone: return cone_t(sc.F("shape3FCone3FArray").data() + soff, r, tmin, tmax);
    case kShapeParaboloid: return paraboloid_t(sc.F("shape3FParaboloid3FArray").data() + soff, r, tmin, tmax);
    case kShapeHyperboloid: return hyperboloid_t(sc.F("shape3FHyperboloid3FArray").data() + soff, r, tmin, tmax);
    case kShapeCuboid: return cuboid_t(sc.F("shape3FRectangularCuboid3FArray").data() + soff, r, tmin, tmax);
    case kShapeTorus: return torus_t(sc.F("shape3FTorus3FArray").data() + soff, r, tmin, tmax);
    case kShapePolygon: return polygon_t(sc.F("shape3FPolygon3FArray").data() + soff, r, tmin, tmax);
    default: return NAN;
  }
}

// Shape3F.intersection(ray, tmin, tmax): full surface record.
inline bool shape_surface(const Scene& sc, int sid, int soff, const Ray& r, float tmin, float tmax, Surface* s, int* tri_out) {
  switch (sid) {
    case kShapeTriangle: {
      Tri tr = load_tri(sc.F("shape3FTriangle3FArray"), soff);
      float t = triangle_t(tr, r, tmin, tmax);
      if (std::isnan(t)) return false;
      *s = triangle_surface(tr, r, t); *tri_out = soff; return true;
    }
    case kShapeMesh: {
      int toff = -1;
      float t = mesh_t(sc, soff, r, tmin, tmax, &toff);
      if (std::isnan(t) || toff < 0) return false;
      *s = triangle_surface(load_tri(sc.F("shape3FTriangle3FArray"), toff), r, t); *tri_out = toff; return true;
    }
    case kShapeSphere: { SphereHit h; if (!sphere_hit(r, tmin, tmax, &h)) return false; *s = sphere_surface(r, h); *tri_out = -1; return true; }
    case kShapeRectangle: {
      Rect q = load_rect(sc.F("shape3FRectangle3FArray"), soff);
      float t = rect_t(q, r, tmin, tmax);
      if (std::isnan(t)) return false;
      *s = rect_surface(q, r, t); *tri_out = -1; return true;
    }
    case kShapePlane: { float t = plane_t(r, tmin, tmax); if (std::isnan(t)) return false; *s = plane_surface(r, t); *tri_out = -1; return true; }
#define DFO_SIMPLE_SHAPE(ID, ARR, TF, SF)                       \
    case ID: {                                                  \
      const float* q = sc.F(ARR).data() + soff;                 \
      const float t = TF(q, r, tmin, tmax);                     \
      if (std::isnan(t)) return false;                          \
      *s = SF(q, r, t); *tri_out = -1; return true;             \
    }
    DFO_SIMPLE_SHAPE(kShapeDisk, "shape3FDisk3FArray", disk_t, disk_surface)
    DFO_SIMPLE_SHAPE(kShapeCylinder, "shape3FCylinder3FArray", cylinder_t, cylinder_surface)
    DFO_SIMPLE_SHAPE(kShapeCone, "shape3FCone3FArray", cone_t, cone_surface)
    DFO_SIMPLE_SHAPE(kShapeParaboloid, "shape3FParaboloid3FArray", paraboloid_t, paraboloid_surface)
    DFO_SIMPLE_SHAPE(kShapeHyperboloid, "shape3FHyperboloid3FArray", hyperboloid_t, hyperboloid_surface)
    DFO_SIMPLE_SHAPE(kShapeCuboid, "shape3FRectangularCuboid3FArray", cuboid_t, cuboid_surface)
    DFO_SIMPLE_SHAPE(kShapeTorus, "shape3FTorus3FArray", torus_t, torus_surface)
    DFO_SIMPLE_SHAPE(kShapePolygon, "shape3FPolygon3FArray", polygon_t, polygon_surface)
#undef DFO_SIMPLE_SHAPE
    default: return false;
  }
}

// geometry/SurfaceIntersection3F.java:372
inline Surface surface_transform(const Surface& in, const M44& m, const M44& minv) {
  Surface o;
  o.g = onb_transform_transpose(minv, in.g);
  ONB s = onb_transform_transpose(minv, in.s);
  o.s = dot(s.w, o.g.w) < 0.0f ? onb_flip_w(s) : s;
  o.tu = in.tu; o.tv = in.tv;
  o.p = transform_point_divide(m, in.p);
  o.ray = transform_ray(m, in.ray);
  o.t = std::fabs(distance(o.ray.o, o.p));
  return o;
}

struct Hit {  // scene/Intersection.java
  int prim = -1;
  int tri = -1;
  Surface w;  // world space
  V3 p_obj;   // object-space surface intersection point (BullseyeTexture, BullseyeMaterial)
};

// geometry/SurfaceIntersector3F.java:188 doTransformT
inline float transform_t(const M44& m, const Ray& old_r, const Ray& new_r, float t) {
  if (!std::isnan(t) && t != 0.0f && t < FLT_MAX) return std::fabs(distance(new_r.o, transform_point_divide(m, old_r.o + old_r.d * t)));
  return t;
}

struct RayStats { long long rays = 0; };

// Diagnostic switch (default off): when set, every candidate primitive sees the
// original world ray instead of the ray the reference's intersector carries
// through each primitive's object space and back (SurfaceIntersector3F.transform).
static int g_no_drift = 0;

// scene/Scene.java:874 intersection(): linear loop over the primitives with
// the Intersector state (the ray is mapped into object space and back for
// every candidate, exactly as SurfaceIntersector3F.transform does).
inline bool scene_intersect(const Scene& sc, const Ray& ray_in, float tmin, float tmax, Hit* hit, RayStats* st) {
  if (st) st->rays++;
  Ray r = ray_in;
  float t = NAN;
  int prim = -1;
  const auto& A = sc.F("boundingVolume3FAxisAlignedBoundingBox3FArray");
  const auto& BS = sc.F("boundingVolume3FBoundingSphere3FArray");
  for (int p = 0; p < sc.prim_count; ++p) {
    const int32_t* P = sc.prims.data() + p * 8;
    int bvid = P[2], bvoff = P[3], sid = P[6], soff = P[7];
    bool bv = bvid == kBVInfinite || (bvid == kBVAabb && aabb_contains_or_intersects(A.data() + (size_t)bvoff * 8, r, tmin, tmax)) ||
              (bvid == kBVSphere && bsphere_contains_or_intersects(BS.data() + (size_t)bvoff * 4, r, tmin, tmax));
    if (!bv) continue;
    const M44& w2o = sc.w2o[p];
    const M44& o2w = sc.o2w[p];
    Ray ro = transform_ray(w2o, r);
    float to = transform_t(w2o, r, ro, t);
    float tmaxo = transform_t(w2o, r, ro, tmax);
    int aux = -1;
    float th = shape_t(sc, sid, soff, ro, tmin, tmaxo, &aux);
    if (!std::isnan(th) && (std::isnan(to) || th < to) && th > tmin && th < tmaxo) { to = th; tmaxo = th; prim = p; }
    Ray rw = transform_ray(o2w, ro);
    t = transform_t(o2w, ro, rw, to);
    tmax = transform_t(o2w, ro, rw, tmaxo);
    if (!g_no_drift) r = rw;
  }
  if (prim < 0) return false;
  if (!hit) return true;
  // scene/Intersector.java computeIntersection()
  const int32_t* P = sc.prims.data() + prim * 8;
  Ray ro = transform_ray(sc.w2o[prim], r);
  Surface so;
  int tri = -1;
  if (!shape_surface(sc, P[6], P[7], ro, kTMinimum, kTMaximum, &so, &tri)) return false;
  hit->prim = prim; hit->tri = tri;
  hit->w = surface_transform(so, sc.o2w[prim], sc.w2o[prim]);
  hit->p_obj = so.p;
  return true;
}

// ---- textures and materials --------------------------------------------------
struct TexRef { int id, off; };
inline void material_slot(const Scene& sc, const std::vector<int32_t>& arr, int base, int slot, TexRef* a, TexRef* b) {
  if (sc.layout == 2) {
    const int32_t* q = arr.data() + base + slot * 4;
    a->id = q[0]; a->off = q[1]; b->id = q[2]; b->off = q[3];
  } else {
    uint32_t v = (uint32_t)arr[base + slot];  // utility/Ints.java:258 pack(a, b, c, d)
    a->id = v & 0xFF; a->off = (v >> 8) & 0xFF; b->id = (v >> 16) & 0xFF; b->off = (v >> 24) & 0xFF;
  }
}
inline int material_int(const Scene& sc, const std::vector<int32_t>& arr, int base, int slot) {
  return sc.layout == 2 ? arr[base + slot * 4] : arr[base + slot];
}
// What a texture sees of the intersection (scene/Intersection.java): world
// point, object-space point, shading normal (after the material's modifier),
// ray direction and texture coordinates.
struct TexCtx { V3 p, p_obj, ns, d; float u, v; };
thread_local const TexCtx* g_tex = nullptr;  // set while a material is evaluated at a hit

inline TexCtx tex_ctx(const Hit& h) { return TexCtx{h.w.p, h.p_obj, h.w.s.w, h.w.ray.d, h.w.tu, h.w.tv}; }

inline float jsin(float a) { return (float)std::sin((double)a); }  // utility/Floats.java sin, cos: Math in double
inline float jcos(float a) { return (float)std::cos((double)a); }
inline float frac(float x) { return x - std::floor(x); }            // Floats.fractionalPart(x, false)
inline float jmod(float x, float y) { return std::fmod(x, y); }     // Java float %
inline float pos_mod(float x, float y) { return x < 0.0f ? jmod(jmod(x, y) + y, y) : jmod(x, y); }  // Floats.positiveModulo
inline int pos_mod_i(int x, int y) { return x < 0 ? (x % y + y) % y : x % y; }                         // Ints.positiveModulo
inline V3 unpack_argb(int c) {  // Color3F.unpack(ARGB): 8-bit channels / 255
  return {(float)((c >> 16) & 0xFF) / 255.0f, (float)((c >> 8) & 0xFF) / 255.0f, (float)(c & 0xFF) / 255.0f};
}
inline V3 lerp3(V3 a, V3 b, V3 t) { return {(1.0f - t.x) * a.x + t.x * b.x, (1.0f - t.y) * a.y + t.y * b.y, (1.0f - t.z) * a.z + t.z * b.z}; }
inline TexRef unpack16(float f) { const int v = (int)f; return TexRef{(v >> 16) & 0xFFFF, v & 0xFFFF}; }

// LDRImageTexture.doGetColorRGB / AbstractLDRImageModifier.getColorRGB over a
// compiled image record (angle radians, scale x, y, resolution x, y, ARGB pixels).
inline V3 image_texel(const float* rec, int x, int y) {
  const int rx = (int)rec[3], ry = (int)rec[4];
  return unpack_argb((int)rec[5 + pos_mod_i(y, ry) * rx + pos_mod_i(x, rx)]);
}
inline void image_point(const float* rec, float u, float v, float* x, float* y) {
  const float c = jcos(rec[0]), s = jsin(rec[0]);  // Point2F.rotateCounterclockwise
  const float ru = u * c - v * s, rv = v * c + u * s;
  const float rx = (float)(int)rec[3], ry = (float)(int)rec[4];
  *x = pos_mod(ru * rec[1] * rx - 0.5f, rx);  // Point2F.scale, Point2F.toImage
  *y = pos_mod(rv * rec[2] * ry - 0.5f, ry);
}
inline V3 image_bilinear(const float* rec, float x, float y) {
  const int x0 = (int)std::floor(x), x1 = (int)std::ceil(x), y0 = (int)std::floor(y), y1 = (int)std::ceil(y);
  if (x0 == x1 && y0 == y1) return image_texel(rec, x0, y0);
  const float tx = x - (float)x0, ty = y - (float)y0;
  const V3 t3{tx, tx, tx}, s3{ty, ty, ty};
  return lerp3(lerp3(image_texel(rec, x0, y0), image_texel(rec, x1, y0), t3), lerp3(image_texel(rec, x0, y1), image_texel(rec, x1, y1), t3), s3);
}

// Texture.getColor(intersection) of every compiled texture (scene/texture/*.java getColor).
inline V3 tex_eval(const Scene& sc, TexRef t, const TexCtx& c, int depth) {
  if (depth > 32) return {0.5f, 0.5f, 0.5f};
  switch (t.id) {
    case kTexConstant: {
      const float* q = sc.F("textureConstantTextureArray").data() + (size_t)t.off * 4;
      return {q[0], q[1], q[2]};
    }
    case kTexBlend: {  // BlendTexture: Color3F.blend(A, B, t1, t2, t3)
      const float* q = sc.F("textureBlendTextureArray").data() + (size_t)t.off * 8;
      return lerp3(tex_eval(sc, unpack16(q[0]), c, depth + 1), tex_eval(sc, unpack16(q[1]), c, depth + 1), V3{q[2], q[3], q[4]});
    }
    case kTexBullseye: {  // BullseyeTexture: object-space distance to the origin
      const float* q = sc.F("textureBullseyeTextureArray").data() + (size_t)t.off * 8;
      const V3 dir = c.p_obj - V3{q[0], q[1], q[2]};
      const float r = jmod(length(dir) * q[5], 1.0f);
      return tex_eval(sc, unpack16(r > 0.5f ? q[3] : q[4]), c, depth + 1);
    }
    case kTexCheckerboard: {
      const float* q = sc.F("textureCheckerboardTextureArray").data() + (size_t)t.off * 8;
      const float cs = jcos(q[1]), sn = jsin(q[1]);
      const bool iu = frac((c.u * cs - c.v * sn) * q[4]) > 0.5f;
      const bool iv = frac((c.v * cs + c.u * sn) * q[5]) > 0.5f;
      return tex_eval(sc, unpack16((iu ^ iv) ? q[2] : q[3]), c, depth + 1);
    }
    case kTexPolkaDot: {
      const float* q = sc.F("texturePolkaDotTextureArray").data() + (size_t)t.off * 8;
      const float cs = jcos(q[1]), sn = jsin(q[1]);
      const float x = frac((c.u * cs - c.v * sn) * q[4]) - 0.5f;
      const float y = frac((c.v * cs + c.u * sn) * q[4]) - 0.5f;
      return tex_eval(sc, unpack16(x * x + y * y < q[5] * q[5] ? q[2] : q[3]), c, depth + 1);
    }
    case kTexDotProduct: {  // |n_s . d|
      const float d = std::fabs(dot(c.ns, c.d));
      return {d, d, d};
    }
    case kTexLDRImage: {
      const int abs_off = sc.I("textureLDRImageTextureOffsetArray")[t.off];
      const float* q = sc.F("textureLDRImageTextureArray").data() + abs_off;
      float x, y;
      image_point(q, c.u, c.v, &x, &y);
      return image_bilinear(q, x, y);
    }
    case kTexMarble: {  // MarbleTexture (colours as compiled: packed ARGB)
      const float* q = sc.F("textureMarbleTextureArray").data() + (size_t)t.off * 8;
      const float x = c.p.x * q[3], y = c.p.y * q[3], z = c.p.z * q[3];
      const float r = q[4] * dfo_noise::perlin_turbulence(x, y, z, (int)q[6]);
      const float s = 2.0f * std::fabs(jsin(x + r));
      const float tt = s < 1.0f ? s : s - 1.0f;
      const V3 ca = unpack_argb((int)q[0]), cb = unpack_argb((int)q[1]), cc = unpack_argb((int)q[2]);
      return lerp3(s < 1.0f ? cc : cb, s < 1.0f ? cb : ca, V3{tt, tt, tt});
    }
    case kTexSimplexFBM: {
      const float* q = sc.F("textureSimplexFractionalBrownianMotionTextureArray").data() + (size_t)t.off * 4;
      const float n = dfo_noise::simplex_fbm(c.p.x, c.p.y, c.p.z, q[1], q[2], 0.0f, 1.0f, (int)q[3]);
      return unpack_argb((int)q[0]) * n;
    }
    case kTexSurfaceNormal: {  // (n_s facing the ray + 1) / 2
      const V3 n = dot(c.ns, c.d) > 0.0f ? -c.ns : c.ns;
      return {(n.x + 1.0f) / 2.0f, (n.y + 1.0f) / 2.0f, (n.z + 1.0f) / 2.0f};
    }
    case kTexUV: return {c.u, c.v, 0.0f};
    default: return {0.5f, 0.5f, 0.5f};
  }
}
inline V3 tex_color(const Scene& sc, TexRef t) {
  if (t.id == kTexConstant) {
    const float* q = sc.F("textureConstantTextureArray").data() + (size_t)t.off * 4;
    return {q[0], q[1], q[2]};
  }
  if (!g_tex) return {0.5f, 0.5f, 0.5f};
  return tex_eval(sc, t, *g_tex, 0);
}
inline float tex_float(const Scene& sc, TexRef t) { V3 c = tex_color(sc, t); return (c.x + c.y + c.z) / 3.0f; }  // ConstantTexture.getFloat = average
inline V3 sat0(V3 c) { return {std::fmax(c.x, 0.0f), std::fmax(c.y, 0.0f), std::fmax(c.z, 0.0f)}; }  // Color3F.saturate(c, 0, MAX)
inline bool black(V3 c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
inline V3 mul(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }

// scene/BXDFType.java flags
enum { kRefl = 1, kTrans = 2, kDiffuse = 4, kGlossy = 8, kSpecular = 16, kAll = 31, kAllButSpecular = 15 };

enum LobeKind {
  kLambert, kOrenNayar, kSpecBRDF, kFresnelSpec, kSpecBTDF, kTSBRDF, kTSBTDF,
  kLambertBTDF,                                                                    // scene/bxdf/LambertianBTDF.java
  kFresnelBlend,                                                                   // scene/bxdf/FresnelBlendBRDF.java
  kDisneyDiffuse, kDisneyFakeSS, kDisneyRetro, kDisneySheen, kDisneyClearCoat      // scene/bxdf/Disney*BRDF.java
};
enum FresKind { kFresConst, kFresDielectric, kFresConductor, kFresDisney };
struct Lobe {
  LobeKind kind; int type;
  V3 scale;            // reflectance / transmittance scale
  float a = 0, b = 0;  // Oren-Nayar A/B
  FresKind fk = kFresConst; float etaI = 1, etaT = 1; V3 cEtaI{1, 1, 1}, cEtaT{1, 1, 1}, cK{0, 0, 0};
  float ax = 0, ay = 0;  // microfacet alphas
  bool separable = false;  // MicrofacetDistribution.isSeparableModel: G = G1(wo) G1(wi)
  float etaA = 1, etaB = 1;
  float roughness = 0;     // Disney retro / fake subsurface
  float gloss = 0, weight = 0;  // Disney clear coat
  V3 r0{0, 0, 0}; float metallic = 0;  // DisneyFresnel(r0, etaT, metallic)
};
constexpr int kMaxLobes = 8;
struct Bsdf {
  int n = 0; Lobe l[kMaxLobes]; float eta = 1.0f; bool present = false;
  ONB s; V3 ng; V3 wo_world; V3 wo; V3 nl;
};

// scene/fresnel/Schlick.java:104 fresnelWeight
inline float schlick_weight(float c) { float m = saturate(1.0f - c, 0.0f, 1.0f); return (m * m) * (m * m) * m; }
inline float lerpf(float a, float b, float t) { return (1.0f - t) * a + t * b; }  // utility/Floats.java:591

// scene/fresnel/DielectricFresnel.java:evaluate
inline float fresnel_dielectric(float cosi, float etaI, float etaT) {
  float c = saturate(cosi, -1.0f, 1.0f);
  bool entering = c > 0.0f;
  float ci = entering ? c : std::fabs(c);
  float ei = entering ? etaI : etaT, et = entering ? etaT : etaI;
  float si = std::sqrt(std::fmax(0.0f, 1.0f - ci * ci));
  float st = ei / et * si;
  if (st >= 1.0f) return 1.0f;
  float ct = std::sqrt(std::fmax(0.0f, 1.0f - st * st));
  float rpa = ((et * ci) - (ei * ct)) / ((et * ci) + (ei * ct));
  float rpe = ((ei * ci) - (et * ct)) / ((ei * ci) + (et * ct));
  return (rpa * rpa + rpe * rpe) / 2.0f;
}
// scene/fresnel/ConductorFresnel.java:evaluate (per channel)
inline float fresnel_conductor1(float cosi, float etai, float etat, float k) {
  float c = saturate(cosi, -1.0f, 1.0f);
  float eta = etat / etai, etak = k / etai;
  float c2 = c * c, s2 = 1.0f - c2, s4 = s2 * s2;
  float eta2 = eta * eta, etak2 = etak * etak;
  float t0 = eta2 - etak2 - s2;
  float a2b2 = std::sqrt(t0 * t0 + eta2 * etak2 * 4.0f);
  float t1 = a2b2 + c2;
  float t2 = std::sqrt((a2b2 + t0) * 0.5f) * (c * 2.0f);
  float t3 = a2b2 * c2 + s4;
  float t4 = t2 * s2;
  float rs = (t1 - t2) / (t1 + t2);
  float rp = rs * (t3 - t4) / (t3 + t4);
  return (rp + rs) * 0.5f;
}
inline V3 fresnel_eval(const Lobe& L, float cosi) {
  switch (L.fk) {
    case kFresConst: return {1, 1, 1};
    case kFresDielectric: { float f = fresnel_dielectric(cosi, L.etaI, L.etaT); return {f, f, f}; }
    case kFresConductor: {
      float c = std::fabs(cosi);
      return {fresnel_conductor1(c, L.cEtaI.x, L.cEtaT.x, L.cK.x), fresnel_conductor1(c, L.cEtaI.y, L.cEtaT.y, L.cK.y), fresnel_conductor1(c, L.cEtaI.z, L.cEtaT.z, L.cK.z)};
    }
    case kFresDisney: {  // scene/fresnel/DisneyFresnel.java:evaluate
      const float d = fresnel_dielectric(cosi, 1.0f, L.etaT);
      const float w = schlick_weight(cosi);
      const V3 s = {lerpf(L.r0.x, 1.0f, w), lerpf(L.r0.y, 1.0f, w), lerpf(L.r0.z, 1.0f, w)};
      return {lerpf(d, s.x, L.metallic), lerpf(d, s.y, L.metallic), lerpf(d, s.z, L.metallic)};
    }
  }
  return {0, 0, 0};
}

// Vector3F local-frame trigonometry (geometry/Vector3F.java:196-390)
inline float cos_t(V3 v) { return v.z; }
inline float sin2_t(V3 v) { return std::fmax(0.0f, 1.0f - v.z * v.z); }
inline float sin_t(V3 v) { return std::sqrt(sin2_t(v)); }
inline float tan2_t(V3 v) { return sin2_t(v) / (v.z * v.z); }
inline float cos_phi(V3 v) { float s = sin_t(v); return s == 0.0f ? 1.0f : saturate(v.x / s, -1.0f, 1.0f); }
inline float sin_phi(V3 v) { float s = sin_t(v); return s == 0.0f ? 0.0f : saturate(v.y / s, -1.0f, 1.0f); }
inline bool same_hemi(V3 a, V3 b) { return a.z * b.z > 0.0f; }

// scene/microfacet/TrowbridgeReitzMicrofacetDistribution.java (visible-area sampling, non-separable G)
inline float tr_D(const Lobe& L, V3 h) {
  float t2 = tan2_t(h);
  if (std::isinf(t2)) return 0.0f;
  float cp = cos_phi(h), sp = sin_phi(h);
  float c4 = (h.z * h.z) * (h.z * h.z);
  float e = (cp * cp / (L.ax * L.ax) + sp * sp / (L.ay * L.ay)) * t2;
  return 1.0f / (kPi * L.ax * L.ay * c4 * (1.0f + e) * (1.0f + e));
}
inline float tr_lambda(const Lobe& L, V3 w) {
  float ta = std::fabs(sin_t(w) / cos_t(w));
  if (std::isinf(ta)) return 0.0f;
  float cp = cos_phi(w), sp = sin_phi(w);
  float alpha = std::sqrt(cp * cp * L.ax * L.ax + sp * sp * L.ay * L.ay);
  float x = (alpha * ta) * (alpha * ta);
  return (-1.0f + std::sqrt(1.0f + x)) / 2.0f;
}
inline float tr_G1(const Lobe& L, V3 w) { return 1.0f / (1.0f + tr_lambda(L, w)); }
inline float tr_G(const Lobe& L, V3 wo, V3 wi) {
  return L.separable ? (1.0f / (1.0f + tr_lambda(L, wo))) * (1.0f / (1.0f + tr_lambda(L, wi))) : 1.0f / (1.0f + tr_lambda(L, wo) + tr_lambda(L, wi));
}
inline float tr_pdf(const Lobe& L, V3 wo, V3 h) { return tr_D(L, h) * tr_G1(L, wo) * std::fabs(dot(wo, h)) / std::fabs(cos_t(wo)); }
inline void tr_slope(float ct, float u, float v, float* sx, float* sy) {
  if (ct > 0.9999f) {
    float r = std::sqrt(u / (1.0f - u)), phi = 2.0f * kPi * v;
    *sx = r * std::cos(phi); *sy = r * std::sin(phi); return;
  }
  float st = std::sqrt(std::fmax(0.0f, 1.0f - ct * ct));
  float tt = st / ct;
  float a = 2.0f / (1.0f + std::sqrt(1.0f + 1.0f / ((1.0f / tt) * (1.0f / tt))));
  float b = 2.0f * u / a - 1.0f;
  float c = std::fmin(1.0f / (b * b - 1.0f), 1.0e10f);
  float d = tt;
  float e = std::sqrt(std::fmax(d * d * c * c - (b * b - d * d) * c, 0.0f));
  float f = d * c - e, g = d * c + e;
  float hs = v > 0.5f ? 1.0f : -1.0f;
  float i = v > 0.5f ? 2.0f * (v - 0.5f) : 2.0f * (0.5f - v);
  float j = (i * (i * (i * 0.27385f - 0.73369f) + 0.46341f)) / (i * (i * (i * 0.093073f + 0.309420f) - 1.0f) + 0.597999f);
  float x = (b < 0.0f || g > 1.0f / tt) ? f : g;
  *sx = x; *sy = hs * j * std::sqrt(1.0f + x * x);
}
inline V3 tr_sample_visible(V3 w, float ax, float ay, float u, float v) {
  V3 ws = normalize(V3{w.x * ax, w.y * ay, w.z});
  float sx, sy;
  tr_slope(cos_t(ws), u, v, &sx, &sy);
  float cp = cos_phi(ws), sp = sin_phi(ws);
  float x = -((cp * sx - sp * sy) * ax);
  float y = -((sp * sx + cp * sy) * ay);
  return normalize(V3{x, y, 1.0f});
}
inline V3 tr_sample_h(const Lobe& L, V3 wo, float u, float v) {
  return wo.z >= 0.0f ? tr_sample_visible(wo, L.ax, L.ay, u, v) : -tr_sample_visible(-wo, L.ax, L.ay, u, v);
}

inline V3 reflect_about(V3 d, V3 n) { return n * (dot(d, n) * 2.0f) - d; }  // Vector3F.reflection(d, n)
inline bool refract(V3 d, V3 n, float eta, V3* out) {                       // Vector3F.java:454
  float ci = dot(d, n);
  float si2 = std::fmax(0.0f, 1.0f - ci * ci);
  float st2 = eta * eta * si2;
  if (st2 >= 1.0f) return false;
  float ct = std::sqrt(1.0f - st2);
  *out = (-d) * eta + n * (eta * ci - ct);
  return true;
}

// geometry/SampleGeneratorF.java:129 concentric disk, :286 cosine hemisphere
inline void concentric(float u, float v, float* x, float* y) {
  if (u == 0.0f && v == 0.0f) { *x = 0; *y = 0; return; }
  float a = u * 2.0f - 1.0f, b = v * 2.0f - 1.0f;
  if (a * a > b * b) { float phi = (kPi / 4.0f) * (b / a); float r = a; *x = r * std::cos(phi); *y = r * std::sin(phi); }
  else { float phi = (kPi / 2.0f) - (kPi / 4.0f) * (a / b); float r = b; *x = r * std::cos(phi); *y = r * std::sin(phi); }
}
inline V3 cosine_hemisphere(float u, float v) {
  float x, y; concentric(u, v, &x, &y);
  return {x, y, std::sqrt(std::fmax(0.0f, 1.0f - x * x - y * y))};
}
inline V3 uniform_hemisphere(float u, float v) {
  float ct = u, st = std::sqrt(std::fmax(0.0f, 1.0f - ct * ct)), phi = 2.0f * kPi * v;
  return {st * std::cos(phi), st * std::sin(phi), ct};
}

// DisneyClearCoatBRDF.java:330 doGTR1, :337 doSmithGGGX
inline float gtr1(float ct, float alpha) {
  const float a = alpha * alpha;
  return (a - 1.0f) / (kPi * std::log(a) * (1.0f + (a - 1.0f) * ct * ct));
}
inline float smith_ggx(float ct, float alpha) {
  const float a = alpha * alpha, b = ct * ct;
  return 1.0f / (ct + std::sqrt(a + b - a * b));
}

// BXDF.evaluateDistributionFunction
inline V3 lobe_f(const Lobe& L, V3 wo, V3 wi) {
  switch (L.kind) {
    case kLambert: return L.scale * (1.0f / kPi);
    case kOrenNayar: {
      float cia = std::fabs(cos_t(wi)), coa = std::fabs(cos_t(wo));
      float sti = sin_t(wi), sto = sin_t(wo);
      float maxc = (sti > 1.0e-4f && sto > 1.0e-4f) ? std::fmax(0.0f, cos_phi(wi) * cos_phi(wo) + sin_phi(wi) * sin_phi(wo)) : 0.0f;
      float sa = cia > coa ? sto : sti;
      float tb = cia > coa ? sti / cia : sto / coa;
      return L.scale * (1.0f / kPi) * (L.a + L.b * maxc * sa * tb);
    }
    case kTSBRDF: {
      float co = std::fabs(cos_t(wo)), ci = std::fabs(cos_t(wi));
      if (co == 0.0f || ci == 0.0f) return {0, 0, 0};
      V3 h = wi + wo;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return {0, 0, 0};
      h = normalize(h);
      float D = tr_D(L, h), G = tr_G(L, wo, wi);
      V3 hf = dot(h, V3{0, 0, 1}) < 0.0f ? -h : h;  // faceForward(h, z)
      V3 F = fresnel_eval(L, dot(wi, hf));
      return mul(L.scale * D * G, F) * (1.0f / (4.0f * ci * co));
    }
    case kTSBTDF: {
      if (same_hemi(wo, wi)) return {0, 0, 0};
      float cti = cos_t(wi), cto = cos_t(wo);
      if (cti == 0.0f || cto == 0.0f) return {0, 0, 0};
      float eta = cto > 0.0f ? L.etaB / L.etaA : L.etaA / L.etaB;
      V3 ht = normalize(wi * eta + wo);
      V3 h = ht.z < 0.0f ? -ht : ht;
      float oh = dot(wo, h), ih = dot(wi, h);
      if (oh * ih > 0.0f) return {0, 0, 0};
      float F = fresnel_dielectric(oh, L.etaA, L.etaB);
      float a = oh + eta * ih;
      float b = 1.0f / eta;  // TransportMode.RADIANCE
      float D = tr_D(L, h), G = tr_G(L, wo, wi);
      float k = std::fabs(D * G * eta * eta * std::fabs(ih) * std::fabs(oh) * b * b / (cti * cto * a * a));
      return L.scale * (1.0f - F) * k;
    }
    case kLambertBTDF: return L.scale * (1.0f / kPi);
    case kFresnelBlend: {  // FresnelBlendBRDF.java:evaluateDistributionFunction (scale: diffuse, cK: specular)
      V3 h = wo + wi;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return {0, 0, 0};
      h = normalize(h);
      auto pow5 = [](float x) { return x * x * x * x * x; };
      const float a = 28.0f / (23.0f * kPi);
      const float b = 1.0f - pow5(1.0f - 0.5f * std::fabs(cos_t(wi)));
      const float c = 1.0f - pow5(1.0f - 0.5f * std::fabs(cos_t(wo)));
      const float d = tr_D(L, h);
      const float e = 4.0f * std::fabs(dot(wi, h)) * std::fmax(std::fabs(cos_t(wi)), std::fabs(cos_t(wo)));
      const float f = d / e;
      const float w = pow5(1.0f - dot(wi, h));
      const V3 ks = L.cK;
      const V3 fr = {ks.x + (1.0f - ks.x) * w, ks.y + (1.0f - ks.y) * w, ks.z + (1.0f - ks.z) * w};  // Schlick.fresnelDielectric
      const V3 diff = mul(L.scale * a, V3{1.0f - ks.x, 1.0f - ks.y, 1.0f - ks.z}) * b * c;
      return diff + fr * f;
    }
    case kDisneyDiffuse: {  // DisneyDiffuseBRDF.java:evaluateDistributionFunction
      const float fo = schlick_weight(std::fabs(cos_t(wo))), fi = schlick_weight(std::fabs(cos_t(wi)));
      const float a = 1.0f - fo / 2.0f, b = 1.0f - fi / 2.0f;
      return {L.scale.x * (1.0f / kPi) * a * b, L.scale.y * (1.0f / kPi) * a * b, L.scale.z * (1.0f / kPi) * a * b};
    }
    case kDisneyFakeSS: case kDisneyRetro: case kDisneySheen: {
      V3 h = wi + wo;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return {0, 0, 0};
      h = normalize(h);
      const float cd = dot(wi, h);
      if (L.kind == kDisneySheen) return L.scale * schlick_weight(cd);  // DisneySheenBRDF.java
      const float co = std::fabs(cos_t(wo)), ci = std::fabs(cos_t(wi));
      const float fo = schlick_weight(co), fi = schlick_weight(ci);
      if (L.kind == kDisneyRetro) {  // DisneyRetroBRDF.java
        const float a = 2.0f * L.roughness * cd * cd;
        const float b = fo + fi + fo * fi * (a - 1.0f);
        return {L.scale.x * (1.0f / kPi) * a * b, L.scale.y * (1.0f / kPi) * a * b, L.scale.z * (1.0f / kPi) * a * b};
      }
      const float f90 = cd * cd * L.roughness;  // DisneyFakeSSBRDF.java
      const float fss = lerpf(1.0f, f90, fo) * lerpf(1.0f, f90, fi);
      const float ss = 1.25f * (fss * (1.0f / (co + ci) - 0.5f) + 0.5f);
      return {L.scale.x * (1.0f / kPi) * ss, L.scale.y * (1.0f / kPi) * ss, L.scale.z * (1.0f / kPi) * ss};
    }
    case kDisneyClearCoat: {  // DisneyClearCoatBRDF.java
      V3 h = wi + wo;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return {0, 0, 0};
      h = normalize(h);
      const float d = gtr1(std::fabs(cos_t(h)), L.gloss);
      const float f = lerpf(0.04f, 1.0f, schlick_weight(dot(wo, h)));
      const float g = smith_ggx(std::fabs(cos_t(wo)), 0.25f) * smith_ggx(std::fabs(cos_t(wi)), 0.25f);
      const float c = L.weight * g * f * d / 4.0f;
      return {c, c, c};
    }
    default: return {0, 0, 0};  // specular lobes
  }
}
inline float lobe_pdf(const Lobe& L, V3 wo, V3 wi) {
  switch (L.kind) {
    case kLambert: case kOrenNayar: case kDisneyDiffuse: case kDisneyFakeSS: case kDisneyRetro: case kDisneySheen:
      return same_hemi(wo, wi) ? std::fabs(cos_t(wi)) * (1.0f / kPi) : 0.0f;
    case kLambertBTDF: return same_hemi(wo, wi) ? 0.0f : std::fabs(cos_t(wi)) * (1.0f / kPi);
    case kFresnelBlend: {
      if (!same_hemi(wo, wi)) return 0.0f;
      const V3 h = normalize(wo + wi);
      return 0.5f * (std::fabs(cos_t(wi)) * (1.0f / kPi) + tr_pdf(L, wo, h) / (4.0f * dot(wo, h)));
    }
    case kDisneyClearCoat: {
      if (!same_hemi(wo, wi)) return 0.0f;
      V3 h = wi + wo;
      if (h.x == 0.0f && h.y == 0.0f && h.z == 0.0f) return 0.0f;
      h = normalize(h);
      const float ch = std::fabs(cos_t(h));
      return gtr1(ch, L.gloss) * ch / (4.0f * dot(wo, h));
    }
    case kTSBRDF: {
      if (!same_hemi(wo, wi)) return 0.0f;
      V3 h = normalize(wo + wi);
      return tr_pdf(L, wo, h) / (4.0f * dot(wo, h));
    }
    case kTSBTDF: {
      if (same_hemi(wo, wi)) return 0.0f;
      float eta = cos_t(wo) > 0.0f ? L.etaB / L.etaA : L.etaA / L.etaB;
      V3 h = normalize(wi * eta + wo);
      float oh = dot(wo, h), ih = dot(wi, h);
      if (oh * ih > 0.0f) return 0.0f;
      float a = oh + eta * ih;
      float b = std::fabs((eta * eta * ih) / (a * a));
      return tr_pdf(L, wo, h) * b;
    }
    default: return 0.0f;
  }
}
struct LobeSample { V3 f; V3 wi; float pdf; int type; };
inline bool lobe_sample(const Lobe& L, V3 wo, float u, float v, LobeSample* s) {
  s->type = L.type;
  switch (L.kind) {
    case kLambert: case kOrenNayar: case kDisneyDiffuse: case kDisneyFakeSS: case kDisneyRetro: case kDisneySheen: {
      V3 wi = cosine_hemisphere(u, v);
      if (wo.z < 0.0f) wi.z = -wi.z;  // faceForwardZ
      s->wi = wi; s->f = lobe_f(L, wo, wi); s->pdf = lobe_pdf(L, wo, wi); return true;
    }
    case kLambertBTDF: {
      V3 wi = cosine_hemisphere(u, v);
      if (wo.z > 0.0f) wi.z = -wi.z;  // faceForwardZNegated
      s->wi = wi; s->f = lobe_f(L, wo, wi); s->pdf = lobe_pdf(L, wo, wi); return true;
    }
    case kFresnelBlend: {  // FresnelBlendBRDF.java:sampleDistributionFunction
      V3 wi;
      if (u < 0.5f) {
        wi = cosine_hemisphere(std::fmin(2.0f * u, 0.99999994f), v);
        if (wo.z < 0.0f) wi.z = -wi.z;
      } else {
        const V3 h = tr_sample_h(L, wo, std::fmin(2.0f * (u - 0.5f), 0.99999994f), v);
        wi = reflect_about(wo, h);
        if (!same_hemi(wo, wi)) return false;
      }
      s->wi = wi; s->f = lobe_f(L, wo, wi); s->pdf = lobe_pdf(L, wo, wi); return true;
    }
    case kDisneyClearCoat: {  // DisneyClearCoatBRDF.java:sampleDistributionFunction
      if (wo.z == 0.0f) return false;
      const float a2 = L.gloss * L.gloss;
      const float ct = std::sqrt(std::fmax(0.0f, (1.0f - std::pow(a2, 1.0f - u)) / (1.0f - a2)));
      const float st = std::sqrt(std::fmax(0.0f, 1.0f - ct * ct));
      const float phi = 2.0f * kPi * v;
      V3 h = {st * std::cos(phi), st * std::sin(phi), ct};
      if (!same_hemi(wo, h)) h = -h;
      const V3 wi = reflect_about(wo, h);
      if (!same_hemi(wo, wi)) return false;
      s->wi = wi; s->f = lobe_f(L, wo, wi); s->pdf = lobe_pdf(L, wo, wi); return true;
    }
    case kSpecBRDF: {
      V3 wi = {-wo.x, -wo.y, wo.z};
      s->wi = wi; s->f = mul(fresnel_eval(L, cos_t(wi)), L.scale) * (1.0f / std::fabs(cos_t(wi))); s->pdf = 1.0f; return true;
    }
    case kSpecBTDF: {
      bool entering = cos_t(wo) > 0.0f;
      float ei = entering ? L.etaA : L.etaB, et = entering ? L.etaB : L.etaA;
      V3 n = dot(V3{0, 0, 1}, wo) < 0.0f ? V3{0, 0, -1} : V3{0, 0, 1};
      V3 wi;
      if (!refract(wo, n, ei / et, &wi)) return false;
      float F = fresnel_dielectric(cos_t(wi), L.etaA, L.etaB);
      s->wi = wi; s->f = L.scale * (1.0f - F) * ((ei * ei) / (et * et)) * (1.0f / std::fabs(cos_t(wi))); s->pdf = 1.0f; return true;
    }
    case kFresnelSpec: {
      float F = fresnel_dielectric(cos_t(wo), L.etaA, L.etaB);
      if (u < F) {
        V3 wi = {-wo.x, -wo.y, wo.z};
        s->type = kSpecular | kRefl; s->wi = wi; s->f = L.scale * F * (1.0f / std::fabs(cos_t(wi))); s->pdf = F; return true;
      }
      bool entering = cos_t(wo) > 0.0f;
      float ei = entering ? L.etaA : L.etaB, et = entering ? L.etaB : L.etaA;
      V3 n = dot(V3{0, 0, 1}, wo) < 0.0f ? V3{0, 0, -1} : V3{0, 0, 1};
      V3 wi;
      if (!refract(wo, n, ei / et, &wi)) return false;
      s->type = kSpecular | kTrans; s->wi = wi;
      s->f = L.cK * (1.0f - F) * ((ei * ei) / (et * et)) * (1.0f / std::fabs(cos_t(wi)));  // cK holds the transmittance scale
      s->pdf = 1.0f - F; return true;
    }
    case kTSBRDF: {
      if (wo.z == 0.0f) return false;
      V3 h = tr_sample_h(L, wo, u, v);
      if (dot(wo, h) < 0.0f) return false;
      V3 wi = reflect_about(wo, h);
      if (!same_hemi(wo, wi)) return false;
      s->wi = wi; s->f = lobe_f(L, wo, wi); s->pdf = tr_pdf(L, wo, h) / (4.0f * dot(wo, h)); return true;
    }
    case kTSBTDF: {
      if (wo.z == 0.0f) return false;
      V3 h = tr_sample_h(L, wo, u, v);
      if (dot(wo, h) < 0.0f) return false;
      float eta = cos_t(wo) > 0.0f ? L.etaA / L.etaB : L.etaB / L.etaA;
      V3 wi;
      if (!refract(wo, h, eta, &wi)) return false;
      s->wi = wi; s->f = lobe_f(L, wo, wi); s->pdf = lobe_pdf(L, wo, wi); return true;
    }
  }
  return false;
}
inline bool type_matches(int lobe_type, int flags) { return (lobe_type & flags) == lobe_type; }
inline bool is_spec(int t) { return (t & kSpecular) != 0; }

// scene/material/MicrofacetDistribution.java:convertRoughnessToAlpha
inline float roughness_to_alpha(float r) {
  float x = std::fmax(r, 1.0e-3f), y = std::log(x);
  return 1.62142f + 0.819955f * y + 0.1734f * y * y + 0.0171201f * y * y * y + 0.000640711f * y * y * y * y;
}
inline Lobe make_tr_lobe(LobeKind k, int type, V3 scale, float ax, float ay) {
  Lobe L{}; L.kind = k; L.type = type; L.scale = scale; L.ax = std::fmax(ax, 0.001f); L.ay = std::fmax(ay, 0.001f); return L;
}

// Material.computeScatteringFunctions for Matte/Mirror/Glass/Metal/Plastic
// (scene/material/*Material.java) decoded from the compiled records
// (scene/compiler/CompiledMaterialCache.java:2830-3294).
// u_material: the random number a material draws when it builds its BSDF
// (ClearCoatMaterial.java:323, Floats.random()).
inline bool build_bsdf_material(const Scene& sc, int mid, int moff, const Hit& h, bool multi, float u_material, Bsdf* B, bool* supported) {
  *supported = true;
  B->n = 0; B->eta = 1.0f; B->present = false;
  TexRef a, b;
  switch (mid) {
    case kMatMatte: {
      const auto& M = sc.I("materialMatteMaterialArray");
      material_slot(sc, M, moff, 1, &a, &b);  // angle, KD
      V3 kd = sat0(tex_color(sc, b));
      float ang = saturate(tex_float(sc, a), 0.0f, 90.0f) * (kPi / 180.0f);
      Lobe L{}; L.type = kRefl | kDiffuse; L.scale = kd;
      if (ang == 0.0f) { L.kind = kLambert; }
      else { L.kind = kOrenNayar; float s2 = ang * ang; L.a = 1.0f - (s2 / (2.0f * (s2 + 0.33f))); L.b = 0.45f * s2 / (s2 + 0.09f); }
      B->l[B->n++] = L; break;
    }
    case kMatMirror: {
      const auto& M = sc.I("materialMirrorMaterialArray");
      material_slot(sc, M, moff, 1, &a, &b);
      V3 kr = sat0(tex_color(sc, a));
      if (black(kr)) return false;
      Lobe L{}; L.kind = kSpecBRDF; L.type = kRefl | kSpecular; L.scale = kr; L.fk = kFresConst;
      B->l[B->n++] = L; break;
    }
    case kMatGlass: {
      const auto& M = sc.I("materialGlassMaterialArray");
      TexRef te, tz, tkr, tkt, tru, trv;
      material_slot(sc, M, moff, 1, &te, &tz);
      material_slot(sc, M, moff, 2, &tkr, &tkt);
      material_slot(sc, M, moff, 3, &tru, &trv);
      bool remap = material_int(sc, M, moff, 4) != 0;
      V3 kr = sat0(tex_color(sc, tkr)), kt = sat0(tex_color(sc, tkt));
      float eta = tex_float(sc, te), ru = tex_float(sc, tru), rv = tex_float(sc, trv);
      if (black(kr) && black(kt)) return false;
      B->eta = eta;
      bool specular = ru == 0.0f && rv == 0.0f;
      if (specular && multi) {
        Lobe L{}; L.kind = kFresnelSpec; L.type = kRefl | kTrans | kSpecular; L.scale = kr; L.cK = kt; L.etaA = 1.0f; L.etaB = eta;
        B->l[B->n++] = L;
      } else if (specular) {
        if (!black(kr)) { Lobe L{}; L.kind = kSpecBRDF; L.type = kRefl | kSpecular; L.scale = kr; L.fk = kFresDielectric; L.etaI = 1.0f; L.etaT = eta; B->l[B->n++] = L; }
        if (!black(kt)) { Lobe L{}; L.kind = kSpecBTDF; L.type = kTrans | kSpecular; L.scale = kt; L.etaA = 1.0f; L.etaB = eta; B->l[B->n++] = L; }
      } else {
        float au = remap ? roughness_to_alpha(ru) : ru, av = remap ? roughness_to_alpha(rv) : rv;
        if (!black(kr)) { Lobe L = make_tr_lobe(kTSBRDF, kRefl | kGlossy, kr, au, av); L.fk = kFresDielectric; L.etaI = 1.0f; L.etaT = eta; B->l[B->n++] = L; }
        if (!black(kt)) { Lobe L = make_tr_lobe(kTSBTDF, kTrans | kGlossy, kt, au, av); L.etaA = 1.0f; L.etaB = eta; B->l[B->n++] = L; }
      }
      break;
    }
    case kMatMetal: {
      const auto& M = sc.I("materialMetalMaterialArray");
      TexRef teta, tk, tru, trv;
      material_slot(sc, M, moff, 1, &teta, &tk);
      material_slot(sc, M, moff, 2, &tru, &trv);
      bool remap = material_int(sc, M, moff, 3) != 0;
      float ru = tex_float(sc, tru), rv = tex_float(sc, trv);
      float au = remap ? roughness_to_alpha(ru) : ru, av = remap ? roughness_to_alpha(rv) : rv;
      Lobe L = make_tr_lobe(kTSBRDF, kRefl | kGlossy, V3{1, 1, 1}, au, av);
      L.fk = kFresConductor; L.cEtaI = {1, 1, 1}; L.cEtaT = tex_color(sc, teta); L.cK = tex_color(sc, tk);
      B->l[B->n++] = L; break;
    }
    case kMatPlastic: {
      const auto& M = sc.I("materialPlasticMaterialArray");
      TexRef tkd, tks, tr, tz;
      material_slot(sc, M, moff, 1, &tkd, &tks);
      material_slot(sc, M, moff, 2, &tr, &tz);
      bool remap = material_int(sc, M, moff, 3) != 0;
      V3 kd = sat0(tex_color(sc, tkd)), ks = sat0(tex_color(sc, tks));
      if (!black(kd)) { Lobe L{}; L.kind = kLambert; L.type = kRefl | kDiffuse; L.scale = kd; B->l[B->n++] = L; }
      if (!black(ks)) {
        float r = tex_float(sc, tr);
        float al = remap ? roughness_to_alpha(r) : r;
        Lobe L = make_tr_lobe(kTSBRDF, kRefl | kGlossy, ks, al, al);
        L.fk = kFresDielectric; L.etaI = 1.5f; L.etaT = 1.0f;
        B->l[B->n++] = L;
      }
      if (B->n == 0) return false;
      break;
    }
    case kMatDisney: {  // scene/material/DisneyMaterial.java:1121-1210 (ConstantTexture values)
      const auto& M = sc.I("materialDisneyMaterialArray");
      TexRef t_aniso, t_z, t_cc, t_ccg, t_color, t_dt, t_eta, t_flat, t_met, t_rough, t_sd, t_sheen, t_sheen_tint, t_spec_tint, t_st, t_thin;
      material_slot(sc, M, moff, 1, &t_aniso, &t_z);  // CompiledMaterialCache.java:2751-2759
      material_slot(sc, M, moff, 2, &t_cc, &t_ccg);
      material_slot(sc, M, moff, 3, &t_color, &t_dt);
      material_slot(sc, M, moff, 4, &t_eta, &t_flat);
      material_slot(sc, M, moff, 5, &t_met, &t_rough);
      material_slot(sc, M, moff, 6, &t_sd, &t_sheen);
      material_slot(sc, M, moff, 7, &t_sheen_tint, &t_spec_tint);
      material_slot(sc, M, moff, 8, &t_st, &t_thin);  // second pair: (isThin, 0)
      const bool thin = t_thin.id != 0;
      const float aniso = tex_float(sc, t_aniso), cc = tex_float(sc, t_cc), dt = tex_float(sc, t_dt) / 2.0f;
      const float eta = tex_float(sc, t_eta), met = tex_float(sc, t_met), rough = tex_float(sc, t_rough);
      const float sheen = tex_float(sc, t_sheen), spec_tint = tex_float(sc, t_spec_tint), st = tex_float(sc, t_st);
      const V3 color = sat0(tex_color(sc, t_color));
      const float lum = color.x * 0.212671f + color.y * 0.715160f + color.z * 0.072169f;  // Color3F.relativeLuminance
      const V3 tint = lum > 0.0f ? V3{color.x / lum, color.y / lum, color.z / lum} : V3{1, 1, 1};
      const float sht = tex_float(sc, t_sheen_tint);
      const V3 sheen_c = sheen > 0.0f ? V3{lerpf(1.0f, tint.x, sht), lerpf(1.0f, tint.y, sht), lerpf(1.0f, tint.z, sht)} : V3{0, 0, 0};
      const float dw = (1.0f - met) * (1.0f - st);
      auto add = [&](Lobe L) { B->l[B->n++] = L; };
      auto diffuse_lobe = [](LobeKind k, V3 scale, float r) { Lobe L{}; L.kind = k; L.type = kRefl | kDiffuse; L.scale = scale; L.roughness = r; return L; };
      if (dw > 0.0f) {
        if (thin) {
          const float flat = tex_float(sc, t_flat);
          add(diffuse_lobe(kDisneyDiffuse, color * (dw * (1.0f - flat) * (1.0f - dt)), 0.0f));
          add(diffuse_lobe(kDisneyFakeSS, color * (dw * (0.0f + flat) * (1.0f - dt)), rough));
        } else if (black(tex_color(sc, t_sd))) {
          add(diffuse_lobe(kDisneyDiffuse, color * dw, 0.0f));
        } else {
          Lobe L{}; L.kind = kSpecBTDF; L.type = kTrans | kSpecular; L.scale = {1, 1, 1}; L.etaA = 1.0f; L.etaB = eta; add(L);
        }
        add(diffuse_lobe(kDisneyRetro, color * dw, rough));
        if (sheen > 0.0f) add(diffuse_lobe(kDisneySheen, sheen_c * (dw * sheen), 0.0f));
      }
      const float aspect = std::sqrt(1.0f - aniso * 0.9f);
      const float ax = std::fmax(0.001f, rough * rough / aspect), ay = std::fmax(0.001f, rough * rough * aspect);
      const float r0 = ((eta - 1.0f) * (eta - 1.0f)) / ((eta + 1.0f) * (eta + 1.0f));
      const V3 tinted = V3{lerpf(1.0f, tint.x, spec_tint), lerpf(1.0f, tint.y, spec_tint), lerpf(1.0f, tint.z, spec_tint)} * r0;
      {
        Lobe L = make_tr_lobe(kTSBRDF, kRefl | kGlossy, V3{1, 1, 1}, ax, ay);
        L.separable = true;
        L.fk = kFresDisney; L.etaT = eta; L.metallic = met;
        L.r0 = {lerpf(tinted.x, color.x, met), lerpf(tinted.y, color.y, met), lerpf(tinted.z, color.z, met)};
        add(L);
      }
      if (cc > 0.0f) {
        Lobe L{}; L.kind = kDisneyClearCoat; L.type = kRefl | kGlossy; L.gloss = lerpf(0.1f, 0.001f, tex_float(sc, t_ccg)); L.weight = cc;
        add(L);
      }
      if (st > 0.0f) {
        const V3 ts = V3{std::sqrt(color.x), std::sqrt(color.y), std::sqrt(color.z)} * st;
        Lobe L;
        if (thin) {
          const float rs = (0.65f * eta - 0.35f) * rough;
          L = make_tr_lobe(kTSBTDF, kTrans | kGlossy, ts, std::fmax(0.001f, rs * rs / aspect), std::fmax(0.001f, rs * rs * aspect));
          L.separable = false;
        } else {
          L = make_tr_lobe(kTSBTDF, kTrans | kGlossy, ts, ax, ay);
          L.separable = true;
        }
        L.etaA = 1.0f; L.etaB = eta;
        add(L);
      }
      if (thin) { Lobe L{}; L.kind = kLambertBTDF; L.type = kTrans | kDiffuse; L.scale = color * dt; add(L); }
      break;
    }
    case kMatClearCoat: {  // scene/material/ClearCoatMaterial.java:computeScatteringFunctions
      const auto& M = sc.I("materialClearCoatMaterialArray");
      material_slot(sc, M, moff, 1, &a, &b);
      const V3 kd = tex_color(sc, a), ks = tex_color(sc, b);
      const V3 d = h.w.ray.d, n = h.w.s.w;
      const V3 nco = dot(n, d) > 0.0f ? -n : n;  // Intersection.getSurfaceNormalSCorrectlyOriented
      const bool entering = dot(n, nco) > 0.0f;
      const float etaI = entering ? 1.0f : 1.5f, etaT = entering ? 1.5f : 1.0f;
      V3 refr;
      Lobe L{};
      if (refract(d, nco, etaI / etaT, &refr)) {  // Vector3F.refraction(direction, normal, eta)
        const float cosi = dot(d, nco);
        const float cosc = entering ? -cosi : dot(refr, n);
        const float R = fresnel_dielectric(cosc, 1.0f, 1.5f), T = 1.0f - R;
        const float p = 0.25f + 0.5f * R;
        if (u_material < p) { L.kind = kSpecBRDF; L.type = kRefl | kSpecular; L.scale = ks * (R / p); L.fk = kFresConst; }
        else { L.kind = kLambert; L.type = kRefl | kDiffuse; L.scale = kd * (T / (1.0f - p)); }
      } else {
        L.kind = kSpecBRDF; L.type = kRefl | kSpecular; L.scale = ks; L.fk = kFresConst;
      }
      B->l[B->n++] = L;
      break;
    }
    case kMatGlossy: {  // scene/material/GlossyMaterial.java: TorranceSparrowBRDF(kr, ConductorFresnel(kr, 1, 1), TR(r, r))
      const auto& M = sc.I("materialGlossyMaterialArray");
      material_slot(sc, M, moff, 1, &a, &b);
      const V3 kr = tex_color(sc, a);
      const float r = tex_float(sc, b);
      Lobe L = make_tr_lobe(kTSBRDF, kRefl | kGlossy, kr, r, r);
      L.fk = kFresConductor; L.cEtaI = kr; L.cEtaT = {1, 1, 1}; L.cK = {1, 1, 1};
      B->l[B->n++] = L;
      break;
    }
    case kMatSubstrate: {  // scene/material/SubstrateMaterial.java
      const auto& M = sc.I("materialSubstrateMaterialArray");
      TexRef tkd, tks, tru, trv;
      material_slot(sc, M, moff, 1, &tkd, &tks);
      material_slot(sc, M, moff, 2, &tru, &trv);
      const bool remap = material_int(sc, M, moff, 3) != 0;
      const V3 kd = sat0(tex_color(sc, tkd)), ks = sat0(tex_color(sc, tks));
      if (black(kd) && black(ks)) return false;
      const float ru = tex_float(sc, tru), rv = tex_float(sc, trv);
      Lobe L = make_tr_lobe(kFresnelBlend, kRefl | kGlossy, kd, remap ? roughness_to_alpha(ru) : ru, remap ? roughness_to_alpha(rv) : rv);
      L.cK = ks;
      B->l[B->n++] = L;
      break;
    }
    case kMatTranslucent: {  // scene/material/TranslucentMaterial.java
      const auto& M = sc.I("materialTranslucentMaterialArray");
      TexRef tkd, tks, trf, ttr, trg, tz;
      material_slot(sc, M, moff, 1, &tkd, &tks);
      material_slot(sc, M, moff, 2, &trf, &ttr);
      material_slot(sc, M, moff, 3, &trg, &tz);  // second pair: (isRemappingRoughness, 0)
      const V3 refl = sat0(tex_color(sc, trf)), tr = sat0(tex_color(sc, ttr));
      if (black(refl) && black(tr)) return false;
      const V3 kd = sat0(tex_color(sc, tkd)), ks = sat0(tex_color(sc, tks));
      if (!black(kd)) {
        if (!black(refl)) { Lobe L{}; L.kind = kLambert; L.type = kRefl | kDiffuse; L.scale = mul(kd, refl); B->l[B->n++] = L; }
        if (!black(tr)) { Lobe L{}; L.kind = kLambertBTDF; L.type = kTrans | kDiffuse; L.scale = mul(kd, tr); B->l[B->n++] = L; }
      }
      if (!black(ks)) {
        const float r = tex_float(sc, trg);
        const float al = tz.id != 0 ? roughness_to_alpha(r) : r;
        if (!black(refl)) {
          Lobe L = make_tr_lobe(kTSBRDF, kRefl | kGlossy, mul(ks, refl), al, al);
          L.fk = kFresDielectric; L.etaI = 1.0f; L.etaT = 1.5f; B->l[B->n++] = L;
        }
        if (!black(tr)) {
          Lobe L = make_tr_lobe(kTSBTDF, kTrans | kGlossy, mul(ks, tr), al, al);
          L.etaA = 1.0f; L.etaB = 1.5f; B->l[B->n++] = L;
        }
      }
      if (B->n == 0) return false;
      break;
    }
    case kMatUber: {  // scene/material/UberMaterial.java
      const auto& M = sc.I("materialUberMaterialArray");
      TexRef tkd, tkr, tks, tkt, teta, top, tru, trv;
      material_slot(sc, M, moff, 1, &tkd, &tkr);
      material_slot(sc, M, moff, 2, &tks, &tkt);
      material_slot(sc, M, moff, 3, &teta, &top);
      material_slot(sc, M, moff, 4, &tru, &trv);
      const bool remap = material_int(sc, M, moff, 5) != 0;
      const V3 op = sat0(tex_color(sc, top));
      const V3 kd = mul(op, sat0(tex_color(sc, tkd))), kr = mul(op, sat0(tex_color(sc, tkr)));
      const V3 ks = mul(op, sat0(tex_color(sc, tks))), kt = mul(op, sat0(tex_color(sc, tkt)));
      const V3 ts = sat0(V3{1.0f - op.x, 1.0f - op.y, 1.0f - op.z});
      const float eta = tex_float(sc, teta);
      const float ru = tex_float(sc, tru), rv = tex_float(sc, trv);
      const float au = remap ? roughness_to_alpha(ru) : ru, av = remap ? roughness_to_alpha(rv) : rv;
      if (!black(ts)) { Lobe L{}; L.kind = kSpecBTDF; L.type = kTrans | kSpecular; L.scale = ts; L.etaA = 1.0f; L.etaB = 1.0f; B->l[B->n++] = L; }
      if (!black(kd)) { Lobe L{}; L.kind = kLambert; L.type = kRefl | kDiffuse; L.scale = kd; B->l[B->n++] = L; }
      if (!black(ks)) { Lobe L = make_tr_lobe(kTSBRDF, kRefl | kGlossy, ks, au, av); L.fk = kFresDielectric; L.etaI = 1.0f; L.etaT = eta; B->l[B->n++] = L; }
      if (!black(kr)) { Lobe L{}; L.kind = kSpecBRDF; L.type = kRefl | kSpecular; L.scale = kr; L.fk = kFresDielectric; L.etaI = 1.0f; L.etaT = eta; B->l[B->n++] = L; }
      if (!black(kt)) { Lobe L{}; L.kind = kSpecBTDF; L.type = kTrans | kSpecular; L.scale = kt; L.etaA = 1.0f; L.etaB = eta; B->l[B->n++] = L; }
      B->eta = black(ts) ? eta : 1.0f;  // BSDF(intersection, bXDFs, false, eta)
      break;  // a BSDF even with no lobes: the path ends there instead of passing through
    }
    default: *supported = false; return false;
  }
  B->present = true;
  B->s = h.w.s; B->ng = h.w.g.w;
  B->wo_world = -h.w.ray.d;
  B->wo = normalize(to_local(B->wo_world, B->s));
  B->nl = normalize(to_local(B->s.w, B->s));
  return true;
}

inline const char* material_array(int mid) {
  switch (mid) {
    case kMatMatte: return "materialMatteMaterialArray";
    case kMatMirror: return "materialMirrorMaterialArray";
    case kMatGlass: return "materialGlassMaterialArray";
    case kMatMetal: return "materialMetalMaterialArray";
    case kMatPlastic: return "materialPlasticMaterialArray";
    case kMatDisney: return "materialDisneyMaterialArray";
    case kMatClearCoat: return "materialClearCoatMaterialArray";
    case kMatGlossy: return "materialGlossyMaterialArray";
    case kMatSubstrate: return "materialSubstrateMaterialArray";
    case kMatTranslucent: return "materialTranslucentMaterialArray";
    case kMatUber: return "materialUberMaterialArray";
    default: return nullptr;
  }
}

// BullseyeMaterial / CheckerboardMaterial / PolkaDotMaterial.doGetMaterial
// (scene/material/*Material.java), repeated while the pick is itself composite.
// Records are float arrays at absolute offsets; A and B are Ints.pack(id, offset).
inline void resolve_material(const Scene& sc, const Hit& h, int* mid, int* moff) {
  for (int guard = 0; guard < 64; ++guard) {
    const float* q;
    bool a;
    if (*mid == kMatBullseye) {
      q = sc.F("materialBullseyeMaterialArray").data() + *moff;
      a = jmod(length(h.p_obj - V3{q[0], q[1], q[2]}) * q[5], 1.0f) > 0.5f;
      q += 3;
    } else if (*mid == kMatCheckerboard) {
      q = sc.F("materialCheckerboardMaterialArray").data() + *moff;
      const float cs = jcos(q[1]), sn = jsin(q[1]), u = h.w.tu, v = h.w.tv;
      a = (frac((u * cs - v * sn) * q[4]) > 0.5f) ^ (frac((v * cs + u * sn) * q[5]) > 0.5f);
      q += 2;
    } else if (*mid == kMatPolkaDot) {
      q = sc.F("materialPolkaDotMaterialArray").data() + *moff;
      const float cs = jcos(q[1]), sn = jsin(q[1]), u = h.w.tu, v = h.w.tv;
      const float x = frac((u * cs - v * sn) * q[4]) - 0.5f, y = frac((v * cs + u * sn) * q[4]) - 0.5f;
      a = x * x + y * y < q[5] * q[5];
      q += 2;
    } else {
      return;
    }
    const TexRef r = unpack16(a ? q[0] : q[1]);
    *mid = r.id; *moff = r.off;
  }
  *mid = -1;  // a cycle: no material
}

// Intersection.setSurfaceNormalS: the shading frame rebuilt around n with the old v (OrthonormalBasis33F(w, v)).
inline void set_normal_s(Hit* h, V3 n) {
  const V3 w = normalize(n);
  const V3 u = normalize(cross(normalize(h->w.s.v), w));
  ONB o;
  o.w = w; o.u = u; o.v = cross(w, u);
  h->w.s = o;
}

// Modifier.modify (scene/modifier/*.java): the material's modifier, slot 0 texture B.
inline void apply_modifier(const Scene& sc, int mid, int moff, Hit* h) {
  const char* name = material_array(mid);
  if (!name) return;
  TexRef e, m;
  material_slot(sc, sc.I(name), moff, 0, &e, &m);
  if (m.id == kModNormalMapLDRImage) {  // NormalMapLDRImageModifier.modify: nearest texel, in the geometric frame
    const int abs_off = sc.I("modifierNormalMapLDRImageModifierOffsetArray")[m.off];
    const float* q = sc.F("modifierNormalMapLDRImageModifierArray").data() + abs_off;
    float x, y;
    image_point(q, h->w.tu, h->w.tv, &x, &y);
    const V3 c = image_texel(q, (int)x, (int)y);
    const V3 l{c.x * 2.0f - 1.0f, c.y * 2.0f - 1.0f, c.z * 2.0f - 1.0f};
    const ONB& g = h->w.g;  // Vector3F.transform(v, ONB): u * v.x + v * v.y + w * v.z
    const V3 n{l.x * g.u.x + l.y * g.v.x + l.z * g.w.x, l.x * g.u.y + l.y * g.v.y + l.z * g.w.y, l.x * g.u.z + l.y * g.v.z + l.z * g.w.z};
    set_normal_s(h, normalize(n));
  } else if (m.id == kModSimplexNoiseNormalMap) {  // SimplexNoiseNormalMapModifier.modify
    const float* q = sc.F("modifierSimplexNoiseNormalMapModifierArray").data() + (size_t)m.off * 2;
    const float freq = q[0], scale = q[1], rf = 1.0f / freq;
    const V3 p = h->w.p, n = h->w.s.w;
    const float x0 = p.x * rf, y0 = p.y * rf, z0 = p.z * rf;
    const float x1 = n.x + dfo_noise::simplex_fbm(x0, y0, z0, freq, 0.5f, -0.25f, 0.25f, 16) * scale;
    const float y1 = n.y + dfo_noise::simplex_fbm(y0, z0, x0, freq, 0.5f, -0.25f, 0.25f, 16) * scale;
    const float z1 = n.z + dfo_noise::simplex_fbm(z0, x0, y0, freq, 0.5f, -0.25f, 0.25f, 16) * scale;
    set_normal_s(h, normalize(V3{x1, y1, z1}));
  }
}

// Material.computeScatteringFunctions: composite materials pick their material,
// the material's modifier changes the shading frame of the hit (kept for the
// rest of the bounce, as the reference's Intersection is), then the textures
// are evaluated at the modified hit.
inline bool build_bsdf(const Scene& sc, int mid, int moff, Hit& h, bool multi, float u_material, Bsdf* B, bool* supported) {
  resolve_material(sc, h, &mid, &moff);
  apply_modifier(sc, mid, moff, &h);
  const TexCtx c = tex_ctx(h);
  g_tex = &c;
  const bool r = build_bsdf_material(sc, mid, moff, h, multi, u_material, B, supported);
  g_tex = nullptr;
  return r;
}

// Material.emittance (the emission texture of every supported material is slot 0, texture A)
inline V3 material_emission(const Scene& sc, const Hit& h, int mid, int moff) {
  resolve_material(sc, h, &mid, &moff);
  const char* name = material_array(mid);
  if (!name) return {0, 0, 0};
  TexRef a, b;
  material_slot(sc, sc.I(name), moff, 0, &a, &b);
  const TexCtx c = tex_ctx(h);
  g_tex = &c;
  const V3 e = tex_color(sc, a);
  g_tex = nullptr;
  return e;
}

// scene/BSDF.java:evaluateDistributionFunction / evaluateProbabilityDensityFunction / sampleDistributionFunction
inline V3 bsdf_f(const Bsdf& B, int flags, V3 wi_world) {
  V3 wi = normalize(to_local(wi_world, B.s));
  float idn = dot(wi_world, B.ng), odn = dot(B.wo_world, B.ng);
  bool refl = idn * odn > 0.0f;
  V3 r = {0, 0, 0};
  for (int k = 0; k < B.n; ++k) {
    const Lobe& L = B.l[k];
    if (type_matches(L.type, flags) && ((refl && (L.type & kRefl)) || (!refl && (L.type & kTrans)))) r = r + lobe_f(L, B.wo, wi);
  }
  return r;
}
inline float bsdf_pdf(const Bsdf& B, int flags, V3 wi_world) {
  if (B.n == 0) return 0.0f;
  V3 wi = normalize(to_local(wi_world, B.s));
  if (B.wo.z == 0.0f) return 0.0f;
  float p = 0.0f; int m = 0;
  for (int k = 0; k < B.n; ++k) if (type_matches(B.l[k].type, flags)) { ++m; p += lobe_pdf(B.l[k], B.wo, wi); }
  if (m > 1) p /= m;
  return p;
}
struct BsdfSample { V3 f; V3 wi; float pdf; int type; };
inline bool bsdf_sample(const Bsdf& B, int flags, float u, float v, BsdfSample* out) {
  if (B.wo.z == 0.0f) return false;
  int idx[kMaxLobes]; int m = 0;
  for (int k = 0; k < B.n; ++k) if (type_matches(B.l[k].type, flags)) idx[m++] = k;
  if (m == 0) return false;
  int match = std::min((int)std::floor(u * m), m - 1);
  const Lobe& L = B.l[idx[match]];
  float ur = std::fmin(u * m - match, 0.99999994f);
  LobeSample s;
  if (!lobe_sample(L, B.wo, ur, v, &s)) return false;
  V3 wiw = normalize(to_world(s.wi, B.s));
  V3 f = s.f; float pdf = s.pdf;
  if (!is_spec(L.type)) {
    float idn = dot(wiw, B.ng), odn = dot(B.wo_world, B.ng);
    bool refl = idn * odn > 0.0f;
    f = {0, 0, 0};
    for (int k = 0; k < m; ++k) {
      const Lobe& O = B.l[idx[k]];
      if (k != match) pdf += lobe_pdf(O, B.wo, s.wi);
      if ((refl && (O.type & kRefl)) || (!refl && (O.type & kTrans))) f = f + lobe_f(O, B.wo, s.wi);
    }
  }
  if (m > 1) pdf /= m;
  out->f = f; out->wi = wiw; out->pdf = pdf; out->type = s.type;
  return true;
}
inline int bsdf_count_nonspecular(const Bsdf& B) { int c = 0; for (int k = 0; k < B.n; ++k) if (!is_spec(B.l[k].type)) ++c; return c; }

// ---- lights ---------------------------------------------------------------
struct LightSample { V3 L; V3 p; V3 wi; float pdf; };

inline float dist1_value(const float* a, int off, int idx) { return a[off + 4 + idx + (int)a[off + 1]]; }
inline float dist1_cdf(const float* a, int off, int idx) { return a[off + 4 + idx]; }
inline int dist1_count(const float* a, int off) { return (int)a[off + 2]; }
inline float dist1_integral(const float* a, int off) { return a[off + 3]; }
// sampler/Distribution1F.java:index (array form)
inline int dist1_index(const float* a, int off, float value) {
  int len = (int)a[off + 1];
  int mn = 0, cl = len;
  while (cl > 0) {
    int half = cl >> 1, mid = mn + half;
    if (dist1_cdf(a, off, mid) <= value) { mn = mid + 1; cl -= half + 1; } else { cl = half; }
  }
  int r = mn - 1;
  return r < 0 ? 0 : (r > len - 2 ? len - 2 : r);
}
inline float dist1_remap(const float* a, int off, float value, int idx) {
  int n = dist1_count(a, off);
  float c0 = dist1_cdf(a, off, idx), c1 = dist1_cdf(a, off, idx + 1);
  if (c1 - c0 > 0.0f) return (idx + ((value - c0) / (c1 - c0))) / n;
  return (idx + (value - c0)) / n;
}
// sampler/Distribution2F.java: continuousRemap / continuousProbabilityDensityFunction(remapped = true)
inline void dist2_remap(const float* a, int off, float su, float sv, float* ou, float* ov) {
  bool uv = (int)a[off] != 0;
  float m = uv ? su : sv, c = uv ? sv : su;
  int offM = off + (int)a[off + 2];
  int iM = dist1_index(a, offM, m);
  int offC = off + (int)a[off + 3 + iM];
  int iC = dist1_index(a, offC, c);
  float mr = dist1_remap(a, offM, m, iM), cr = dist1_remap(a, offC, c, iC);
  *ou = uv ? mr : cr; *ov = uv ? cr : mr;
}
inline float dist2_pdf_remapped(const float* a, int off, float su, float sv) {
  bool uv = (int)a[off] != 0;
  float m = uv ? su : sv, c = uv ? sv : su;
  int offM = off + (int)a[off + 2];
  int nM = dist1_count(a, offM);
  int iM = std::max(0, std::min((int)(m * nM), nM - 1));
  int offC = off + (int)a[off + 3 + iM];
  int nC = dist1_count(a, offC);
  int iC = std::max(0, std::min((int)(c * nC), nC - 1));
  return dist1_value(a, offC, iC) / dist1_integral(a, offM);
}

inline V3 xyz_to_srgb_linear(V3 c);  // below

// scene/light/ImageLight.java:544 doRadianceSky over the compiled record
// (CompiledLightCache.java:1393-1460: angle +32, scale +33, resolution +36,
// image +2352): Point2F.sphericalCoordinates -> rotateCounterclockwise ->
// scale -> toImage, then ImageF.getColorRGB(x, y, WRAP_AROUND) (bilinear).
inline V3 image_sky(const float* q, V3 d) {
  const float phi = spherical_phi(d.x, d.y);  // Vector3F.sphericalPhi
  const float theta = std::acos(saturate(d.z, -1.0f, 1.0f));
  const float u = phi * (1.0f / (2.0f * kPi)), v = theta * (1.0f / kPi);
  const float c = std::cos(q[32]), s = std::sin(q[32]);
  const float ur = u * c - v * s, vr = v * c + u * s;
  const float us = ur * q[33], vs = vr * q[34];
  const float rx = q[36], ry = q[37];
  auto posmod = [](float x, float y) { return x < 0.0f ? std::fmod(std::fmod(x, y) + y, y) : std::fmod(x, y); };
  const float x = posmod(us * rx - 0.5f, rx), y = posmod(vs * ry - 0.5f, ry);
  const int w = (int)rx, h = (int)ry;
  const int x0 = (int)std::floor(x), x1 = (int)std::ceil(x), y0 = (int)std::floor(y), y1 = (int)std::ceil(y);
  auto px = [&](int ix, int iy) {
    ix = ((ix % w) + w) % w; iy = ((iy % h) + h) % h;  // PixelOperation.WRAP_AROUND
    const float* p = q + 2352 + ((size_t)iy * w + ix) * 3;
    return V3{p[0], p[1], p[2]};
  };
  if (x0 == x1 && y0 == y1) return px(x0, y0);
  const float xf = x - (float)x0, yf = y - (float)y0;
  auto lerp3 = [](V3 a, V3 b, float t) { return V3{lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t)}; };
  return lerp3(lerp3(px(x0, y0), px(x1, y0), xf), lerp3(px(x0, y1), px(x1, y1), xf), yf);
}

// scene/light/PerezLight.java:doRadianceSky (GPU form: renderer/gpu/AbstractLightKernel.java:1615)
inline V3 perez_sky(const float* q, V3 dir) {
  if (dir.z < 0.0f) return {0, 0, 0};
  V3 ds = normalize(V3{dir.x, dir.y, std::fmax(dir.z, 0.001f)});
  double T = q[41];
  double theta = std::acos(saturate(ds.z, -1.0f, 1.0f));
  V3 sun = {q[35], q[36], q[37]};
  double gamma = std::acos(saturate(dot(ds, sun), -1.0f, 1.0f));
  double thS = q[46];
  double pl[5] = {0.17872 * T - 1.46303, -0.35540 * T + 0.42749, -0.02266 * T + 5.32505, 0.12064 * T - 2.57705, -0.06696 * T + 0.37027};
  double px[5] = {-0.01925 * T - 0.25922, -0.06651 * T + 0.00081, -0.00041 * T + 0.21247, -0.06409 * T - 0.89887, -0.00325 * T + 0.04517};
  double py[5] = {-0.01669 * T - 0.26078, -0.09495 * T + 0.00921, -0.00792 * T + 0.21023, -0.04405 * T - 1.65369, -0.01092 * T + 0.05291};
  auto perez = [&](const double* l, double lvz) {
    double den = (1.0 + l[0] * std::exp(l[1])) * (1.0 + l[2] * std::exp(l[3] * thS) + l[4] * std::cos(thS) * std::cos(thS));
    double num = (1.0 + l[0] * std::exp(l[1] / std::cos(theta))) * (1.0 + l[2] * std::exp(l[3] * gamma) + l[4] * std::cos(gamma) * std::cos(gamma));
    return lvz * num / den;
  };
  double Y = perez(pl, q[42]) * 0.0001;
  double x = perez(px, q[43]);
  double y = perez(py, q[44]);
  // curve/ChromaticSpectralCurveF.java:167 (CIE daylight basis integrated to XYZ)
  float fx = (float)x, fy = (float)y;
  float m1 = (-1.3515f - 1.7703f * fx + 5.9114f * fy) / (0.0241f + 0.2562f * fx - 0.7341f * fy);
  float m2 = (0.03f - 31.4424f * fx + 30.0717f * fy) / (0.0241f + 0.2562f * fx - 0.7341f * fy);
  float X = 95.6824722290f + m1 * 1.7548348904f + m2 * 1.9917192459f;
  float Yc = 99.7036819458f + m1 * 1.8025954962f + m2 * 0.7136800885f;
  float Z = 115.5248031616f + m1 * 32.5218048096f + m2 * -2.1984319687f;
  V3 xyz = {(float)(X * Y / Yc), (float)Y, (float)(Z * Y / Yc)};
  return xyz_to_srgb_linear(xyz);
}

struct ColorSpace {  // color/ColorSpaceF.java:116; the default is sRGB (:85)
  float xyz2rgb[9];
  float rgb2xyz[9];
  float breakPoint, gammaV, slope, slopeMatch, segmentOffset;
  ColorSpace() : ColorSpace(0.00304f, 2.4f, 0.64f, 0.33f, 0.3f, 0.6f, 0.15f, 0.06f, 0.31271f, 0.32902f) {}
  ColorSpace(float bp, float g, float xR, float yR, float xG, float yG, float xB, float yB, float xW, float yW) {
    breakPoint = bp; gammaV = g;
    slope = bp > 0.0f ? 1.0f / (g / (float)std::pow((double)bp, (double)(1.0f / g - 1.0f)) - g * bp + bp) : 1.0f;
    slopeMatch = bp > 0.0f ? g * slope / (float)std::pow((double)bp, (double)(1.0f / g - 1.0f)) : 1.0f;
    segmentOffset = bp > 0.0f ? slopeMatch * (float)std::pow((double)bp, (double)(1.0f / g)) - slope * bp : 0.0f;
    float zR = 1.0f - (xR + yR), zG = 1.0f - (xG + yG), zB = 1.0f - (xB + yB), zW = 1.0f - (xW + yW);
    float rX = (yG * zB) - (yB * zG), rY = (xB * zG) - (xG * zB), rZ = (xG * yB) - (xB * yG);
    float rW = ((rX * xW) + (rY * yW) + (rZ * zW)) / yW;
    float gX = (yB * zR) - (yR * zB), gY = (xR * zB) - (xB * zR), gZ = (xB * yR) - (xR * yB);
    float gW = ((gX * xW) + (gY * yW) + (gZ * zW)) / yW;
    float bX = (yR * zG) - (yG * zR), bY = (xG * zR) - (xR * zG), bZ = (xR * yG) - (xG * yR);
    float bW = ((bX * xW) + (bY * yW) + (bZ * zW)) / yW;
    float m[9] = {rX / rW, rY / rW, rZ / rW, gX / gW, gY / gW, gZ / gW, bX / bW, bY / bW, bZ / bW};
    std::memcpy(xyz2rgb, m, sizeof m);
    float a = m[0] * (m[4] * m[8] - m[7] * m[5]);
    float b = m[1] * (m[3] * m[8] - m[6] * m[5]);
    float c = m[2] * (m[3] * m[7] - m[6] * m[4]);
    float s = 1.0f / (a - b + c);
    float r[9] = {s * (m[4] * m[8] - m[5] * m[7]), s * (m[5] * m[6] - m[3] * m[8]), s * (m[3] * m[7] - m[4] * m[6]),
                  s * (m[2] * m[7] - m[1] * m[8]), s * (m[0] * m[8] - m[2] * m[6]), s * (m[1] * m[6] - m[0] * m[7]),
                  s * (m[1] * m[5] - m[2] * m[4]), s * (m[2] * m[3] - m[0] * m[5]), s * (m[0] * m[4] - m[1] * m[3])};
    std::memcpy(rgb2xyz, r, sizeof r);
  }
  V3 to_rgb(V3 c) const { const float* m = xyz2rgb; return {m[0] * c.x + m[1] * c.y + m[2] * c.z, m[3] * c.x + m[4] * c.y + m[5] * c.z, m[6] * c.x + m[7] * c.y + m[8] * c.z}; }
  V3 to_xyz(V3 c) const { const float* m = rgb2xyz; return {m[0] * c.x + m[3] * c.y + m[6] * c.z, m[1] * c.x + m[4] * c.y + m[7] * c.z, m[2] * c.x + m[5] * c.y + m[8] * c.z}; }
  float redo(float v) const { return v <= breakPoint ? v * slope : slopeMatch * (float)std::pow((double)v, (double)(1.0f / gammaV)) - segmentOffset; }
  float undo(float v) const { return v <= breakPoint * slope ? v * (1.0f / slope) : (float)std::pow((double)((v + segmentOffset) * (1.0f / slopeMatch)), (double)gammaV); }
};
inline const ColorSpace& srgb() { static ColorSpace cs; return cs; }
inline V3 xyz_to_srgb_linear(V3 c) { return srgb().to_rgb(c); }
inline float luminance(V3 c) { return c.x * 0.212671f + c.y * 0.715160f + c.z * 0.072169f; }  // color/Color3F.java:2532

struct LightRef { int id, rel, abs; };
inline LightRef light_ref(const Scene& sc, int index) {
  uint32_t v = (uint32_t)sc.lights[index];
  LightRef r; r.id = (v >> 16) & 0xFFFF; r.rel = v & 0xFFFF;
  switch (r.id) {
    case kLightDiffuseArea: r.abs = r.rel * 40; break;
    case kLightDirectional: r.abs = r.rel * 8; break;
    case kLightPoint: r.abs = r.rel * 8; break;
    case kLightSpot: r.abs = r.rel * 24; break;
    case kLightPerez: r.abs = sc.I("lightPerezLightOffsetArray")[r.rel]; break;
    case kLightImage: r.abs = sc.I("lightImageLightOffsetArray")[r.rel]; break;
    default: r.abs = 0;
  }
  return r;
}
inline bool light_is_delta(int id) { return id == kLightPoint || id == kLightSpot || id == kLightDirectional; }
inline M44 load_m44(const float* q) { M44 m; std::memcpy(m.m, q, sizeof m.m); return m; }

// geometry/shape/Triangle3F.java:sample + geometry/Shape3F.java:123 (the solid-angle
// conversion there keeps dist^2/|cos| and drops the 1/area factor of the area sample).
// geometry/shape/Sphere3F.java:156 for the unit sphere.
inline bool shape_sample(const Scene& sc, int sid, int soff, V3 ref, float u, float v, V3* p, V3* n, float* pdf) {
  if (sid == kShapeTriangle) {
    Tri tr = load_tri(sc.F("shape3FTriangle3FArray"), soff);
    float su = std::sqrt(u);
    float b0 = 1.0f - su, b1 = v * su, b2 = 1.0f - b0 - b1;
    V3 pt = {tr.a.x * b0 + tr.b.x * b1 + tr.c.x * b2, tr.a.y * b0 + tr.b.y * b1 + tr.c.y * b2, tr.a.z * b0 + tr.b.z * b1 + tr.c.z * b2};
    V3 nn = normalize(tr.na * b0 + tr.nb * b1 + tr.nc * b2);
    V3 inc = pt - ref;
    if (dot(inc, inc) == 0.0f) return false;
    V3 incn = normalize(inc);
    float pd = distance_squared(pt, ref) / std::fabs(dot(nn, -incn));
    if (std::isinf(pd) || std::isnan(pd)) return false;
    *p = pt; *n = nn; *pdf = pd; return true;
  }
  if (sid == kShapeSphere) {
    V3 c = {0, 0, 0};
    if (distance_squared(c, ref) <= 1.0f) {
      // Sphere3F.sample(Point2F): uniform over the sphere, pdf 1/area
      float ct = 1.0f - 2.0f * u, st = std::sqrt(std::fmax(0.0f, 1.0f - ct * ct)), phi = v * 2.0f * kPi;
      V3 d = {st * std::cos(phi), st * std::sin(phi), ct};
      V3 pt = d, nn = normalize(d);
      V3 inc = pt - ref;
      if (dot(inc, inc) == 0.0f) return false;
      V3 incn = normalize(inc);
      float pd = distance_squared(pt, ref) / std::fabs(dot(nn, -incn));
      if (std::isinf(pd) || std::isnan(pd)) return false;
      *p = pt; *n = nn; *pdf = pd; return true;
    }
    float dist = distance(c, ref), dr = 1.0f / dist;
    V3 dc = (c - ref) * dr;
    ONB o = onb_from_w(dc);
    V3 x = -o.u, y = -o.v, z = -o.w;
    float stm = 1.0f * dr, stm2 = stm * stm, stmr = 1.0f / stm;
    float ctm = std::sqrt(std::fmax(0.0f, 1.0f - stm2));
    float ct = stm2 < 0.00068523f ? std::sqrt(1.0f - stm2 * u) : (ctm - 1.0f) * u + 1.0f;
    float st2 = stm2 < 0.00068523f ? stm2 * u : 1.0f - ct * ct;
    float ca = st2 * stmr + ct * std::sqrt(std::fmax(0.0f, 1.0f - st2 * stmr * stmr));
    float sa = std::sqrt(std::fmax(0.0f, 1.0f - ca * ca));
    float phi = v * 2.0f * kPi;
    V3 sd = x * (sa * std::cos(phi)) + y * (sa * std::sin(phi)) + z * ca;
    *p = c + sd; *n = normalize(sd); *pdf = 1.0f / (2.0f * kPi * (1.0f - ctm));
    return true;
  }
  return false;  // Shape3F.sample default: no sample
}
inline float shape_area(const Scene& sc, int sid, int soff) {
  if (sid == kShapeTriangle) return triangle_area(load_tri(sc.F("shape3FTriangle3FArray"), soff));
  if (sid == kShapeSphere) return 4.0f * kPi;
  return 0.0f;
}
// Shape3F.evaluateProbabilityDensityFunction (geometry/Shape3F.java:199) and the
// Sphere3F override (geometry/shape/Sphere3F.java:460, which multiplies by the area).
inline float shape_pdf(const Scene& sc, int sid, int soff, V3 ref, V3 wi) {
  Ray r = make_ray(ref, wi);
  Surface s; int tri;
  if (!shape_surface(sc, sid, soff, r, 0.001f, FLT_MAX, &s, &tri)) return 0.0f;
  float area = shape_area(sc, sid, soff);
  float pd;
  if (sid == kShapeSphere) pd = distance_squared(s.p, ref) / std::fabs(dot(s.s.w, -wi)) * area;
  else pd = distance_squared(s.p, ref) / (std::fabs(dot(s.s.w, -wi)) * area);
  if (std::isinf(pd) || std::isnan(pd)) return 0.0f;
  return pd;
}

struct PathCtx { uint32_t key; int bounce; };

// Light.sampleRadianceIncoming
inline bool light_sample(const Scene& sc, const LightRef& lr, const Hit& h, float u, float v, float sun_pick, LightSample* out) {
  V3 p = h.w.p;
  switch (lr.id) {
    case kLightDiffuseArea: {
      const float* q = sc.F("lightDiffuseAreaLightArray").data() + lr.abs;
      M44 o2w = load_m44(q), w2o = load_m44(q + 16);
      V3 Le = {q[32], q[33], q[34]};
      int sid = (int)q[35], soff = (int)q[36];
      bool two = q[38] != 0.0f;
      V3 ref = transform_point_divide(w2o, p);
      V3 sp, sn; float pdf;
      if (!shape_sample(sc, sid, soff, ref, u, v, &sp, &sn, &pdf)) return false;
      V3 pw = transform_point_divide(o2w, sp);
      V3 nw = normalize(transform_vector_transpose(w2o, sn));
      V3 wi = normalize(pw - p);
      if (pdf > 0.0f && (two || dot(nw, -wi) > 0.0f)) { *out = LightSample{Le, pw, wi, pdf}; return true; }
      return false;
    }
    case kLightPoint: {
      const float* q = sc.F("lightPointLightArray").data() + lr.abs;
      V3 I = {q[0], q[1], q[2]}, pos = {q[3], q[4], q[5]};
      *out = LightSample{I * (1.0f / distance_squared(p, pos)), pos, normalize(pos - p), 1.0f};
      return true;
    }
    case kLightSpot: {
      const float* q = sc.F("lightSpotLightArray").data() + lr.abs;
      M44 w2o = load_m44(q);
      V3 I = {q[16], q[17], q[18]}, pos = {q[19], q[20], q[21]};
      float cc = q[22], cd = q[23];
      V3 wi = normalize(pos - p);
      V3 dobj = normalize(transform_vector(w2o, -wi));
      float ct = dobj.z, fall;
      if (ct < cc) fall = 0.0f; else if (ct >= cd) fall = 1.0f; else { float d = (ct - cc) / (cd - cc); fall = (d * d) * (d * d); }
      *out = LightSample{I * fall * (1.0f / distance_squared(p, pos)), pos, wi, 1.0f};
      return true;
    }
    case kLightDirectional: {
      const float* q = sc.F("lightDirectionalLightArray").data() + lr.abs;
      V3 L = {q[0], q[1], q[2]}, d = {q[3], q[4], q[5]};
      float rad = q[6];
      *out = LightSample{L, p + d * (2.0f * rad), d, 1.0f};
      return true;
    }
    case kLightPerez: {
      const float* q = sc.F("lightPerezLightArray").data() + lr.abs;
      M44 o2w = load_m44(q);
      V3 sunW = {q[38], q[39], q[40]}, sunO = {q[35], q[36], q[37]};
      float radius = q[45];
      const float* dist = q;  // distribution starts at +48
      bool sun = dot(sunW, h.w.g.w) > sun_pick && dot(sunW, h.w.s.w) > sun_pick;
      if (sun) {
        float st = sin_t(sunO);
        if (st != 0.0f) {
          float phi = std::atan2(sunO.y, sunO.x); if (phi < 0.0f) phi += 2.0f * kPi;
          float su = phi * (1.0f / (2.0f * kPi)), sv = std::acos(saturate(sunO.z, -1.0f, 1.0f)) * (1.0f / kPi);
          float pdf = dist2_pdf_remapped(dist, 48, su, sv) / (2.0f * kPi * kPi * st);
          if (pdf != 0.0f) { *out = LightSample{V3{q[32], q[33], q[34]}, p + sunW * (2.0f * radius), sunW, pdf}; return true; }
        }
      }
      float ru, rv;
      dist2_remap(dist, 48, u, v, &ru, &rv);
      float pr = dist2_pdf_remapped(dist, 48, ru, rv);
      if (pr == 0.0f) return false;
      float phi = ru * 2.0f * kPi, th = rv * kPi;
      V3 dobj = {std::sin(th) * std::cos(phi), std::sin(th) * std::sin(phi), std::cos(th)};
      V3 dw = normalize(transform_vector(o2w, dobj));
      float st = sin_t(dobj);
      if (st == 0.0f) return false;
      V3 L = sat0(perez_sky(q, dobj));
      *out = LightSample{L, p + dw * (2.0f * radius), dw, pr / (2.0f * kPi * kPi * st)};
      return true;
    }
    case kLightImage: {  // scene/light/ImageLight.java:207 sampleRadianceIncoming
      const float* q = sc.F("lightImageLightArray").data() + lr.abs;
      float ru, rv;
      dist2_remap(q, 40, u, v, &ru, &rv);
      const float pr = dist2_pdf_remapped(q, 40, ru, rv);
      if (pr == 0.0f) return false;
      const float phi = ru * 2.0f * kPi, th = rv * kPi;
      const V3 dobj = {std::sin(th) * std::cos(phi), std::sin(th) * std::sin(phi), std::cos(th)};
      const V3 dw = normalize(transform_vector(load_m44(q), dobj));
      const float st = sin_t(dobj);
      if (st == 0.0f) return false;
      *out = LightSample{image_sky(q, dobj), p + dw * (2.0f * q[35]), dw, pr / (2.0f * kPi * kPi * st)};
      return true;
    }
  }
  return false;
}

// Light.evaluateProbabilityDensityFunctionRadianceIncoming
inline float light_pdf(const Scene& sc, const LightRef& lr, const Hit& h, V3 wi) {
  if (lr.id == kLightDiffuseArea) {
    const float* q = sc.F("lightDiffuseAreaLightArray").data() + lr.abs;
    M44 w2o = load_m44(q + 16);
    V3 wo = normalize(transform_vector(w2o, wi));
    V3 ref = transform_point_divide(w2o, h.w.p);
    return shape_pdf(sc, (int)q[35], (int)q[36], ref, wo);
  }
  if (lr.id == kLightPerez) {
    const float* q = sc.F("lightPerezLightArray").data() + lr.abs;
    M44 w2o = load_m44(q + 16);
    V3 d = normalize(transform_vector(w2o, wi));
    float st = std::sin(std::acos(saturate(d.z, -1.0f, 1.0f)));
    if (st == 0.0f) return 0.0f;
    float phi = std::atan2(d.y, d.x); if (phi < 0.0f) phi += 2.0f * kPi;
    float su = phi * (1.0f / (2.0f * kPi)), sv = std::acos(saturate(d.z, -1.0f, 1.0f)) * (1.0f / kPi);
    return dist2_pdf_remapped(q, 48, su, sv) / (2.0f * kPi * kPi * st);
  }
  if (lr.id == kLightImage) {  // ImageLight.java:348
    const float* q = sc.F("lightImageLightArray").data() + lr.abs;
    const V3 d = normalize(transform_vector(load_m44(q + 16), wi));
    const float st = std::sin(std::acos(saturate(d.z, -1.0f, 1.0f)));
    if (st == 0.0f) return 0.0f;
    float phi = std::atan2(d.y, d.x); if (phi < 0.0f) phi += 2.0f * kPi;
    const float su = phi * (1.0f / (2.0f * kPi)), sv = std::acos(saturate(d.z, -1.0f, 1.0f)) * (1.0f / kPi);
    return dist2_pdf_remapped(q, 40, su, sv) / (2.0f * kPi * kPi * st);
  }
  return 0.0f;
}

// Light.evaluateRadianceEmitted(Ray3F): only the Perez and image lights emit along a missed ray.
inline V3 light_Le_ray(const Scene& sc, const LightRef& lr, const Ray& r) {
  if (lr.id == kLightPerez) {
    const float* q = sc.F("lightPerezLightArray").data() + lr.abs;
    M44 w2o = load_m44(q + 16);
    V3 d = normalize(transform_vector(w2o, r.d));
    return sat0(perez_sky(q, d));
  }
  if (lr.id == kLightImage) {  // ImageLight.java:165
    const float* q = sc.F("lightImageLightArray").data() + lr.abs;
    return image_sky(q, normalize(transform_vector(load_m44(q + 16), r.d)));
  }
  return {0, 0, 0};
}

// Intersection.evaluateRadianceEmitted(direction)
inline V3 hit_Le(const Scene& sc, const Hit& h, V3 dir) {
  const int32_t* P = sc.prims.data() + h.prim * 8;
  uint32_t al = (uint32_t)P[1];
  if (al != 0) {
    int id = (al >> 16) & 0xFFFF, rel = al & 0xFFFF;
    if (id == kLightDiffuseArea) {
      const float* q = sc.F("lightDiffuseAreaLightArray").data() + rel * 40;
      bool two = q[38] != 0.0f;
      return (two || dot(h.w.s.w, dir) > 0.0f) ? V3{q[32], q[33], q[34]} : V3{0, 0, 0};
    }
  }
  return material_emission(sc, h, P[4], P[5]);
}
inline bool hit_is_light(const Scene& sc, const Hit& h, const LightRef& lr) {
  uint32_t al = (uint32_t)sc.prims[h.prim * 8 + 1];
  return al != 0 && (int)((al >> 16) & 0xFFFF) == lr.id && (int)(al & 0xFFFF) == lr.rel;
}

// scene/Scene.java:1066 checkLightVisibility
inline bool visible(const Scene& sc, const Hit& h, const LightRef& lr, const LightSample& ls, RayStats* st) {
  Ray r = make_ray(h.w.p, ls.p - h.w.p);
  float tmax = std::fabs(distance(h.w.p, ls.p)) + 0.001f;
  if (lr.id == kLightDiffuseArea) {
    Hit hh;
    if (scene_intersect(sc, r, 0.001f, tmax, &hh, st)) return hit_is_light(sc, hh, lr);
    return false;
  }
  return !scene_intersect(sc, r, 0.001f, tmax, nullptr, st);
}

inline float power_heuristic(float a, float b) { return (a * a) / (a * a + b * b); }

// scene/Scene.java:1530 doEstimateDirectLight (isSpecular = false)
inline V3 estimate_direct(const Scene& sc, const Bsdf& B, const Hit& h, const LightRef& lr, float ua, float va, float ub, float vb, float sun_pick, RayStats* st) {
  V3 Ld = {0, 0, 0};
  const int flags = kAllButSpecular;
  LightSample ls;
  bool have = light_sample(sc, lr, h, ua, va, sun_pick, &ls);
  V3 n = h.w.s.w;
  if (light_is_delta(lr.id)) {
    if (have && !black(ls.L) && ls.pdf > 0.0f) {
      V3 f = bsdf_f(B, flags, ls.wi) * std::fabs(dot(ls.wi, n));
      if (!black(f) && visible(sc, h, lr, ls, st)) Ld = Ld + mul(f, ls.L) * (1.0f / ls.pdf);
    }
    return Ld;
  }
  if (have && !black(ls.L) && ls.pdf > 0.0f) {
    V3 f = bsdf_f(B, flags, ls.wi) * std::fabs(dot(ls.wi, n));
    float sp = bsdf_pdf(B, flags, ls.wi);
    if (!black(f) && visible(sc, h, lr, ls, st)) {
      float w = power_heuristic(ls.pdf, sp);
      Ld = Ld + mul(f, ls.L) * w * (1.0f / ls.pdf);
    }
  }
  BsdfSample bs;
  if (bsdf_sample(B, flags, ub, vb, &bs)) {
    V3 f = bs.f * std::fabs(dot(bs.wi, n));
    bool spec = is_spec(bs.type);
    if (!black(f) && bs.pdf > 0.0f) {
      float w = 1.0f;
      if (!spec) {
        float lp = light_pdf(sc, lr, h, bs.wi);
        if (lp == 0.0f) return Ld;
        w = power_heuristic(bs.pdf, lp);
      }
      Ray r = make_ray(h.w.p, bs.wi);
      Hit hl;
      if (scene_intersect(sc, r, 0.001f, FLT_MAX, &hl, st)) {
        if (hit_is_light(sc, hl, lr)) {
          V3 Li = hit_Le(sc, hl, -bs.wi);
          if (!black(Li)) Ld = Ld + mul(f, Li) * w * (1.0f / bs.pdf);
        }
      } else {
        V3 Li = light_Le_ray(sc, lr, r);
        if (!black(Li)) Ld = Ld + mul(f, Li) * w * (1.0f / bs.pdf);
      }
    }
  }
  return Ld;
}

struct Params {
  int algo, width, height, spp, sample_base, max_bounce, min_rr, ao_samples;
  float ao_distance;
  int preview;
  uint32_t seed;
  int row_begin, row_end;
  int row_step;  // render rows row_begin, row_begin + row_step, ... below row_end (0 or 1: every row)
};

// scene/Scene.java:451 radiancePathTracer
// scene/Scene.java:786 doRadianceRayTracer (Whitted): at each hit, emission,
// every light sampled once (Light.sampleRadianceIncoming, checkLightVisibility),
// then, below the bounce limit, the specular reflection and the specular
// transmission samples of the BSDF (built with isAllowingMultipleLobes = false)
// traced recursively; a material without a BSDF passes the ray through.
// Random numbers: node n of a sample's tree (root 0; reflection, transmission
// and pass-through children 3n+1, 3n+2, 3n+3) has key rng_path_key(key, n, kRtSalt);
// dims 0-1 reflection, 2-3 transmission, 4 the material draw, 8+3k.. light k.
// A tree is cut after kRtMaxNodes nodes (counted in *overflow).
constexpr uint32_t kRtSalt = 0x52545243u;
constexpr int kRtMaxNodes = 4096;
struct RtCtx { uint32_t key; int nodes; bool overflow; };
inline V3 rt_node(const Scene& sc, Ray ray, const Params& P, RtCtx& C, uint32_t nid, int bounce, RayStats* st, bool* unsupported) {
  if (++C.nodes > kRtMaxNodes) { C.overflow = true; return {0, 0, 0}; }
  const uint32_t nk = rng_path_key(C.key, nid, kRtSalt);
  Hit h;
  if (!scene_intersect(sc, ray, kTMinimum, kTMaximum, &h, st)) {
    V3 L = {0, 0, 0};
    for (int k = 0; k < (int)sc.lights.size(); ++k) L = L + light_Le_ray(sc, light_ref(sc, k), ray);
    return L;
  }
  const int32_t* pr = sc.prims.data() + h.prim * 8;
  Bsdf B; bool sup;
  if (!build_bsdf(sc, pr[4], pr[5], h, false, rng_uniform(nk, 4), &B, &sup)) {
    if (!sup) *unsupported = true;
    return rt_node(sc, make_ray(h.w.p, ray.d), P, C, nid * 3u + 3u, bounce, st, unsupported);
  }
  const V3 n = h.w.s.w, wo = -ray.d;
  V3 L = hit_Le(sc, h, wo);
  for (int k = 0; k < (int)sc.lights.size(); ++k) {
    const LightRef lr = light_ref(sc, k);
    LightSample ls;
    if (!light_sample(sc, lr, h, rng_uniform(nk, 8 + 3 * k), rng_uniform(nk, 9 + 3 * k), rng_uniform(nk, 10 + 3 * k), &ls)) continue;
    if (black(ls.L) || !(ls.pdf > 0.0f)) continue;
    const V3 f = bsdf_f(B, kAll, ls.wi);
    if (!black(f) && visible(sc, h, lr, ls, st)) L = L + mul(f, ls.L) * std::fabs(dot(ls.wi, n)) * (1.0f / ls.pdf);
  }
  if (bounce + 1 < P.max_bounce) {
    const int flags[2] = {kSpecular | kRefl, kSpecular | kTrans};
    for (int b = 0; b < 2; ++b) {  // doComputeSpecularReflection, doComputeSpecularTransmission
      BsdfSample bs;
      if (!bsdf_sample(B, flags[b], rng_uniform(nk, 2 * b), rng_uniform(nk, 2 * b + 1), &bs)) continue;
      const float c = std::fabs(dot(bs.wi, n));
      if (black(bs.f) || !(bs.pdf > 0.0f) || !(c > 0.0f)) continue;
      const V3 Li = rt_node(sc, make_ray(h.w.p, bs.wi), P, C, nid * 3u + 1u + (uint32_t)b, bounce + 1, st, unsupported);
      L = L + mul(bs.f, Li) * c * (1.0f / bs.pdf);
    }
  }
  return L;
}

inline V3 radiance_path(const Scene& sc, Ray ray, const Params& P, uint32_t key, RayStats* st, bool* unsupported) {
  const int nl = (int)sc.lights.size();
  V3 L = {0, 0, 0}, beta = {1, 1, 1};
  bool specb = false;
  float etaScale = 1.0f;
  int dimb = 0;  // bounce index used for random dimensions (advances on every loop iteration)
  for (int bounce = 0;; ++bounce, ++dimb) {
    Hit h;
    if (dimb > 4096) break;
    if (scene_intersect(sc, ray, kTMinimum, kTMaximum, &h, st)) {
      V3 wo = -ray.d;
      if (bounce == 0 || specb) L = L + mul(beta, hit_Le(sc, h, wo));
      if (bounce >= P.max_bounce) break;
      const int32_t* pr = sc.prims.data() + h.prim * 8;
      Bsdf B; bool sup;
      if (!build_bsdf(sc, pr[4], pr[5], h, true, rng_uniform(key, bounce_dim(dimb, kDimMaterial)), &B, &sup)) {
        if (!sup) *unsupported = true;
        ray = make_ray(h.w.p, ray.d);
        --bounce;
        continue;
      }
      if (bsdf_count_nonspecular(B) > 0 && nl > 0) {
        float up = rng_uniform(key, bounce_dim(dimb, kDimLightPick));
        int li = std::min((int)(up * nl), nl - 1);
        LightRef lr = light_ref(sc, li);
        V3 Ld = estimate_direct(sc, B, h, lr, rng_uniform(key, bounce_dim(dimb, kDimLightSampleU)), rng_uniform(key, bounce_dim(dimb, kDimLightSampleV)),
                                rng_uniform(key, bounce_dim(dimb, kDimMisSampleU)), rng_uniform(key, bounce_dim(dimb, kDimMisSampleV)),
                                rng_uniform(key, bounce_dim(dimb, kDimSunPick)), st);
        L = L + mul(beta, Ld * (1.0f / (1.0f / nl)));
      }
      BsdfSample bs;
      if (!bsdf_sample(B, kAll, rng_uniform(key, bounce_dim(dimb, kDimBsdfU)), rng_uniform(key, bounce_dim(dimb, kDimBsdfV)), &bs)) break;
      if (black(bs.f) || bs.pdf == 0.0f) break;
      beta = mul(beta, bs.f * std::fabs(dot(bs.wi, h.w.s.w)) * (1.0f / bs.pdf));
      specb = is_spec(bs.type);
      if ((bs.type & kTrans) && is_spec(bs.type)) etaScale *= dot(wo, h.w.g.w) > 0.0f ? B.eta * B.eta : 1.0f / (B.eta * B.eta);
      ray = make_ray(h.w.p, bs.wi);
      V3 rr = beta * etaScale;
      float mx = std::fmax(rr.x, std::fmax(rr.y, rr.z));
      if (mx < 1.0f && bounce >= P.min_rr) {
        float q = std::fmax(0.05f, 1.0f - mx);
        if (rng_uniform(key, bounce_dim(dimb, kDimRoulette)) < q) break;
        beta = beta * (1.0f / (1.0f - q));
      }
    } else if (bounce == 0 && P.preview) {
      L = {1, 1, 1}; break;
    } else if (bounce == 0 || specb) {
      for (int k = 0; k < nl; ++k) L = L + mul(beta, light_Le_ray(sc, light_ref(sc, k), ray));
      break;
    } else {
      break;
    }
  }
  return L;
}

// scene/Scene.java:675 radianceRayCaster
inline V3 radiance_raycast(const Scene& sc, const Ray& ray, const Params& P, RayStats* st, Hit* hout) {
  Hit h;
  if (scene_intersect(sc, ray, kTMinimum, kTMaximum, &h, st)) {
    *hout = h;
    float c = std::fabs(dot(h.w.s.w, ray.d));
    return V3{0.5f, 0.5f, 0.5f} * c;
  }
  if (P.preview) return {1, 1, 1};
  V3 L = {0, 0, 0};
  for (int k = 0; k < (int)sc.lights.size(); ++k) L = L + light_Le_ray(sc, light_ref(sc, k), ray);
  return L;
}

// scene/Scene.java:327 radianceDepthCamera
inline V3 radiance_depth(const Scene& sc, const Ray& ray, const Params& P, RayStats* st, Hit* hout) {
  Hit h;
  if (scene_intersect(sc, ray, kTMinimum, kTMaximum, &h, st)) {
    *hout = h;
    float d2 = distance_squared(h.w.ray.o, h.w.p);
    float in = 1.0f / (d2 * 0.5f);
    in = std::fmin(std::fmax(in, 0.0f), 1.0f);
    return {in, in, in};
  }
  return P.preview ? V3{1, 1, 1} : V3{0, 0, 0};
}

// scene/Scene.java:272 radianceAmbientOcclusion (geometric basis)
inline V3 radiance_ao(const Scene& sc, const Ray& ray, const Params& P, uint32_t key, RayStats* st, Hit* hout) {
  Hit h;
  if (!scene_intersect(sc, ray, kTMinimum, kTMaximum, &h, st)) return P.preview ? V3{1, 1, 1} : V3{0, 0, 0};
  *hout = h;
  float acc = 0.0f;
  for (int s = 0; s < P.ao_samples; ++s) {
    V3 d = uniform_hemisphere(rng_uniform(key, kDimBounceBase + 2 * s), rng_uniform(key, kDimBounceBase + 2 * s + 1));
    V3 dw = normalize(to_world(d, h.w.g));
    Ray r = make_ray(h.w.p, dw);
    if (P.ao_distance > 0.0f) {
      Hit hs;
      if (scene_intersect(sc, r, kTMinimum, kTMaximum, &hs, st)) {
        float t = hs.w.t;
        float sat = std::fmin(std::fmax(t, 0.0f), P.ao_distance);
        acc += (sat - 0.0f) / (P.ao_distance - 0.0f);
      } else {
        acc += 1.0f;
      }
    } else if (!scene_intersect(sc, r, kTMinimum, kTMaximum, nullptr, st)) {
      acc += 1.0f;
    }
  }
  float v = acc * (kPi / P.ao_samples);
  v = v / kPi;
  return {v, v, v};
}

// scene/Camera.java:243 createPrimaryRay (pinhole/thin lens, rectilinear and fisheye)
inline bool primary_ray(const float* c, float ix, float iy, float px, float py, float lu, float lv, Ray* out) {
  float fx = c[0], fy = c[1];
  int lens = (int)c[2];
  V3 U = {c[3], c[4], c[5]}, Vv = {c[6], c[7], c[8]}, W = {c[9], c[10], c[11]}, eye = {c[12], c[13], c[14]};
  float ap = c[15], fd = c[16], rx = c[17], ry = c[18];
  float cx = 2.0f * ((ix + px) / (rx - 1.0f)) - 1.0f;
  float cy = 2.0f * ((iy + py) / (ry - 1.0f)) - 1.0f;
  float wf = 1.0f;
  if (lens == 0) {  // Lens.FISHEYE
    float dp = cx * cx + cy * cy;
    if (dp > 1.0f) return false;
    wf = std::sqrt(1.0f - dp);
  }
  float dx, dy;
  concentric(lu, lv, &dx, &dy);
  V3 pp = (U * (fx * cx) + Vv * (fy * cy)) + (eye + W * wf);
  V3 pip = eye + normalize(pp - eye) * fd;
  V3 o = ap > 0.00001f ? eye + (U * (dx * ap) + Vv * (dy * ap)) : eye;
  *out = make_ray(o, normalize(pip - o));
  return true;
}

}  // namespace dfo

using namespace dfo;

extern "C" {

void* dfo_scene_new(void) { return new Scene(); }
void dfo_set_no_drift(int v) { g_no_drift = v; }
void dfo_scene_free(void* s) { delete (Scene*)s; }

int dfo_scene_put(void* s, const char* name, const void* data, long long count, int is_int) {
  Scene* sc = (Scene*)s;
  if (!sc || !name || count < 0 || (count > 0 && !data)) return -1;
  if (is_int) sc->i[name].assign((const int32_t*)data, (const int32_t*)data + count);
  else sc->f[name].assign((const float*)data, (const float*)data + count);
  return 0;
}

int dfo_scene_commit(void* s, int layout) {
  Scene* sc = (Scene*)s;
  if (layout != 1 && layout != 2) return -1;
  sc->layout = layout;
  sc->prims = sc->I("primitiveArray");
  const auto& mats = sc->F("primitiveMatrix44FArray");
  sc->prim_count = (int)(sc->prims.size() / 8);
  if ((int)mats.size() < sc->prim_count * 32) return -2;
  sc->o2w.resize(sc->prim_count); sc->w2o.resize(sc->prim_count);
  for (int p = 0; p < sc->prim_count; ++p) { sc->o2w[p] = load_m44(mats.data() + p * 32); sc->w2o[p] = load_m44(mats.data() + p * 32 + 16); }
  // record-sized shapes: the offset must leave a whole record in its array
  struct { int id; const char* arr; size_t len; } recs[] = {
      {kShapeDisk, "shape3FDisk3FArray", 4}, {kShapeCylinder, "shape3FCylinder3FArray", 4}, {kShapeCone, "shape3FCone3FArray", 4},
      {kShapeParaboloid, "shape3FParaboloid3FArray", 4}, {kShapeHyperboloid, "shape3FHyperboloid3FArray", 12},
      {kShapeCuboid, "shape3FRectangularCuboid3FArray", 6}, {kShapeTorus, "shape3FTorus3FArray", 2},
      {kShapeRectangle, "shape3FRectangle3FArray", 12}, {kShapeTriangle, "shape3FTriangle3FArray", 24}};
  for (int p = 0; p < sc->prim_count; ++p) {
    const int sid = sc->prims[p * 8 + 6], soff = sc->prims[p * 8 + 7];
    for (const auto& rc : recs)
      if (rc.id == sid && (soff < 0 || (size_t)soff + rc.len > sc->F(rc.arr).size())) return -4;
    if (sid == kShapePolygon) {  // variable length: 13 + 2 * count floats
      const auto& A = sc->F("shape3FPolygon3FArray");
      if (soff < 0 || (size_t)soff + 13 > A.size()) return -4;
      const float cnt = A[soff + 12];
      if (!(cnt >= 3.0f) || (size_t)soff + 13 + 2 * (size_t)cnt > A.size()) return -4;
    }
  }
  sc->lights = sc->I("lightIDAndOffsetArray");
  const auto& cam = sc->F("cameraArray");
  if (cam.size() < 19) return -3;
  std::memcpy(sc->cam, cam.data(), sizeof sc->cam);
  return 0;
}

typedef struct dfo_params {
  int algo, width, height, spp, sample_base, max_bounce, min_rr, ao_samples;
  float ao_distance;
  int preview;
  unsigned int seed;
  int row_begin, row_end;
  int row_step;
} dfo_params;

// Renders rows row_begin, row_begin + row_step, ... below row_end (every row
// of [row_begin, row_end) when row_step <= 1) with spp samples per pixel (samples
// sample_base .. sample_base + spp - 1).  Outputs (any may be NULL), each
// W*H entries, only the rendered rows written:
//   sum_rgb   sum of the accepted samples (AbstractCPURenderer.java:231 guard)
//   sumsq_rgb sum of squares of the accepted samples
//   count     accepted samples
//   hit_prim  primitive index of the first sample's primary hit (-1 miss)
//   hit_t     world-space t of the first sample's primary hit
// Returns the number of rays traced, or a negative error.
// One camera sample of pixel (x, y): AbstractCPURenderer.java:215-236 up to
// the radiance (CPURenderer.java:20-37 dispatch).  Returns false when the
// camera gives no ray.  *fx, *fy receive the film position x + jitter.
static bool render_sample(const Scene& sc, const Params& P, int x, int y, int k, bool want_hit, V3* c, Hit* h, RayStats* st, bool* unsup,
                          bool* rt_over, float* fx, float* fy) {
  const size_t pix = (size_t)y * P.width + x;
  uint32_t key = rng_path_key(P.seed, (uint32_t)pix, (uint32_t)(P.sample_base + k));
  float jx = rng_uniform(key, kDimPixelX), jy = rng_uniform(key, kDimPixelY);
  if (fx) *fx = (float)x + jx;
  if (fy) *fy = (float)y + jy;
  Ray r;
  if (!primary_ray(sc.cam, (float)x, (float)y, jx, jy, rng_uniform(key, kDimLensU), rng_uniform(key, kDimLensV), &r)) return false;
  switch (P.algo) {
    case kAlgoAO: *c = radiance_ao(sc, r, P, key, st, h); break;
    case kAlgoDepth: *c = radiance_depth(sc, r, P, st, h); break;
    case kAlgoRayCast: *c = radiance_raycast(sc, r, P, st, h); break;
    case kAlgoRayTrace: {
      RtCtx C{key, 0, false};
      *c = rt_node(sc, r, P, C, 0u, 0, st, unsup);
      if (C.overflow) *rt_over = true;
      if (want_hit) { RayStats dummy; scene_intersect(sc, r, kTMinimum, kTMaximum, h, &dummy); }
      break;
    }
    case kAlgoPath: default: {
      *c = radiance_path(sc, r, P, key, st, unsup);
      if (want_hit) { RayStats dummy; scene_intersect(sc, r, kTMinimum, kTMaximum, h, &dummy); }
      break;
    }
  }
  return true;
}

float dfo_gaussian_filter(float x, float y, float rx, float ry, float falloff);

// The CPU renderer's film (image/PixelImageF.java:569 filmAddColorXYZ with
// GaussianFilter2F(2, 2, 2), the 16x16 table of filter/Filter2F.java:119):
// every accepted sample converted to XYZ and added, filter-weighted, to the
// pixels within the filter radius of its film position.  out: per pixel X, Y,
// Z sums and the weight sum.  Samples are computed in parallel, then splatted
// in row, column, sample order.
long long dfo_render_pixel_film(void* s, const dfo_params* pp, float* xyzw, int threads) {
  Scene* sc = (Scene*)s;
  Params P;
  std::memcpy(&P, pp, sizeof P);
  if (P.width <= 0 || P.height <= 0 || P.spp < 0) return -1;
  const int W = P.width, H = P.height, S = P.spp;
  struct Smp { float fx, fy; V3 xyz; bool ok; };
  std::vector<Smp> smp((size_t)W * H * S);
  if (threads < 1) threads = 1;
  std::atomic<int> next_row(0);
  std::atomic<long long> rays(0);
  std::atomic<int> bad(0);
  auto work = [&]() {
    RayStats st;
    bool unsup = false, over = false;
    for (;;) {
      const int y = next_row.fetch_add(1);
      if (y >= H) break;
      for (int x = 0; x < W; ++x)
        for (int k = 0; k < S; ++k) {
          Smp& m = smp[((size_t)y * W + x) * S + k];
          Hit h;
          V3 c;
          m.ok = render_sample(*sc, P, x, y, k, false, &c, &h, &st, &unsup, &over, &m.fx, &m.fy) &&
                 std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z) && luminance(c) >= -1.0e-5f;
          if (m.ok) m.xyz = srgb().to_xyz(c);  // AbstractCPURenderer.java:231-233
        }
    }
    rays += st.rays;
    if (unsup || over) bad = 1;
  };
  std::vector<std::thread> pool;
  for (int i = 0; i < threads; ++i) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  if (bad.load()) return -2;
  float table[16 * 16];
  for (int ty = 0; ty < 16; ++ty)
    for (int tx = 0; tx < 16; ++tx)
      table[ty * 16 + tx] = dfo_gaussian_filter((tx + 0.5f) * 2.0f * (1.0f / 16.0f), (ty + 0.5f) * 2.0f * (1.0f / 16.0f), 2.0f, 2.0f, 2.0f);
  std::memset(xyzw, 0, sizeof(float) * 4 * (size_t)W * H);
  for (const Smp& m : smp) {
    if (!m.ok) continue;
    const float dx = m.fx - 0.5f, dy = m.fy - 0.5f;
    const int x0 = (int)std::fmax(std::ceil(dx - 2.0f), 0.0f), x1 = (int)std::fmin(std::floor(dx + 2.0f), (float)(W - 1));
    const int y0 = (int)std::fmax(std::ceil(dy - 2.0f), 0.0f), y1 = (int)std::fmin(std::floor(dy + 2.0f), (float)(H - 1));
    for (int fy = y0; fy <= y1; ++fy) {
      const int oy = std::min((int)std::floor(std::fabs((fy - dy) * 0.5f * 16.0f)), 15);
      for (int fx = x0; fx <= x1; ++fx) {
        const int ox = std::min((int)std::floor(std::fabs((fx - dx) * 0.5f * 16.0f)), 15);
        const float w = table[oy * 16 + ox];
        float* q = xyzw + ((size_t)fy * W + fx) * 4;
        q[0] += m.xyz.x * w; q[1] += m.xyz.y * w; q[2] += m.xyz.z * w; q[3] += w;  // PixelF.addColorXYZ, sample weight 1
      }
    }
  }
  return rays.load();
}

long long dfo_render(void* s, const dfo_params* pp, float* sum_rgb, float* sumsq_rgb, int* count, int* hit_prim, float* hit_t, int threads) {
  Scene* sc = (Scene*)s;
  Params P;
  std::memcpy(&P, pp, sizeof P);
  if (P.width <= 0 || P.height <= 0 || P.spp < 0) return -1;
  int rb = std::max(0, P.row_begin), re = std::min(P.height, P.row_end <= 0 ? P.height : P.row_end);
  const int step = std::max(1, P.row_step);
  if (threads < 1) threads = 1;
  std::atomic<int> next_row(0);
  std::atomic<long long> rays(0);
  std::atomic<int> unsupported(0);
  std::atomic<int> rt_overflow(0);
  auto work = [&]() {
    RayStats st;
    bool unsup = false;
    for (;;) {
      const int y = rb + next_row.fetch_add(1) * step;
      if (y >= re) break;
      for (int x = 0; x < P.width; ++x) {
        const size_t pix = (size_t)y * P.width + x;
        V3 acc = {0, 0, 0}, acc2 = {0, 0, 0};
        int n = 0;
        for (int k = 0; k < P.spp; ++k) {
          Hit h;
          V3 c;
          bool over = false;
          if (!render_sample(*sc, P, x, y, k, k == 0 && (hit_prim || hit_t), &c, &h, &st, &unsup, &over, nullptr, nullptr)) {
            if (k == 0) { if (hit_prim) hit_prim[pix] = -1; if (hit_t) hit_t[pix] = NAN; }
            continue;
          }
          if (over) rt_overflow = 1;
          if (k == 0) {
            if (hit_prim) hit_prim[pix] = h.prim;
            if (hit_t) hit_t[pix] = h.prim >= 0 ? h.w.t : NAN;
          }
          bool finite = std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z);
          if (finite && luminance(c) >= -1.0e-5f) { acc = acc + c; acc2 = acc2 + mul(c, c); ++n; }
        }
        if (sum_rgb) { sum_rgb[pix * 3] = acc.x; sum_rgb[pix * 3 + 1] = acc.y; sum_rgb[pix * 3 + 2] = acc.z; }
        if (sumsq_rgb) { sumsq_rgb[pix * 3] = acc2.x; sumsq_rgb[pix * 3 + 1] = acc2.y; sumsq_rgb[pix * 3 + 2] = acc2.z; }
        if (count) count[pix] = n;
      }
    }
    rays += st.rays;
    if (unsup) unsupported = 1;
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  if (unsupported.load()) return -2;
  if (rt_overflow.load()) return -5;  // a RAY_TRACING tree exceeded kRtMaxNodes
  return rays.load();
}

// ---- primitive math exported for the golden-vector tests -------------------
// out: t, point xyz, G.w xyz, G.v xyz, G.u xyz, S.w xyz, uv -> 18 floats
static void put_surface(const Surface& s, float* out) {
  float v[18] = {s.t, s.p.x, s.p.y, s.p.z, s.g.w.x, s.g.w.y, s.g.w.z, s.g.v.x, s.g.v.y, s.g.v.z, s.g.u.x, s.g.u.y, s.g.u.z, s.s.w.x, s.s.w.y, s.s.w.z, s.tu, s.tv};
  std::memcpy(out, v, sizeof v);
}
int dfo_plane_intersection(const float* o, const float* d, float tmin, float tmax, float* out) {
  Ray r = make_ray(V3{o[0], o[1], o[2]}, V3{d[0], d[1], d[2]});
  float t = plane_t(r, tmin, tmax);
  if (std::isnan(t)) return 0;
  put_surface(plane_surface(r, t), out);
  return 1;
}
float dfo_sphere_intersection_t(const float* o, const float* d, float tmin, float tmax) {
  Ray r = make_ray(V3{o[0], o[1], o[2]}, V3{d[0], d[1], d[2]});
  SphereHit h;
  return sphere_hit(r, tmin, tmax, &h) ? h.t : NAN;
}
int dfo_sphere_intersection(const float* o, const float* d, float tmin, float tmax, float* out) {
  Ray r = make_ray(V3{o[0], o[1], o[2]}, V3{d[0], d[1], d[2]});
  SphereHit h;
  if (!sphere_hit(r, tmin, tmax, &h)) return 0;
  put_surface(sphere_surface(r, h), out);
  return 1;
}
float dfo_triangle_intersection_t(const float* tri24, const float* o, const float* d, float tmin, float tmax) {
  std::vector<float> T(tri24, tri24 + 24);
  return triangle_t(load_tri(T, 0), make_ray(V3{o[0], o[1], o[2]}, V3{d[0], d[1], d[2]}), tmin, tmax);
}
int dfo_aabb_intersection(const float* bb8, const float* o, const float* d, float tmin, float tmax, float* t_out) {
  Ray r = make_ray(V3{o[0], o[1], o[2]}, V3{d[0], d[1], d[2]});
  V3 mx = {bb8[0], bb8[1], bb8[2]}, mn = {bb8[3], bb8[4], bb8[5]};
  V3 rc = {1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z};
  V3 a = {(mx.x - r.o.x) * rc.x, (mx.y - r.o.y) * rc.y, (mx.z - r.o.z) * rc.z};
  V3 b = {(mn.x - r.o.x) * rc.x, (mn.y - r.o.y) * rc.y, (mn.z - r.o.z) * rc.z};
  float t0 = std::fmax(std::fmax(std::fmin(a.x, b.x), std::fmin(a.y, b.y)), std::fmin(a.z, b.z));
  float t1 = std::fmin(std::fmin(std::fmax(a.x, b.x), std::fmax(a.y, b.y)), std::fmax(a.z, b.z));
  float t = t0 > t1 ? NAN : (t0 > tmin && t0 < tmax ? t0 : (t1 > tmin && t1 < tmax ? t1 : NAN));
  *t_out = t;
  return aabb_contains_or_intersects(bb8, r, tmin, tmax) ? 1 : 0;
}
void dfo_ray_transform(const float* m16, const float* o, const float* d, float* out6) {
  M44 m = load_m44(m16);
  Ray r = transform_ray(m, make_ray(V3{o[0], o[1], o[2]}, V3{d[0], d[1], d[2]}));
  out6[0] = r.o.x; out6[1] = r.o.y; out6[2] = r.o.z; out6[3] = r.d.x; out6[4] = r.d.y; out6[5] = r.d.z;
}
void dfo_onb_from_w(const float* w, float* out9) { ONB b = onb_from_w(V3{w[0], w[1], w[2]}); float v[9] = {b.w.x, b.w.y, b.w.z, b.v.x, b.v.y, b.v.z, b.u.x, b.u.y, b.u.z}; std::memcpy(out9, v, sizeof v); }
void dfo_onb_from_wv(const float* w, const float* vv, float* out9) { ONB b = onb_from_wv(V3{w[0], w[1], w[2]}, V3{vv[0], vv[1], vv[2]}); float v[9] = {b.w.x, b.w.y, b.w.z, b.v.x, b.v.y, b.v.z, b.u.x, b.u.y, b.u.z}; std::memcpy(out9, v, sizeof v); }
void dfo_rgb_to_xyz(const float* c, float* out) { V3 r = srgb().to_xyz(V3{c[0], c[1], c[2]}); out[0] = r.x; out[1] = r.y; out[2] = r.z; }
void dfo_xyz_to_rgb(const float* c, float* out) { V3 r = srgb().to_rgb(V3{c[0], c[1], c[2]}); out[0] = r.x; out[1] = r.y; out[2] = r.z; }
// Generic colour space (ColorSpaceF(breakPoint, gamma, xR, yR, xG, yG, xB, yB, xW, yW)):
// op 0 RGB->XYZ, 1 XYZ->RGB, 2 redo gamma, 3 undo gamma.
void dfo_colorspace(const float* p10, int op, const float* c, float* out) {
  ColorSpace cs(p10[0], p10[1], p10[2], p10[3], p10[4], p10[5], p10[6], p10[7], p10[8], p10[9]);
  V3 v = {c[0], c[1], c[2]}, r;
  if (op == 0) r = cs.to_xyz(v);
  else if (op == 1) r = cs.to_rgb(v);
  else if (op == 2) r = {cs.redo(v.x), cs.redo(v.y), cs.redo(v.z)};
  else r = {cs.undo(v.x), cs.undo(v.y), cs.undo(v.z)};
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
// OrthonormalBasis33F.transform(matrix, onb): onb9/out9 = w, v, u
void dfo_onb_transform(const float* m16, const float* onb9, float* out9) {
  M44 m = load_m44(m16);
  ONB b{V3{onb9[0], onb9[1], onb9[2]}, V3{onb9[3], onb9[4], onb9[5]}, V3{onb9[6], onb9[7], onb9[8]}};
  V3 u = normalize(transform_vector(m, b.u)), v = normalize(transform_vector(m, b.v)), w = normalize(transform_vector(m, b.w));
  float o[9] = {w.x, w.y, w.z, v.x, v.y, v.z, u.x, u.y, u.z};
  std::memcpy(out9, o, sizeof o);
}
float dfo_srgb_redo(float v) { return srgb().redo(v); }
float dfo_srgb_undo(float v) { return srgb().undo(v); }
// filter/GaussianFilter2F.java: evaluate(x, y) with resolution (rx, ry) and falloff
float dfo_gaussian_filter(float x, float y, float rx, float ry, float falloff) {
  float ex = std::exp(-falloff * rx * rx), ey = std::exp(-falloff * ry * ry);
  auto g = [&](float d, float e) { return std::fmax(0.0f, std::exp(-falloff * d * d) - e); };
  return g(x, ex) * g(y, ey);
}
// filter/TriangleFilter2F.java: evaluate(x, y)
float dfo_triangle_filter(float x, float y, float rx, float ry) { return std::fmax(0.0f, rx - std::fabs(x)) * std::fmax(0.0f, ry - std::fabs(y)); }
unsigned int dfo_rng_path_key(unsigned int seed, unsigned int pixel, unsigned int sample) { return rng_path_key(seed, pixel, sample); }
float dfo_rng_uniform(unsigned int key, unsigned int dim) { return rng_uniform(key, dim); }
int dfo_primary_ray(void* s, float ix, float iy, float px, float py, float* out6) {
  Scene* sc = (Scene*)s;
  Ray r;
  if (!primary_ray(sc->cam, ix, iy, px, py, 0.5f, 0.5f, &r)) return 0;
  out6[0] = r.o.x; out6[1] = r.o.y; out6[2] = r.o.z; out6[3] = r.d.x; out6[4] = r.d.y; out6[5] = r.d.z;
  return 1;
}
// One candidate of a primary hit, for the near-tie check of hit-id mismatches:
// the primary ray of pixel (x, y), sample 0 of `seed` on a film `width` pixels
// wide (the render's jitter, moved by (dpx, dpy) pixels), tested against
// primitive `prim` alone in its object space (no bounding volume, no drift).
// Returns 1 with the world t of a hit in (tMinimum, tMaximum), 0 on a miss,
// -1 for bad arguments.
int dfo_primary_prim_t(void* s, unsigned int seed, int width, int x, int y, float dpx, float dpy, int prim, float* t_out) {
  Scene* sc = (Scene*)s;
  if (!sc || !t_out || prim < 0 || prim >= sc->prim_count || width <= 0 || x < 0 || y < 0) return -1;
  const uint32_t key = rng_path_key(seed, (uint32_t)((size_t)y * width + x), 0u);
  Ray r;
  if (!primary_ray(sc->cam, (float)x, (float)y, rng_uniform(key, kDimPixelX) + dpx, rng_uniform(key, kDimPixelY) + dpy,
                   rng_uniform(key, kDimLensU), rng_uniform(key, kDimLensV), &r))
    return 0;
  const int32_t* P = sc->prims.data() + (size_t)prim * 8;
  const Ray ro = transform_ray(sc->w2o[prim], r);
  int aux = -1;
  const float tmaxo = transform_t(sc->w2o[prim], r, ro, kTMaximum);
  const float th = shape_t(*sc, P[6], P[7], ro, kTMinimum, tmaxo, &aux);
  if (std::isnan(th) || !(th > kTMinimum) || !(th < tmaxo)) return 0;
  const Ray rw = transform_ray(sc->o2w[prim], ro);
  *t_out = transform_t(sc->o2w[prim], ro, rw, th);
  return 1;
}
// noise/PerlinNoiseF.java, noise/SimplexNoiseF.java
float dfo_perlin(float x, float y, float z) { return dfo_noise::perlin(x, y, z); }
float dfo_perlin_turbulence(float x, float y, float z, int octaves) { return dfo_noise::perlin_turbulence(x, y, z, octaves); }
float dfo_simplex(float x, float y, float z) { return dfo_noise::simplex(x, y, z); }
float dfo_simplex_fbm(float x, float y, float z, float frequency, float gain, float minimum, float maximum, int octaves) {
  return dfo_noise::simplex_fbm(x, y, z, frequency, gain, minimum, maximum, octaves);
}

}  // extern "C"
