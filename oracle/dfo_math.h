// Oracle math kernel: a CPU restatement of the Dayflower float geometry the
// CPURenderer path uses.  TEST INFRASTRUCTURE ONLY: the renderer product never
// links or calls anything under oracle/.
//
// Each helper names the reference function it restates (paths are relative to
// src/main/java/org/dayflower/ in macroing/Dayflower).
#pragma once

#include <cmath>
#include <cstdint>
#include <cfloat>
#include <limits>

namespace dfo {

constexpr float kPi = 3.14159265358979323846f;                 // utility/Floats.java:94
constexpr float kTMinimum = 0.001f;                            // scene/Scene.java:70
constexpr float kTMaximum = FLT_MAX;                           // scene/Scene.java:65
inline float next_up(float v) { return std::nextafter(v, std::numeric_limits<float>::infinity()); }
inline float next_down(float v) { return std::nextafter(v, -std::numeric_limits<float>::infinity()); }
inline float machine_epsilon() { return std::nextafter(1.0f, 2.0f) - 1.0f; }  // ulp(1) ...
// utility/Floats.java:44 MACHINE_EPSILON = ulp(1) * 0.5
inline float kMachineEpsilon() { return machine_epsilon() * 0.5f; }
// utility/Floats.java:565 gamma(n) = n e / (1 - n e)
inline float gamma_n(int n) { float e = kMachineEpsilon(); return (n * e) / (1.0f - n * e); }
inline bool is_zero(float v) { return v == 0.0f; }
inline float saturate(float v, float a, float b) { float lo = std::fmin(a, b), hi = std::fmax(a, b); return v < lo ? lo : (v > hi ? hi : v); }

struct V3 { float x, y, z; };
inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 divide(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
// geometry/Vector3F.java:1000 normalize(): vectors whose length is within
// [nextDown^3(1), nextUp(1)] are returned unchanged.
inline V3 normalize(V3 v) {
  static const float lo = next_down(next_down(next_down(1.0f)));
  static const float hi = next_up(1.0f);
  float l = length(v);
  if (l >= lo && l <= hi) return v;
  return divide(v, l);
}
inline float distance(V3 a, V3 b) { return length(b - a); }
inline float distance_squared(V3 a, V3 b) { V3 d = b - a; return dot(d, d); }
inline float max_component(V3 a) { return std::fmax(a.x, std::fmax(a.y, a.z)); }

// geometry/Matrix44F.java: row-major element11..element44, array order as
// Matrix44F.toArray() (row by row).
struct M44 { float m[16]; };
inline V3 transform_point_divide(const M44& M, V3 p) {  // geometry/Point3F.java:700
  const float* m = M.m;
  float x = m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3];
  float y = m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7];
  float z = m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11];
  float w = m[12] * p.x + m[13] * p.y + m[14] * p.z + m[15];
  return (w == 1.0f || w == 0.0f) ? V3{x, y, z} : V3{x / w, y / w, z / w};
}
inline V3 transform_vector(const M44& M, V3 v) {  // geometry/Vector3F.java:1235
  const float* m = M.m;
  return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z, m[8] * v.x + m[9] * v.y + m[10] * v.z};
}
inline V3 transform_vector_transpose(const M44& M, V3 v) {  // geometry/Vector3F.java:1298
  const float* m = M.m;
  return {m[0] * v.x + m[4] * v.y + m[8] * v.z, m[1] * v.x + m[5] * v.y + m[9] * v.z, m[2] * v.x + m[6] * v.y + m[10] * v.z};
}

struct Ray { V3 o, d; };
// geometry/Ray3F.java:53 the constructor normalizes the direction.
inline Ray make_ray(V3 o, V3 d) { return Ray{o, normalize(d)}; }
// geometry/Ray3F.java:219
inline Ray transform_ray(const M44& M, const Ray& r) { return make_ray(transform_point_divide(M, r.o), transform_vector(M, r.d)); }

// geometry/OrthonormalBasis33F.java
struct ONB { V3 w, v, u; };
inline V3 compute_v(V3 w) {  // geometry/Vector3F.java:527
  V3 n = normalize(w);
  float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
  if (ax < ay && ax < az) return normalize(V3{0.0f, n.z, -n.y});
  if (ay < az) return normalize(V3{n.z, 0.0f, -n.x});
  return normalize(V3{n.y, -n.x, 0.0f});
}
inline ONB onb_from_w(V3 w) {  // OrthonormalBasis33F.java:88
  ONB o; o.w = normalize(w); o.v = compute_v(w); o.u = cross(o.v, o.w); return o;
}
inline ONB onb_from_wv(V3 w, V3 v) {  // OrthonormalBasis33F.java:110
  ONB o; o.w = normalize(w); o.u = normalize(cross(normalize(v), o.w)); o.v = cross(o.w, o.u); return o;
}
inline ONB onb_transform_transpose(const M44& M, const ONB& b) {  // OrthonormalBasis33F.java:402
  ONB o; o.u = normalize(transform_vector_transpose(M, b.u)); o.v = normalize(transform_vector_transpose(M, b.v)); o.w = normalize(transform_vector_transpose(M, b.w)); return o;
}
inline ONB onb_flip_w(const ONB& b) { ONB o = b; o.w = -b.w; return o; }  // OrthonormalBasis33F.java:350
inline V3 to_world(V3 v, const ONB& b) { return b.u * v.x + b.v * v.y + b.w * v.z; }        // Vector3F.java:1256
inline V3 to_local(V3 v, const ONB& b) { return V3{dot(v, b.u), dot(v, b.v), dot(v, b.w)}; }  // Vector3F.java:1277

// ---------------------------------------------------------------------------
// Counter-based random numbers.  The Java CPURenderer draws from an unseeded
// per-thread generator (NRooksSampler + Randoms.nextFloat), so its stream is
// not reproducible; this build keys every draw by (seed, pixel, sample,
// dimension) instead, identically on the CPU and on the GPU, so that a sample
// in the oracle and the same sample on the device use the same numbers.
inline uint32_t rng_hash(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16; return x;
}
inline uint32_t rng_path_key(uint32_t seed, uint32_t pixel, uint32_t sample) {
  return rng_hash(seed ^ rng_hash(pixel ^ rng_hash(sample + 0x632be5abu)));
}
inline float rng_uniform(uint32_t key, uint32_t dim) {
  return (float)(rng_hash(key + dim * 0x9e3779b9u) >> 8) * (1.0f / 16777216.0f);
}
// Dimension layout (shared with the device renderer).
enum : uint32_t {
  kDimPixelX = 0, kDimPixelY = 1, kDimLensU = 2, kDimLensV = 3,
  kDimBounceBase = 8, kDimBounceStride = 16,
  kDimLightPick = 0, kDimLightSampleU = 1, kDimLightSampleV = 2, kDimMisSampleU = 3, kDimMisSampleV = 4,
  kDimSunPick = 5, kDimBsdfU = 6, kDimBsdfV = 7, kDimRoulette = 8, kDimMaterial = 9,
};
inline uint32_t bounce_dim(int bounce, uint32_t which) { return kDimBounceBase + (uint32_t)bounce * kDimBounceStride + which; }

}  // namespace dfo
