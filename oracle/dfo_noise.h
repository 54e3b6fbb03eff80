// Oracle (test infrastructure): the reference's noise functions, restated.
//
// noise/PerlinNoiseF.java  noiseXYZ (:113), turbulenceXYZ(x, y, z, octaves) (:231)
// noise/SimplexNoiseF.java noiseXYZ (:404), fractionalBrownianMotionXYZ (:246)
//
// Perlin's improved noise with the reference's own gradient selection
// (u = x unless hash in 8..11 or 14..15, v = y for hash < 4 or 12..13, else z)
// and Gustavson's 3D simplex noise.  Both use Ken Perlin's published
// permutation table as the reference holds it: entry 156 is 23 where
// Perlin's table has 223, so 23 occurs twice and 223 not at all.
#pragma once
#include <cmath>
#include <cstdint>

namespace dfo_noise {

inline int perm(int i) {
  static const unsigned char kP[256] = {
      151, 160, 137, 91,  90,  15,  131, 13,  201, 95,  96,  53,  194, 233, 7,   225, 140, 36,  103, 30,  69,  142,
      8,   99,  37,  240, 21,  10,  23,  190, 6,   148, 247, 120, 234, 75,  0,   26,  197, 62,  94,  252, 219, 203,
      117, 35,  11,  32,  57,  177, 33,  88,  237, 149, 56,  87,  174, 20,  125, 136, 171, 168, 68,  175, 74,  165,
      71,  134, 139, 48,  27,  166, 77,  146, 158, 231, 83,  111, 229, 122, 60,  211, 133, 230, 220, 105, 92,  41,
      55,  46,  245, 40,  244, 102, 143, 54,  65,  25,  63,  161, 1,   216, 80,  73,  209, 76,  132, 187, 208, 89,
      18,  169, 200, 196, 135, 130, 116, 188, 159, 86,  164, 100, 109, 198, 173, 186, 3,   64,  52,  217, 226, 250,
      124, 123, 5,   202, 38,  147, 118, 126, 255, 82,  85,  212, 207, 206, 59,  227, 47,  16,  58,  17,  182, 189,
      28,  42,  23,  183, 170, 213, 119, 248, 152, 2,   44,  154, 163, 70,  221, 153, 101, 155, 167, 43,  172, 9,
      129, 22,  39,  253, 19,  98,  108, 110, 79,  113, 224, 232, 178, 185, 112, 104, 218, 246, 97,  228, 251, 34,
      242, 193, 238, 210, 144, 12,  191, 179, 162, 241, 81,  51,  145, 235, 249, 14,  239, 107, 49,  192, 214, 31,
      181, 199, 106, 157, 184, 84,  204, 176, 115, 121, 50,  45,  127, 4,   150, 254, 138, 236, 205, 93,  222, 114,
      67,  29,  24,  72,  243, 141, 128, 195, 78,  66,  215, 61,  156, 180};
  return kP[i & 255];  // the doubled table of the reference repeats the 256 entries
}

inline float clampf(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Gradient dot product of the reference's Perlin variant for corner offsets (dx, dy, dz).
inline float perlin_grad(int hash, float dx, float dy, float dz) {
  const bool su = hash < 8 || hash == 12 || hash == 13;
  const bool sv = hash < 4 || hash == 12 || hash == 13;
  const float gu = su ? dx : dy;
  const float gv = sv ? dy : dz;
  return ((hash & 1) == 0 ? gu : -gu) + ((hash & 2) == 0 ? gv : -gv);
}

// PerlinNoiseF.noiseXYZ
inline float perlin(float x, float y, float z) {
  if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z)) return 0.0f;
  const float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  const int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
  const float x1 = x - fx, y1 = y - fy, z1 = z - fz;
  const float u = x1 * x1 * x1 * (x1 * (x1 * 6.0f - 15.0f) + 10.0f);
  const float v = y1 * y1 * y1 * (y1 * (y1 * 6.0f - 15.0f) + 10.0f);
  const float w = z1 * z1 * z1 * (z1 * (z1 * 6.0f - 15.0f) + 10.0f);
  const int a0 = perm(X) + Y, a1 = perm(a0) + Z, a2 = perm(a0 + 1) + Z;
  const int b0 = perm(X + 1) + Y, b1 = perm(b0) + Z, b2 = perm(b0 + 1) + Z;
  const float g0 = perlin_grad(perm(a1) & 15, x1, y1, z1);
  const float g1 = perlin_grad(perm(b1) & 15, x1 - 1.0f, y1, z1);
  const float g2 = perlin_grad(perm(a2) & 15, x1, y1 - 1.0f, z1);
  const float g3 = perlin_grad(perm(b2) & 15, x1 - 1.0f, y1 - 1.0f, z1);
  const float g4 = perlin_grad(perm(a1 + 1) & 15, x1, y1, z1 - 1.0f);
  const float g5 = perlin_grad(perm(b1 + 1) & 15, x1 - 1.0f, y1, z1 - 1.0f);
  const float g6 = perlin_grad(perm(a2 + 1) & 15, x1, y1 - 1.0f, z1 - 1.0f);
  const float g7 = perlin_grad(perm(b2 + 1) & 15, x1 - 1.0f, y1 - 1.0f, z1 - 1.0f);
  const float l0 = g0 + u * (g1 - g0), l1 = g2 + u * (g3 - g2), l2 = g4 + u * (g5 - g4), l3 = g6 + u * (g7 - g6);
  const float l4 = l0 + v * (l1 - l0), l5 = l2 + v * (l3 - l2);
  return clampf(l4 + w * (l5 - l4), -1.0f, 1.0f);
}

// PerlinNoiseF.turbulenceXYZ(x, y, z, octaves): octave i at frequency 2^i, weight 2^-i
inline float perlin_turbulence(float x, float y, float z, int octaves) {
  float n = std::fabs(perlin(x, y, z));
  float weight = 1.0f;
  for (int i = 1; i < octaves; ++i) {
    weight *= 2.0f;
    n += std::fabs(perlin(x * weight, y * weight, z * weight)) / weight;
  }
  return n;
}

inline int fast_floor(float v) { const int i = (int)v; return v < (float)i ? i - 1 : i; }

// SimplexNoiseF.noiseXYZ (Gustavson): skew to the simplex grid, pick the
// simplex by the order of the offsets, sum four corner kernels (0.6 - r^2)^4.
inline float simplex(float x, float y, float z) {
  if (!std::isfinite(x) || !std::isfinite(y) || !std::isfinite(z)) return 0.0f;
  static const float kG[12][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1},
                                  {1, 0, -1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1}};
  const float F3 = 1.0f / 3.0f, G3 = 1.0f / 6.0f;
  const float s = (x + y + z) * F3;
  const int i = fast_floor(x + s), j = fast_floor(y + s), k = fast_floor(z + s);
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
  const float c[4][3] = {{x0, y0, z0},
                         {x0 - i1 + G3, y0 - j1 + G3, z0 - k1 + G3},
                         {x0 - i2 + 2.0f * G3, y0 - j2 + 2.0f * G3, z0 - k2 + 2.0f * G3},
                         {x0 - 1.0f + 3.0f * G3, y0 - 1.0f + 3.0f * G3, z0 - 1.0f + 3.0f * G3}};
  const int ii = i & 255, jj = j & 255, kk = k & 255;
  const int gi[4] = {perm(ii + perm(jj + perm(kk))) % 12, perm(ii + i1 + perm(jj + j1 + perm(kk + k1))) % 12,
                     perm(ii + i2 + perm(jj + j2 + perm(kk + k2))) % 12, perm(ii + 1 + perm(jj + 1 + perm(kk + 1))) % 12};
  float n = 0.0f;
  for (int q = 0; q < 4; ++q) {
    const float tq = 0.6f - c[q][0] * c[q][0] - c[q][1] * c[q][1] - c[q][2] * c[q][2];
    if (tq >= 0.0f) n += (tq * tq) * (tq * tq) * (kG[gi[q]][0] * c[q][0] + kG[gi[q]][1] * c[q][1] + kG[gi[q]][2] * c[q][2]);
  }
  return clampf(32.0f * n, -1.0f, 1.0f);
}

// SimplexNoiseF.fractionalBrownianMotionXYZ: amplitude-normalised octave sum mapped to [minimum, maximum]
inline float simplex_fbm(float x, float y, float z, float frequency, float gain, float minimum, float maximum, int octaves) {
  float amp = 1.0f, amp_sum = 0.0f, f = frequency, n = 0.0f;
  for (int i = 0; i < octaves; ++i) {
    n += simplex(x * f, y * f, z * f) * amp;
    amp_sum += amp;
    amp *= gain;
    f *= 2.0f;
  }
  n /= amp_sum;
  return n * (maximum - minimum) / 2.0f + (maximum + minimum) / 2.0f;
}

}  // namespace dfo_noise
