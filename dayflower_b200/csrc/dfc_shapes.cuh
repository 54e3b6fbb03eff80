// Device intersection and surfaces of the record-sized analytic shapes: disk,
// cylinder, cone, paraboloid, hyperboloid, rectangular cuboid and torus, in
// object space over their compiled records (scene/compiler/
// CompiledShape3FCache.java:90-310).  Each follows the CPU shape class
// (geometry/shape/<Shape>3F.java, intersectionT and doCreate*) operation by
// operation; the build's -fmad=false keeps every float operation separately
// rounded as in Java.  A miss returns -1.
#pragma once

#include "dfc_device.cuh"

namespace dfc {

// java.lang.Math.min/max on floats: NaN propagates, -0 < +0.
DFC_D float jmin(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == 0.0f && b == 0.0f) return signbit(a) ? a : b;
  return a <= b ? a : b;
}
DFC_D float jmax(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == 0.0f && b == 0.0f) return signbit(a) ? b : a;
  return a >= b ? a : b;
}

// geometry/Point3F.java:223 sphericalPhi; the reference's atan2 is Math.atan2 in double.
DFC_D float spherical_phi(float x, float y) {
  const float phi = (float)atan2((double)y, (double)x);
  return phi < 0.0f ? phi + 2.0f * kPi : phi;
}

// utility/Floats.java:1227 solveQuadraticSystem (NaN, NaN without real roots).
DFC_D void solve_quadratic(float a, float b, float c, float* r0, float* r1) {
  const float disc2 = b * b - 4.0f * a * c;
  const float nan = __int_as_float(0x7fffffff);
  *r0 = nan; *r1 = nan;
  if (disc2 == 0.0f) {
    const float q = -0.5f * b / a;
    *r0 = q; *r1 = q;
  } else if (disc2 > 0.0f) {
    const float disc = sqrtf(disc2);
    const float q = -0.5f * (b > 0.0f ? b + disc : b - disc);
    const float x0 = q / a, x1 = c / q;
    *r0 = jmin(x0, x1); *r1 = jmax(x0, x1);
  }
}

DFC_D V3 point_at(V3 o, V3 d, float t) { return V3{o.x + d.x * t, o.y + d.y * t, o.z + d.z * t}; }
DFC_D float len2d(V3 p) { return sqrtf(p.x * p.x + p.y * p.y); }

// Record layouts (floats): disk phiMax, ri, ro, zMax | cylinder phiMax, r, zMax,
// zMin | cone phiMax, r, zMax | paraboloid phiMax, r, zMax, zMin | hyperboloid
// phiMax, A, B, aH, cH, rMax, zMax, zMin | cuboid max, min | torus ri, ro.

DFC_D V3 cylinder_point(const float* q, V3 o, V3 d, float t) {
  const V3 p = point_at(o, d, t);
  const float s = q[1] / len2d(p);
  return V3{p.x * s, p.y * s, p.z};
}

DFC_D float hyperboloid_phi_v(const float* q, V3 p, float v) {
  const float ax = (1.0f - v) * q[1] + v * q[4], ay = (1.0f - v) * q[2] + v * q[5];
  return spherical_phi(p.x * ax + p.y * ay, p.y * ax - p.x * ay);
}
DFC_D float hyperboloid_phi(const float* q, V3 p) { return hyperboloid_phi_v(q, p, (p.z - q[3]) / (q[6] - q[3])); }

// The quadric root loop shared by Cylinder3F, Cone3F, Paraboloid3F and
// Hyperboloid3F: the first root in (tmin, tmax) whose point is inside the
// clipped surface; a NaN root ends the search.
DFC_D bool quadric_inside(int shape, const float* q, V3 p) {
  switch (shape) {
    case kShapeCylinder: return p.z >= q[3] && p.z <= q[2] && spherical_phi(p.x, p.y) <= q[0];
    case kShapeCone: return p.z >= 0.0f && p.z <= q[2] && spherical_phi(p.x, p.y) <= q[0];
    case kShapeParaboloid: return p.z >= q[3] && p.z <= q[2] && spherical_phi(p.x, p.y) <= q[0];
    default: return p.z >= q[11] && p.z <= q[10] && hyperboloid_phi(q, p) <= q[0];  // hyperboloid
  }
}

DFC_D float quadric_root_t(int shape, const float* q, V3 o, V3 d, float tmin, float tmax) {
  float a, b, c;
  if (shape == kShapeCylinder) {
    a = d.x * d.x + d.y * d.y;
    b = 2.0f * (d.x * o.x + d.y * o.y);
    c = o.x * o.x + o.y * o.y - q[1] * q[1];
  } else if (shape == kShapeCone) {
    const float k = (q[1] / q[2]) * (q[1] / q[2]);
    a = d.x * d.x + d.y * d.y - k * d.z * d.z;
    b = 2.0f * (d.x * o.x + d.y * o.y - k * d.z * (o.z - q[2]));
    c = o.x * o.x + o.y * o.y - k * (o.z - q[2]) * (o.z - q[2]);
  } else if (shape == kShapeParaboloid) {
    const float k = q[2] / (q[1] * q[1]);
    a = k * (d.x * d.x + d.y * d.y);
    b = 2.0f * k * (d.x * o.x + d.y * o.y) - d.z;
    c = k * (o.x * o.x + o.y * o.y) - o.z;
  } else {
    const float aH = q[7], cH = q[8];
    a = aH * d.x * d.x + aH * d.y * d.y - cH * d.z * d.z;
    b = 2.0f * (aH * d.x * o.x + aH * d.y * o.y - cH * d.z * o.z);
    c = aH * o.x * o.x + aH * o.y * o.y - cH * o.z * o.z - 1.0f;
  }
  float ts[2];
  solve_quadratic(a, b, c, &ts[0], &ts[1]);
  for (int i = 0; i < 2; ++i) {
    const float t = ts[i];
    if (t != t) return -1.0f;
    if (t > tmin && t < tmax) {
      const V3 p = shape == kShapeCylinder ? cylinder_point(q, o, d, t) : point_at(o, d, t);
      if (quadric_inside(shape, q, p)) return t;
    }
  }
  return -1.0f;
}

// geometry/shape/Disk3F.java:342
DFC_D float disk_t(const float* q, V3 o, V3 d, float tmin, float tmax) {
  if (d.z == 0.0f) return -1.0f;
  const float t = (q[3] - o.z) / d.z;
  if (t <= tmin || t >= tmax) return -1.0f;
  V3 p = point_at(o, d, t);
  p.z = q[3];
  const float l2 = p.x * p.x + p.y * p.y;
  if (l2 > q[2] * q[2] || l2 < q[1] * q[1] || spherical_phi(p.x, p.y) > q[0]) return -1.0f;
  return t;
}

// geometry/shape/RectangularCuboid3F.java intersectionT
DFC_D float cuboid_t(const float* q, V3 o, V3 d, float tmin, float tmax) {
  const V3 rd = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  const V3 da = {(q[3] - o.x) * rd.x, (q[4] - o.y) * rd.y, (q[5] - o.z) * rd.z};
  const V3 db = {(q[0] - o.x) * rd.x, (q[1] - o.y) * rd.y, (q[2] - o.z) * rd.z};
  const float t0 = jmax(jmax(jmin(da.x, db.x), jmin(da.y, db.y)), jmin(da.z, db.z));
  const float t1 = jmin(jmin(jmax(da.x, db.x), jmax(da.y, db.y)), jmax(da.z, db.z));
  if (t0 > t1) return -1.0f;
  if (t0 > tmin && t0 < tmax) return t0;
  if (t1 > tmin && t1 < tmax) return t1;
  return -1.0f;
}

// geometry/shape/Torus3F.java: the quartic in double precision with the
// reference's resolvent-cubic solution (doSolveCubicForQuartic, doSolveQuartic).
DFC_D double torus_cubic(double p, double q, double r) {
  const double p2 = p * p;
  const double q0 = (p2 - 3.0 * q) / 9.0;
  const double q0c = q0 * q0 * q0;
  const double r0 = (p * (p2 - 4.5 * q) + 13.5 * r) / 27.0;
  const double r02 = r0 * r0;
  const double dd = q0c - r02;
  const double e = p / 3.0;
  if (dd >= 0.0) {
    const double theta = acos(r0 / sqrt(q0c)) / 3.0;
    return -2.0 * sqrt(q0) * cos(theta) - e;
  }
  const double q1 = pow(sqrt(r02 - q0c) + fabs(r0), 1.0 / 3.0);
  return r0 < 0.0 ? (q1 + q0 / q1) - e : -(q1 + q0 / q1) - e;
}

DFC_D int torus_quartic(double a, double b, double c, double d, double e, double* out) {
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
    d2 = sqrt(d2);
  } else {
    d1 = sqrt(d1);
    d2 = 0.5 * q / d1;
  }
  const double q1 = d1 * d1, q2 = -0.25 * bA;
  const double pm = q1 - 4.0 * (z - d2), pp = q1 - 4.0 * (z + d2);
  if (pm >= 0.0 && pp >= 0.0) {
    const double pms = sqrt(pm), pps = sqrt(pp);
    out[0] = -0.5 * (d1 + pms) + q2;
    out[1] = -0.5 * (d1 - pms) + q2;
    out[2] = 0.5 * (d1 + pps) + q2;
    out[3] = 0.5 * (d1 - pps) + q2;
    for (int i = 1; i < 4; ++i)
      for (int j = i; j > 0 && out[j - 1] > out[j]; --j) { const double s = out[j]; out[j] = out[j - 1]; out[j - 1] = s; }
    return 4;
  }
  if (pm >= 0.0) {
    const double pms = sqrt(pm);
    out[0] = -0.5 * (d1 + pms) + q2;
    out[1] = -0.5 * (d1 - pms) + q2;
    return 2;
  }
  if (pp >= 0.0) {
    const double pps = sqrt(pp);
    out[0] = 0.5 * (d1 - pps) + q2;
    out[1] = 0.5 * (d1 + pps) + q2;
    return 2;
  }
  return 0;
}

DFC_D float torus_t(const float* q, V3 o, V3 d, float tmin, float tmax) {
  const float ri2 = q[0] * q[0], ro2 = q[1] * q[1];
  const double f0 = (double)dot(d, d);
  const double f1 = (double)dot(o, d) * 2.0;
  const double f2 = ri2, f3 = ro2;
  const double f4 = (double)dot(o, o) - f2 - f3;
  const double f5 = d.z, f6 = o.z;
  const double a = f0 * f0;
  const double b = f0 * 2.0 * f1;
  const double c = f1 * f1 + 2.0 * f0 * f4 + 4.0 * f3 * f5 * f5;
  const double dq = f1 * 2.0 * f4 + 8.0 * f3 * f6 * f5;
  const double e = f4 * f4 + 4.0 * f3 * f6 * f6 - 4.0 * f3 * f2;
  double ts[4];
  const int n = torus_quartic(a, b, c, dq, e, ts);
  if (n == 0) return -1.0f;
  if (ts[0] >= tmax || ts[n - 1] <= tmin) return -1.0f;
  for (int i = 0; i < n; ++i)
    if (ts[i] > tmin) return (float)ts[i];
  return -1.0f;
}

// geometry/shape/Polygon3F.java over the compiled record: points 0, 1 and n-1
// at +0, +3, +6, surface normal +9, point count +12, the polygon projected on
// its plane at +13 (two floats per point).  Containment is Polygon2F.contains:
// on an edge (LineSegment2F.contains) or inside by the crossing test.
DFC_D bool polygon_contains(const float* q, V3 p) {
  const V3 a = ld3(q), w = ld3(q + 9);
  const V3 u = normalize(ld3(q + 3) - a), v = cross(w, u);
  const V3 ap = p - a;
  const float px = dot(ap, u), py = dot(ap, v);
  const int n = (int)q[12];
  const float* P = q + 13;
  for (int i = 0, j = 1; i < n; ++i, j = (j + 1) % n) {
    const float ax = P[2 * i], ay = P[2 * i + 1], bx = P[2 * j], by = P[2 * j + 1];
    const float dx = px - ax, dy = py - ay, ex = bx - ax, ey = by - ay;
    if (dx * ey - dy * ex != 0.0f) continue;
    if (fabsf(ex) >= fabsf(ey) ? (ex > 0.0f ? ax <= px && px <= bx : bx <= px && px <= ax)
                               : (ey > 0.0f ? ay <= py && py <= by : by <= py && py <= ay))
      return true;
  }
  bool inside = false;
  for (int i = 0, j = n - 1; i < n; j = i++) {
    const float ix = P[2 * i], iy = P[2 * i + 1], jx = P[2 * j], jy = P[2 * j + 1];
    if ((iy > py) != (jy > py) && px < (jx - ix) * (py - iy) / (jy - iy) + ix) inside = !inside;
  }
  return inside;
}
DFC_D float polygon_t(const float* q, V3 o, V3 d, float tmin, float tmax) {  // Polygon3F.java:321
  const V3 n = ld3(q + 9);
  const float dp = dot(n, d);
  if (dp == 0.0f) return -1.0f;
  const float t = dot(ld3(q) - o, n) / dp;
  if (t > tmin && t < tmax && polygon_contains(q, point_at(o, d, t))) return t;
  return -1.0f;
}

// Object-space t of one record shape; -1 on a miss.  Out of line, so that
// its double-precision torus solve stays out of the traversal loop's frame.
static __device__ __noinline__ float record_shape_t(int shape, const float* q, V3 o, V3 d, float tmin, float tmax) {
  switch (shape) {
    case kShapeDisk: return disk_t(q, o, d, tmin, tmax);
    case kShapeCuboid: return cuboid_t(q, o, d, tmin, tmax);
    case kShapeTorus: return torus_t(q, o, d, tmin, tmax);
    case kShapePolygon: return polygon_t(q, o, d, tmin, tmax);
    case kShapeCylinder: case kShapeCone: case kShapeParaboloid: case kShapeHyperboloid:
      return quadric_root_t(shape, q, o, d, tmin, tmax);
    default: return -1.0f;
  }
}

DFC_D ONB uv_frame(V3 u, V3 v) {
  u = normalize(u);
  v = normalize(v);
  ONB g;
  g.w = cross(u, v); g.v = v; g.u = u;  // OrthonormalBasis33F(w, v, u) keeps the vectors as given
  return g;
}

// Surface of a record shape at object-space distance t (doCreateSurfaceIntersection
// of each shape class).  Out of line: shading reaches it only for these shapes.
static __device__ __noinline__ Surface record_shape_surface(int shape, const float* q, V3 o, V3 d, float t) {
  Surface s;
  V3 p = point_at(o, d, t);
  const V3 pu = {-q[0] * p.y, q[0] * p.x, 0.0f};
  switch (shape) {
    case kShapeDisk: {
      p.z = q[3];
      const float l = len2d(p);
      s.g = uv_frame(V3{-q[0] * p.y, q[0] * p.x, 0.0f}, V3{p.x * (q[1] - q[2]) / l, p.y * (q[1] - q[2]) / l, 0.0f});
      s.tu = spherical_phi(p.x, p.y) / q[0];
      s.tv = (q[2] - l) / (q[2] - q[1]);
      break;
    }
    case kShapeCylinder: {
      p = cylinder_point(q, o, d, t);
      s.g = uv_frame(V3{-q[0] * p.y, q[0] * p.x, 0.0f}, V3{0.0f, 0.0f, q[2] - q[3]});
      s.tu = spherical_phi(p.x, p.y) / q[0];
      s.tv = (p.z - q[3]) / (q[2] - q[3]);
      break;
    }
    case kShapeCone: {
      const float value = 1.0f - (p.z / q[2]);
      s.g = uv_frame(pu, V3{-p.x / value, -p.y / value, q[2]});
      s.tu = spherical_phi(p.x, p.y) / q[0];
      s.tv = p.z / q[2];
      break;
    }
    case kShapeParaboloid: {
      const float dz = q[2] - q[3];
      s.g = uv_frame(pu, V3{dz * (p.x / (2.0f * p.z)), dz * (p.y / (2.0f * p.z)), dz});
      s.tu = spherical_phi(p.x, p.y) / q[0];
      s.tv = (p.z - q[3]) / dz;
      break;
    }
    case kShapeHyperboloid: {
      const float phi = hyperboloid_phi(q, p);
      const float c = (float)cos((double)phi), sn = (float)sin((double)phi);
      s.g = uv_frame(pu, V3{(q[4] - q[1]) * c - (q[5] - q[2]) * sn, (q[4] - q[1]) * sn + (q[5] - q[2]) * c, q[6] - q[3]});
      s.tv = (p.z - q[3]) / (q[6] - q[3]);
      s.tu = hyperboloid_phi_v(q, p, s.tv) / q[0];
      break;
    }
    case kShapeCuboid: {
      const V3 mid = {(q[0] + q[3]) * 0.5f, (q[1] + q[4]) * 0.5f, (q[2] + q[5]) * 0.5f};
      const V3 half = {(q[0] - q[3]) * 0.5f, (q[1] - q[4]) * 0.5f, (q[2] - q[5]) * 0.5f};
      const bool x0 = p.x + half.x - 0.0001f < mid.x, x1 = p.x - half.x + 0.0001f > mid.x;
      const bool y0 = p.y + half.y - 0.0001f < mid.y, y1 = p.y - half.y + 0.0001f > mid.y;
      const bool z0 = p.z + half.z - 0.0001f < mid.z, z1 = p.z - half.z + 0.0001f > mid.z;
      if (x0) s.g = onb_w(V3{-1, 0, 0});
      else if (x1) s.g = onb_w(V3{1, 0, 0});
      else if (y0) s.g = onb_w(V3{0, -1, 0});
      else if (y1) s.g = onb_w(V3{0, 1, 0});
      else if (z0) s.g = onb_w(V3{0, 0, -1});
      else if (z1) s.g = onb_w(V3{0, 0, 1});
      else { s.g.w = V3{0, 0, 1}; s.g.v = V3{0, 1, 0}; s.g.u = V3{1, 0, 0}; }
      auto nrm = [](float v, float a, float b) { const float mx = jmax(a, b), mn = jmin(a, b); return (v - mn) / (mx - mn); };
      s.tu = 0.0f; s.tv = 0.0f;
      if (x0 || x1) { s.tu = nrm(p.z, q[5], q[2]); s.tv = nrm(p.y, q[4], q[1]); }
      else if (y0 || y1) { s.tu = nrm(p.x, q[3], q[0]); s.tv = nrm(p.z, q[5], q[2]); }
      else if (z0 || z1) { s.tu = nrm(p.x, q[3], q[0]); s.tv = nrm(p.y, q[4], q[1]); }
      break;
    }
    case kShapePolygon: {  // Polygon3F.doCreateSurfaceIntersection / doCreateTextureCoordinates
      const V3 n = ld3(q + 9);
      const V3 na = {fabsf(n.x), fabsf(n.y), fabsf(n.z)};
      const bool isx = na.x > na.y && na.x > na.z, isy = na.y > na.z;
      auto px = [&](const float* c) { return isx ? c[1] : isy ? c[2] : c[0]; };
      auto py = [&](const float* c) { return isx ? c[2] : isy ? c[0] : c[1]; };
      // vB from the last point, vC from the second, as the reference pairs them
      const float ax = px(q), ay = py(q), abx = px(q + 6) - ax, aby = py(q + 6) - ay, acx = px(q + 3) - ax, acy = py(q + 3) - ay;
      const float dr = 1.0f / (abx * acy - aby * acx);
      const float hu = isx ? p.y : isy ? p.z : p.x, hv = isx ? p.z : isy ? p.x : p.y;
      s.g = onb_w(n);
      s.tu = hu * (-aby * dr) + hv * (abx * dr) + (ax * aby - ay * abx) * dr;
      s.tv = hu * (acy * dr) + hv * (-acx * dr) + (acx * ay - acy * ax) * dr;
      break;
    }
    default: {  // torus
      const float ri2 = q[0] * q[0], ro2 = q[1] * q[1];
      const float der = dot(p, p) - ri2 - ro2;
      s.g = onb_w(normalize(V3{p.x * der, p.y * der, p.z * der + 2.0f * ro2 * p.z}));
      const float phi = (float)asin((double)clampf(p.z / q[0], -1.0f, 1.0f));
      s.tu = spherical_phi(p.x, p.y) * (1.0f / (2.0f * kPi));
      s.tv = (phi + kPi / 2.0f) * (1.0f / kPi);
      break;
    }
  }
  s.s = s.g;
  s.p = p;
  return s;
}

}  // namespace dfc
