// Ray traversal of the two-level 4-wide hierarchy (device code shared by the
// kernels that trace rays: dfc_trace.cu, dfc_raytrace.cu and the batch engine's
// traversal).  trace_ray walks one ray on one thread; trace_rays is the
// persistent traversal over a ray list with per-lane refill.
#pragma once

#include <cuda_runtime.h>

#include "dfc_device.cuh"
#include "dfc_kernels.h"
#include "dfc_shapes.cuh"

namespace dfc {

namespace {

constexpr int kStack = 48;  // traversal stack entries per thread (shared memory)
constexpr int kTraceBlock = 128;

DFC_D unsigned warp_append(unsigned* counter, bool pred) {
  const unsigned mask = __ballot_sync(0xffffffffu, pred);
  const unsigned lane = threadIdx.x & 31u;
  const int leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (mask != 0u && (int)lane == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader < 0 ? 0 : leader);
  return base + (unsigned)__popc(mask & ((1u << lane) - 1u));
}

// ---- traversal --------------------------------------------------------------
struct Hit { float t; int prim; int aux; float t_obj; };

// Inverse direction for the slab tests.  A component that is exactly zero
// (a camera ray through the image's centre row or column) would give an
// infinite inverse, and the slab's fma(bound, inv, -origin * inv) would then
// be inf - inf = NaN and cull every box the ray is inside of; components
// below 2^-80 are taken as +-2^-80 instead, so the products stay finite for
// coordinates up to ~1e14 and the slabs of such a ray are (-huge, +huge) or
// empty as the exact ones would be.
DFC_D float safe_inv(float d) {
  const float tiny = 8.2718061e-25f;  // 2^-80
  return 1.0f / (fabsf(d) > tiny ? d : copysignf(tiny, d));
}
DFC_D V3 safe_inv(V3 d) { return V3{safe_inv(d.x), safe_inv(d.y), safe_inv(d.z)}; }

struct ObjRay { V3 o, d, inv; float s; };
DFC_D ObjRay obj_ray(const DPrim& pr, V3 o, V3 d) {
  ObjRay r;
  if (pr.identity) { r.o = o; r.d = d; r.s = 1.0f; }
  else {
    r.o = xf_point(pr.w2o, o);
    V3 dr = xf_vec(pr.w2o, d);
    float l = len(dr);
    if (l >= 0.99999982f && l <= 1.00000012f) { r.d = dr; r.s = 1.0f; }
    else { r.d = V3{dr.x / l, dr.y / l, dr.z / l}; r.s = l; }
  }
  r.inv = safe_inv(r.d);
  return r;
}

// Object-space test of one analytic primitive; returns the object distance or -1.
// Out of line: called at top-level leaves only, it keeps the traversal loop small.
// Its arguments are plain values (no references to the kernel's parameters or
// to a ray struct), so a call passes them in registers and the caller keeps no
// copy of the scene or the ray in local memory.  kRecords adds disk ... torus
// (the double-precision torus solve enlarges the call tree enough to cost the
// traversal loop registers, so scenes without those shapes run the
// instantiation without them).
template <bool kRecords>
__device__ __noinline__ float prim_t_v(const float* tri_attr, const float* rects, const float* shapes, int shape, int data, float ox, float oy, float oz,
               float dx, float dy, float dz, float tmax_obj) {
  const V3 o = {ox, oy, oz}, d = {dx, dy, dz};
  switch (shape) {
    case kShapeSphere: return sphere_t(o, d, kTMin, tmax_obj);
    case kShapeTriangle: {
      const float* q = tri_attr + (size_t)data * 24;
      return tri_t(ld3(q), ld3(q + 3), ld3(q + 6), o, d, kTMin, tmax_obj);
    }
    case kShapeRectangle: return rect_t(rects + (size_t)data * 16, o, d, kTMin, tmax_obj);
    case kShapePlane: return plane_t(o, d, kTMin, tmax_obj);
    default: return kRecords ? record_shape_t(shape, shapes + data, o, d, kTMin, tmax_obj) : -1.0f;
  }
}
template <bool kRecords>
DFC_D float prim_t(const SceneView& S, const DPrim& pr, const ObjRay& r, float tmax_obj) {
  return prim_t_v<kRecords>(S.tri_attr, S.rects, S.shapes, pr.shape, pr.data, r.o.x, r.o.y, r.o.z, r.d.x, r.d.y, r.d.z, tmax_obj);
}

// Conservative world-space rejection of a top-level item by its bounding
// sphere (centre, radius): false only when the ray line passes outside the
// sphere by a clear margin, or the whole sphere lies beyond the current best.
DFC_D bool sphere_may_hit(float4 bs, V3 o, V3 d, float best) {
  const float ox = bs.x - o.x, oy = bs.y - o.y, oz = bs.z - o.z;
  const float tca = ox * d.x + oy * d.y + oz * d.z;
  const float oc2 = ox * ox + oy * oy + oz * oz;
  const float d2 = oc2 - tca * tca;
  const float r2 = bs.w * bs.w;
  if (d2 > r2 * 1.001f + 1.0e-5f * oc2 + 1.0e-12f) return false;
  if (tca - bs.w * 1.001f > best * 1.0001f + 1.0e-6f * fabsf(tca)) return false;
  return true;
}

// Three-operand min and max (one instruction each on sm_100).  Like fminf and
// fmaxf they return the other operands' extreme when one operand is NaN.
DFC_D float fmin3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
DFC_D float fmax3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// 4 child slab tests of one node; returns a hit mask and the entry distances.
// (ox, oy, oz) = -origin * inverse direction, per axis.
DFC_D unsigned node_hits_oi(const BVH4Node* nodes, int ni, float ox, float oy, float oz, V3 inv, float tmin, float tmax, float tn[4]) {
  const float4* p = reinterpret_cast<const float4*>(nodes + ni);
  const float4 lx = __ldg(p + 0), ly = __ldg(p + 1), lz = __ldg(p + 2), hx = __ldg(p + 3), hy = __ldg(p + 4), hz = __ldg(p + 5);
  const float lxa[4] = {lx.x, lx.y, lx.z, lx.w}, lya[4] = {ly.x, ly.y, ly.z, ly.w}, lza[4] = {lz.x, lz.y, lz.z, lz.w};
  const float hxa[4] = {hx.x, hx.y, hx.z, hx.w}, hya[4] = {hy.x, hy.y, hy.z, hy.w}, hza[4] = {hz.x, hz.y, hz.z, hz.w};
  unsigned mask = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float x0 = fmaf(lxa[k], inv.x, ox), x1 = fmaf(hxa[k], inv.x, ox);
    float y0 = fmaf(lya[k], inv.y, oy), y1 = fmaf(hya[k], inv.y, oy);
    float z0 = fmaf(lza[k], inv.z, oz), z1 = fmaf(hza[k], inv.z, oz);
    float tnear = fmax3f(fminf(x0, x1), fminf(y0, y1), fmaxf(fminf(z0, z1), tmin));
    float tfar = fmin3f(fmaxf(x0, x1), fmaxf(y0, y1), fminf(fmaxf(z0, z1), tmax)) * 1.0000004f;
    tn[k] = tnear;
    if (tnear <= tfar && lxa[k] <= hxa[k]) mask |= 1u << k;
  }
  return mask;
}
DFC_D unsigned node_hits(const BVH4Node* nodes, int ni, V3 o, V3 inv, float tmin, float tmax, float tn[4]) {
  return node_hits_oi(nodes, ni, -o.x * inv.x, -o.y * inv.y, -o.z * inv.z, inv, tmin, tmax, tn);
}

// Closest (or any) hit in (kTMin, tmax) along a world ray.  stack points at
// this thread's column of the block's shared stack (stride kTraceBlock).
// Stack entries: >= 0 node index; -1 end of a bottom level (back to world
// space); <= -2 enter the bottom level of mesh primitive (-2 - entry).
template <bool kRecords>
DFC_D bool trace_ray(const SceneView& S, V3 o, V3 d, float tmax, bool kAny, Hit* out, int* stack, unsigned* overflow) {
  float best = tmax;
  bool found = false;
  // A ray with a non-finite origin or direction hits nothing in the reference
  // (every bounding-volume and shape test compares false against NaN); here a
  // NaN would pass every slab test (fmaxf drops NaN), so stop it up front.
  if (!isfinite(o.x + o.y + o.z + d.x + d.y + d.z)) { out->t = tmax; return false; }
  int sp = 0;
  if (S.tlas_root >= 0) stack[(sp++) * kTraceBlock] = S.tlas_root;
  for (int u = 0; u < S.unbounded_count; ++u) {
    const int pi = S.unbounded[u];
    const DPrim& pr = S.prims[pi];
    if (pr.shape == kShapeMesh) {  // entered before the top level (pushed last, popped first)
      if (sp < kStack) stack[(sp++) * kTraceBlock] = -2 - pi;
      else atomicAdd(overflow, 1u);
      continue;
    }
    ObjRay r = obj_ray(pr, o, d);
    float to = prim_t<kRecords>(S, pr, r, best * r.s);
    if (to > kTMin) {  // SurfaceIntersector3F.intersection: t > tMinimum
      float tw = to / r.s;
      if (tw < best) {
        best = tw; found = true; out->prim = pi; out->aux = pr.data; out->t_obj = to;
        if (kAny) { out->t = best; return true; }
      }
    }
  }
  if (sp == 0) { out->t = best; return found; }
  const V3 winv = safe_inv(d);
  bool in_blas = false;
  ObjRay br;
  br.s = 1.0f;
  int bprim = -1;
  float bbest = 0.0f;
  while (sp > 0) {
    const int e = stack[(--sp) * kTraceBlock];
    if (e == -1) {
      in_blas = false;
      best = fminf(best, bbest / br.s);
      continue;
    }
    if (e <= -2) {
      bprim = -2 - e;
      const DPrim& pm = S.prims[bprim];
      br = obj_ray(pm, o, d);
      bbest = best * br.s;
      in_blas = true;
      if (sp + 2 > kStack) { atomicAdd(overflow, 1u); in_blas = false; continue; }
      stack[(sp++) * kTraceBlock] = -1;
      stack[(sp++) * kTraceBlock] = pm.data;
      continue;
    }
    float tn[4];
    const unsigned mask = in_blas ? node_hits(S.nodes, e, br.o, br.inv, 0.0f, bbest, tn) : node_hits(S.nodes, e, o, winv, 0.0f, best, tn);
    if (!mask) continue;
    const int4 ch = __ldg(reinterpret_cast<const int4*>(S.nodes + e) + 6);  // stack entries (encode_node_entries)
    const int cha[4] = {ch.x, ch.y, ch.z, ch.w};
    int ent[4];
    float entt[4];
    int nent = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!(mask & (1u << k))) continue;
      const int c = cha[k];
      if (c >= 0) { ent[nent] = c; entt[nent] = tn[k]; ++nent; continue; }
      const int first = (int)(((unsigned)c & 0x3FFFFFFFu) >> 2), cnt = (c & 3) + 1;
      if (in_blas) {
        for (int j = 0; j < cnt; ++j) {
          const int ti = first + j;
          const float4* tp = reinterpret_cast<const float4*>(S.tri_pos) + 3 * ti;
          const float4 a = __ldg(tp), b = __ldg(tp + 1), cc = __ldg(tp + 2);
          const float t = tri_t(V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, V3{cc.x, cc.y, cc.z}, br.o, br.d, kTMin, bbest);
          if (t > kTMin && t < bbest) {
            bbest = t; found = true;
            out->prim = bprim; out->aux = __float_as_int(a.w); out->t_obj = t;
            if (kAny) { out->t = t / br.s; return true; }
          }
        }
      } else {
        for (int j = 0; j < cnt; ++j) {
          const int pi = S.tlas_items[first + j];
          const float4 bs = __ldg(reinterpret_cast<const float4*>(S.tlas_bound) + first + j);
          if (bs.w < 0.0f) {
            if (nent < 4) { ent[nent] = -2 - pi; entt[nent] = tn[k]; ++nent; }
            else if (sp < kStack) stack[(sp++) * kTraceBlock] = -2 - pi;
            else atomicAdd(overflow, 1u);
            continue;
          }
          if (!sphere_may_hit(bs, o, d, best)) continue;
          const DPrim& pr = S.prims[pi];
          ObjRay r = obj_ray(pr, o, d);
          const float to = prim_t<kRecords>(S, pr, r, best * r.s);
          if (to > kTMin) {  // SurfaceIntersector3F.intersection: t > tMinimum
            const float tw = to / r.s;
            if (tw < best) {
              best = tw; found = true; out->prim = pi; out->aux = pr.data; out->t_obj = to;
              if (kAny) { out->t = best; return true; }
            }
          }
        }
      }
    }
    // push far-to-near so that the nearest entry is popped first
    for (int x = 1; x < nent; ++x) {
      for (int y = x; y > 0 && entt[y - 1] < entt[y]; --y) {
        const float tt = entt[y]; entt[y] = entt[y - 1]; entt[y - 1] = tt;
        const int ii = ent[y]; ent[y] = ent[y - 1]; ent[y - 1] = ii;
      }
    }
    for (int x = 0; x < nent; ++x) {
      if (sp >= kStack) { atomicAdd(overflow, 1u); break; }
      stack[(sp++) * kTraceBlock] = ent[x];
    }
  }
  if (in_blas) best = fminf(best, bbest / br.s);
  out->t = best;
  return found;
}

}  // namespace

// ---- path state --------------------------------------------------------------
constexpr unsigned kAlive = kFlagAlive, kPendShadow = kFlagPendShadow, kPendMis = kFlagPendMis, kShadowAny = kFlagShadowAny,
                   kNoSample = kFlagNoSample;

// Stack entries (32 bits):
//   0x00000000 | node                 an interior node
//   0x80000000 | first << 2 | (n - 1) a leaf of n items starting at `first`
//   0xC0000000 | prim                 enter the bottom level of mesh primitive `prim`
//   0xFFFFFFFF                        end of a bottom level (back to world space)
constexpr unsigned kTagMask = 0xC0000000u, kTagLeaf = 0x80000000u, kTagMesh = 0xC0000000u, kEndBlas = 0xFFFFFFFFu;

// ---- persistent traversal with per-lane refill ---------------------------
// The same walk as trace_ray, held in registers across iterations so that a
// lane whose ray is done takes a new ray from the queue instead of idling
// until the slowest lane of its warp finishes (ray costs are heavy-tailed).
// Each round has a node phase and a leaf phase (the while-while loop of Aila
// and Laine, "Understanding the efficiency of ray traversal on GPUs", HPG
// 2009): lanes walk interior nodes until every lane of the warp holds a leaf
// (a lane that already holds one keeps walking nodes speculatively), then all
// lanes test their leaves together, one item per iteration, so node and leaf
// code do not interleave within a warp.
struct Trav {
  V3 o, d;          // world ray
  V3 co, cinv;      // origin and inverse direction in the current space (world, or a mesh's object space)
  float cbest;      // closest hit so far in the current space
  float wbest;      // world closest hit, saved while in a bottom level
  float s;          // length of the object-space direction before normalisation
  Shear sh;         // triangle shear of cd
  int sp, bprim;
  bool any, in_blas;
  int prim, aux;    // closest hit so far (prim -1: none)
  float t_obj;
};

template <bool kRecords>
DFC_D void trav_init(const SceneView& S, Trav& T, V3 o, V3 d, float tmax, bool any, int* stack, unsigned* overflow) {
  T.o = o; T.d = d; T.co = o; T.cbest = tmax; T.wbest = tmax; T.s = 1.0f;
  T.any = any; T.in_blas = false;
  T.sp = 0; T.bprim = -1;
  T.prim = -1; T.aux = -1; T.t_obj = 0.0f;
  if (!isfinite(o.x + o.y + o.z + d.x + d.y + d.z)) return;  // misses everything (see trace_ray)
  T.cinv = safe_inv(d);
  if (S.tlas_root >= 0) { stack[0] = S.tlas_root; T.sp = 1; }
  for (int u = 0; u < S.unbounded_count; ++u) {
    const int pi = S.unbounded[u];
    const DPrim& pr = S.prims[pi];
    if (pr.shape == kShapeMesh) {  // entered before the top level (pushed last, popped first)
      if (T.sp < kStack) stack[(T.sp++) * kTraceBlock] = (int)(kTagMesh | (unsigned)pi);
      else atomicAdd(overflow, 1u);
      continue;
    }
    ObjRay r = obj_ray(pr, o, d);
    const float to = prim_t<kRecords>(S, pr, r, T.cbest * r.s);
    if (to > kTMin) {
      const float tw = to / r.s;
      if (tw < T.cbest) {
        T.cbest = tw; T.prim = pi; T.aux = pr.data; T.t_obj = to;
        if (any) { T.sp = 0; return; }
      }
    }
  }
}


#define DFC_CSWAP(ta, ea, tb, eb) \
  if (tb < ta) { const float tt_ = ta; ta = tb; tb = tt_; const unsigned ee_ = ea; ea = eb; eb = ee_; }

// One step of the node phase.  Pops the top entry: an interior node pushes its
// hit children far-to-near, a leaf is taken as this lane's pending leaf, and
// the bottom-level markers switch the ray's space.  A lane that already holds
// a leaf only walks interior nodes (the leaf must be tested in the space it
// came from); it returns true when the top entry is anything else.
DFC_D bool node_step(const SceneView& S, Trav& T, int* stack, unsigned* overflow, int& lf_first, int& lf_cnt) {
  const unsigned e = (unsigned)stack[(T.sp - 1) * kTraceBlock];
  const unsigned tag = e & kTagMask;
  if (tag != 0u && lf_cnt > 0) return true;
  --T.sp;
  if (tag == 0u) {
    float tn[4];
    const unsigned mask = node_hits(S.nodes, (int)e, T.co, T.cinv, 0.0f, T.cbest, tn);
    if (!mask) return false;
    // the node's children, already in stack-entry form (encode_node_entries)
    const int4 ch = __ldg(reinterpret_cast<const int4*>(S.nodes + e) + 6);
    const float inf = __int_as_float(0x7f800000);
    float t0 = (mask & 1u) ? tn[0] : inf, t1 = (mask & 2u) ? tn[1] : inf, t2 = (mask & 4u) ? tn[2] : inf, t3 = (mask & 8u) ? tn[3] : inf;
    unsigned e0 = (unsigned)ch.x, e1 = (unsigned)ch.y, e2 = (unsigned)ch.z, e3 = (unsigned)ch.w;
    DFC_CSWAP(t0, e0, t1, e1);
    DFC_CSWAP(t2, e2, t3, e3);
    DFC_CSWAP(t0, e0, t2, e2);
    DFC_CSWAP(t1, e1, t3, e3);
    DFC_CSWAP(t1, e1, t2, e2);
    const int n = __popc(mask);
    if (T.sp + n > kStack) { atomicAdd(overflow, 1u); return false; }
    // ascending t0 <= t1 <= t2 <= t3 (misses last as +inf): push the n hits far first
    if (n > 3) stack[(T.sp++) * kTraceBlock] = (int)e3;
    if (n > 2) stack[(T.sp++) * kTraceBlock] = (int)e2;
    if (n > 1) stack[(T.sp++) * kTraceBlock] = (int)e1;
    // the nearest child, when it is a leaf, becomes this lane's pending leaf at
    // once (it would be the next entry popped), saving the node step that pops it
    if ((e0 & kTagMask) == kTagLeaf && lf_cnt == 0) {
      lf_first = (int)((e0 & ~kTagMask) >> 2);
      lf_cnt = (int)(e0 & 3u) + 1;
      return false;
    }
    stack[(T.sp++) * kTraceBlock] = (int)e0;
    return false;
  }
  if (tag == kTagLeaf) {
    lf_first = (int)((e & ~kTagMask) >> 2);
    lf_cnt = (int)(e & 3u) + 1;
    return false;
  }
  if (e == kEndBlas) {
    T.in_blas = false;
    T.cbest = fminf(T.wbest, T.cbest / T.s);
    T.co = T.o;
    T.cinv = safe_inv(T.d);
      T.s = 1.0f;
    return false;
  }
  // enter a mesh's bottom level
  if (T.sp + 2 > kStack) { atomicAdd(overflow, 1u); return false; }
  T.bprim = (int)(e & ~kTagMask);
  const DPrim& pm = S.prims[T.bprim];
  const ObjRay r = obj_ray(pm, T.o, T.d);
  T.co = r.o; T.cinv = r.inv; T.s = r.s;
  T.wbest = T.cbest;
  T.cbest = T.wbest * r.s;
  T.sh = make_shear(r.d);
  T.in_blas = true;
  stack[(T.sp++) * kTraceBlock] = (int)kEndBlas;
  stack[(T.sp++) * kTraceBlock] = pm.data;
  return false;
}

// One item of this lane's pending leaf: a triangle of the current bottom
// level, or a top-level item (a mesh is queued for its bottom level).
template <bool kRecords>
DFC_D void leaf_step(const SceneView& S, Trav& T, int* stack, unsigned* overflow, int& lf_first, int& lf_cnt) {
  const int i = lf_first++;
  --lf_cnt;
  if (T.in_blas) {
    const float4* tp = reinterpret_cast<const float4*>(S.tri_pos) + 3 * i;
    const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    const float t = tri_t_sheared(a, b, c, T.co, T.sh, kTMin, T.cbest);
    if (t > kTMin && t < T.cbest) {
      T.cbest = t;
      T.prim = T.bprim; T.aux = __float_as_int(a.w); T.t_obj = t;
      if (T.any) { T.cbest = t / T.s; T.in_blas = false; T.sp = 0; lf_cnt = 0; }
    }
    return;
  }
  const int pi = S.tlas_items[i];
  const float4 bs = __ldg(reinterpret_cast<const float4*>(S.tlas_bound) + i);
  if (bs.w < 0.0f) {  // a mesh: enter its bottom level in a later node phase
    if (T.sp < kStack) stack[(T.sp++) * kTraceBlock] = (int)(kTagMesh | (unsigned)pi);
    else atomicAdd(overflow, 1u);
    return;
  }
  if (!sphere_may_hit(bs, T.o, T.d, T.cbest)) return;
  const DPrim& pr = S.prims[pi];
  ObjRay r = obj_ray(pr, T.o, T.d);
  const float to = prim_t<kRecords>(S, pr, r, T.cbest * r.s);
  if (to > kTMin) {
    const float tw = to / r.s;
    if (tw < T.cbest) {
      T.cbest = tw; T.prim = pi; T.aux = pr.data; T.t_obj = to;
      if (T.any) { T.sp = 0; lf_cnt = 0; }
    }
  }
}

constexpr unsigned kNoRay = 0xffffffffu;
#ifndef DFC_REFILL
#define DFC_REFILL 8
#endif
constexpr int kRefill = DFC_REFILL;  // refill a warp's idle lanes once this many are idle
// Node-phase bound and resident blocks, measured on the 2.1M-triangle benchmark
// scene with device-built hierarchies and path-ordered ray lists: 4, 6, 8, 16, 32
// steps gave 132.2, 134.1, 138.6, 133.8, 132.1M paths/s; 7 blocks (72 registers)
// added 0.5% over 6.
#ifndef DFC_NODE_STEPS
#define DFC_NODE_STEPS 8
#endif
#ifndef DFC_SPECULATE
#define DFC_SPECULATE 0  // speculative node steps measured 1.1% slower on the benchmark scene
#endif
constexpr int kNodeSteps = DFC_NODE_STEPS;  // bound of one node phase (the warp then tests its leaves and refills)
constexpr bool kSpeculate = DFC_SPECULATE != 0;  // lanes holding a leaf keep walking interior nodes

// Every vote below is taken by all 32 lanes at the same point of the loop
// (lanes without work only skip the work), so full masks are exact.
#ifndef DFC_TRACE_MIN_BLOCKS
#define DFC_TRACE_MIN_BLOCKS 7
#endif
// The scene a kernel works on: the launch's own (per-job renderer) or, in
// the batch engine, the table entry of the ray's or path's job.
template <bool kMulti, typename Args>
DFC_D const SceneView& scene_at(const Args& a, int si) {
  if constexpr (kMulti) return a.scenes[si];
  else return a.scene;
}

template <bool kRecords, bool kMulti>
__device__ __forceinline__ void trace_rays(const TraceArgs& a) {
  __shared__ int stack_smem[kStack * kTraceBlock];
  int* stack = stack_smem + threadIdx.x;
  const unsigned n = *a.ray_count;
  const unsigned lane = threadIdx.x & 31u;
  Trav T;
  T.sp = 0;
  unsigned cur = kNoRay;
  unsigned slot = 0;
  int si = 0;  // scene of this lane's ray (batch engine)
  int lf_first = 0, lf_cnt = 0;
  bool pool_empty = false;  // warp-uniform
  while (true) {
    const bool idle = cur == kNoRay;
    const unsigned idle_mask = __ballot_sync(0xffffffffu, idle);
    if (!pool_empty && __popc(idle_mask) >= kRefill) {
      const int leader = __ffs(idle_mask) - 1;
      unsigned base = 0;
      if ((int)lane == leader) base = atomicAdd(a.fetch, (unsigned)__popc(idle_mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (base + (unsigned)__popc(idle_mask) >= n) pool_empty = true;
      if (idle) {
        const unsigned i = base + (unsigned)__popc(idle_mask & ((1u << lane) - 1u));
        if (i < n) {
          cur = i;
          const unsigned ref = a.ray_list[i];
          const unsigned p = ref >> 3, type = ref & 3u;
          slot = type * a.paths + p;
          if constexpr (kMulti) si = a.jobs[a.slot_job[p]].scene;
          const float4 ro = a.ray_o[slot], rd = a.ray_d[slot];
          trav_init<kRecords>(scene_at<kMulti>(a, si), T, V3{ro.x, ro.y, ro.z}, V3{rd.x, rd.y, rd.z}, rd.w, (ref & 4u) != 0u, stack, a.overflow);
          lf_cnt = 0;
        }
      }
    }
    const bool act = cur != kNoRay;
    if (pool_empty && !__any_sync(0xffffffffu, act)) break;
    // node phase
    bool blocked = false;
    for (int k = 0; k < kNodeSteps; ++k) {
      const bool searching = act && T.sp > 0 && lf_cnt == 0;
      if (!__any_sync(0xffffffffu, searching)) break;
      if (kSpeculate ? (act && T.sp > 0 && !blocked) : searching)
        blocked = node_step(scene_at<kMulti>(a, si), T, stack, a.overflow, lf_first, lf_cnt);
    }
    // leaf phase
    while (__any_sync(0xffffffffu, lf_cnt > 0)) {
      if (lf_cnt > 0) leaf_step<kRecords>(scene_at<kMulti>(a, si), T, stack, a.overflow, lf_first, lf_cnt);
    }
    if (act && T.sp == 0) {
      a.hits[slot] = make_float4(T.cbest, __int_as_float(T.prim), __int_as_float(T.aux), T.t_obj);
      cur = kNoRay;
    }
  }
}

}  // namespace dfc
