// Wavefront kernels of the B200 render path.
//
// One render pass (renderer/gpu/AbstractGPURenderer.java:231-297: one sample
// per pixel) runs as
//   raygen -> [trace -> shade] x bounces -> final shade
// over fixed per-path slots.  A path owns three ray slots (extension, shadow,
// MIS) and a state record; shade appends the rays it spawns to a compacted
// ray list and the paths that still have work to a compacted work list, both
// with one atomic per warp (ballot + popc).  The trace kernel is a persistent
// grid-stride loop over the ray list walking the two-level 4-wide BVH with a
// per-thread stack in shared memory.  The path semantics are those of
// scene/Scene.java:451-619 (radiancePathTracer) with doEstimateDirectLight
// (:1530) split into a shadow ray and a MIS ray whose results are folded in
// by the next shade step.
#include <cuda_runtime.h>

#include "dfc_device.cuh"
#include "dfc_kernels.h"
#include "dfc_shapes.cuh"
#include "dfc_texture.cuh"

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
  r.inv = V3{1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z};
  return r;
}

// Object-space test of one analytic primitive; returns the object distance or -1.
// Out of line: called at top-level leaves only, it keeps the traversal loop small.
// kRecords adds disk ... torus (the double-precision torus solve enlarges the
// call tree enough to cost the traversal loop registers, so scenes without
// those shapes run the instantiation without them).
template <bool kRecords>
__device__ __noinline__ float prim_t(const SceneView& S, const DPrim& pr, const ObjRay& r, float tmax_obj) {
  switch (pr.shape) {
    case kShapeSphere: return sphere_t(r.o, r.d, kTMin, tmax_obj);
    case kShapeTriangle: {
      const float* q = S.tri_attr + (size_t)pr.data * 24;
      return tri_t(ld3(q), ld3(q + 3), ld3(q + 6), r.o, r.d, kTMin, tmax_obj);
    }
    case kShapeRectangle: return rect_t(S.rects + (size_t)pr.data * 16, r.o, r.d, kTMin, tmax_obj);
    case kShapePlane: return plane_t(r.o, r.d, kTMin, tmax_obj);
    default: return kRecords ? record_shape_t(pr.shape, S.shapes + pr.data, r.o, r.d, kTMin, tmax_obj) : -1.0f;
  }
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

// 4 child slab tests of one node; returns a hit mask and the entry distances.
DFC_D unsigned node_hits(const BVH4Node* nodes, int ni, V3 o, V3 inv, float tmin, float tmax, float tn[4]) {
  const float4* p = reinterpret_cast<const float4*>(nodes + ni);
  const float4 lx = __ldg(p + 0), ly = __ldg(p + 1), lz = __ldg(p + 2), hx = __ldg(p + 3), hy = __ldg(p + 4), hz = __ldg(p + 5);
  const float ox = -o.x * inv.x, oy = -o.y * inv.y, oz = -o.z * inv.z;
  const float lxa[4] = {lx.x, lx.y, lx.z, lx.w}, lya[4] = {ly.x, ly.y, ly.z, ly.w}, lza[4] = {lz.x, lz.y, lz.z, lz.w};
  const float hxa[4] = {hx.x, hx.y, hx.z, hx.w}, hya[4] = {hy.x, hy.y, hy.z, hy.w}, hza[4] = {hz.x, hz.y, hz.z, hz.w};
  unsigned mask = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float x0 = fmaf(lxa[k], inv.x, ox), x1 = fmaf(hxa[k], inv.x, ox);
    float y0 = fmaf(lya[k], inv.y, oy), y1 = fmaf(hya[k], inv.y, oy);
    float z0 = fmaf(lza[k], inv.z, oz), z1 = fmaf(hza[k], inv.z, oz);
    float tnear = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
    float tfar = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax)) * 1.0000004f;
    tn[k] = tnear;
    if (tnear <= tfar && lxa[k] <= hxa[k]) mask |= 1u << k;
  }
  return mask;
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
  for (int u = 0; u < S.unbounded_count; ++u) {
    const int pi = S.unbounded[u];
    const DPrim& pr = S.prims[pi];
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
  if (S.tlas_root < 0) { out->t = best; return found; }
  const V3 winv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  int sp = 0;
  stack[(sp++) * kTraceBlock] = S.tlas_root;
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
    const int4* cp = reinterpret_cast<const int4*>(S.nodes + e) + 6;
    const int4 ch = __ldg(cp), cn = __ldg(cp + 1);
    const int cha[4] = {ch.x, ch.y, ch.z, ch.w}, cna[4] = {cn.x, cn.y, cn.z, cn.w};
    int ent[4];
    float entt[4];
    int nent = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!(mask & (1u << k))) continue;
      const int c = cha[k];
      if (c >= 0) { ent[nent] = c; entt[nent] = tn[k]; ++nent; continue; }
      const int first = ~c, cnt = cna[k];
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
DFC_D void trav_init(const SceneView& S, Trav& T, V3 o, V3 d, float tmax, bool any, int* stack) {
  T.o = o; T.d = d; T.co = o; T.cbest = tmax; T.wbest = tmax; T.s = 1.0f;
  T.any = any; T.in_blas = false;
  T.sp = 0; T.bprim = -1;
  T.prim = -1; T.aux = -1; T.t_obj = 0.0f;
  if (!isfinite(o.x + o.y + o.z + d.x + d.y + d.z)) return;  // misses everything (see trace_ray)
  for (int u = 0; u < S.unbounded_count; ++u) {
    const int pi = S.unbounded[u];
    const DPrim& pr = S.prims[pi];
    ObjRay r = obj_ray(pr, o, d);
    const float to = prim_t<kRecords>(S, pr, r, T.cbest * r.s);
    if (to > kTMin) {
      const float tw = to / r.s;
      if (tw < T.cbest) {
        T.cbest = tw; T.prim = pi; T.aux = pr.data; T.t_obj = to;
        if (any) return;
      }
    }
  }
  T.cinv = V3{1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  if (S.tlas_root >= 0) { stack[0] = S.tlas_root; T.sp = 1; }
}

// Stack entries (32 bits):
//   0x00000000 | node                 an interior node
//   0x80000000 | first << 2 | (n - 1) a leaf of n items starting at `first`
//   0xC0000000 | prim                 enter the bottom level of mesh primitive `prim`
//   0xFFFFFFFF                        end of a bottom level (back to world space)
constexpr unsigned kTagMask = 0xC0000000u, kTagLeaf = 0x80000000u, kTagMesh = 0xC0000000u, kEndBlas = 0xFFFFFFFFu;

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
    const int4* cp = reinterpret_cast<const int4*>(S.nodes + e) + 6;
    const int4 ch = __ldg(cp), cn = __ldg(cp + 1);
    const float inf = __int_as_float(0x7f800000);
    auto entry = [](int c, int n) -> unsigned { return c >= 0 ? (unsigned)c : (kTagLeaf | ((unsigned)(~c) << 2) | (unsigned)(n - 1)); };
    float t0 = (mask & 1u) ? tn[0] : inf, t1 = (mask & 2u) ? tn[1] : inf, t2 = (mask & 4u) ? tn[2] : inf, t3 = (mask & 8u) ? tn[3] : inf;
    unsigned e0 = entry(ch.x, cn.x), e1 = entry(ch.y, cn.y), e2 = entry(ch.z, cn.z), e3 = entry(ch.w, cn.w);
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
    T.cinv = V3{1.0f / T.d.x, 1.0f / T.d.y, 1.0f / T.d.z};
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
constexpr int kRefill = 8;        // refill a warp's idle lanes once this many are idle
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
          trav_init<kRecords>(scene_at<kMulti>(a, si), T, V3{ro.x, ro.y, ro.z}, V3{rd.x, rd.y, rd.z}, rd.w, (ref & 4u) != 0u, stack);
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

__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace(TraceArgs a) { trace_rays<false, false>(a); }
__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace_records(TraceArgs a) { trace_rays<true, false>(a); }
__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace_batch(TraceArgs a) { trace_rays<false, true>(a); }
__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace_batch_records(TraceArgs a) { trace_rays<true, true>(a); }

__global__ void k_raygen(RaygenArgs a) {
  // No early return: every lane of the warp takes part in warp_append's ballot.
  const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in_range = p < a.paths;
  bool ok = false;
  if (in_range) {
    const unsigned pix = p % a.pixels;
    const unsigned sample = a.sample_base + p / a.pixels;
    const unsigned x = pix % a.width, y = pix / a.width;
    const uint32_t key = rng_path_key(a.seed, pix, sample);
    V3 o = {0, 0, 0}, d = {0, 0, 1};
    ok = camera_ray(a.scene.camera, (float)x, (float)y, rng_uniform(key, kDimPixelX), rng_uniform(key, kDimPixelY),
                    rng_uniform(key, kDimLensU), rng_uniform(key, kDimLensV), &o, &d);
    a.beta[p] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);  // w: etaScale
    a.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    a.meta[p] = make_uint4(pix, key, 0u, ok ? kAlive : kNoSample);  // z: bounce | dimension step << 16
    a.ray_o[p] = make_float4(o.x, o.y, o.z, kTMin);
    a.ray_d[p] = make_float4(d.x, d.y, d.z, kFltMax);
    // a path without a camera ray (fisheye outside the disc) still goes through
    // shade once to be retired; it traces nothing and adds no film sample.
    a.work_list[p] = p;
  }
  const unsigned slot = warp_append(a.ray_count, ok);
  if (ok) a.ray_list[slot] = p << 3;
  if (p == 0) *a.work_count = a.paths;
}

template <bool kRecords>
DFC_D V3 surface_of(const SceneView& S, const DPrim& pr, int aux, V3 o, V3 d, float t_obj, Surface* sf) {
  // the object ray as the intersector saw it
  V3 oo = o, od = d;
  if (!pr.identity) {
    oo = xf_point(pr.w2o, o);
    od = normalize(xf_vec(pr.w2o, d));
  }
  switch (pr.shape) {
    case kShapeSphere: *sf = sphere_surface(oo, od, t_obj); break;
    case kShapeRectangle: *sf = rect_surface(S.rects + (size_t)pr.data * 16, oo, od, t_obj); break;
    case kShapePlane: *sf = plane_surface(oo, od, t_obj); break;
    case kShapeTriangle: case kShapeMesh: *sf = triangle_surface(S.tri_attr + (size_t)aux * 24, oo, od, t_obj); break;
    default:
      if (kRecords) *sf = record_shape_surface(pr.shape, S.shapes + pr.data, oo, od, t_obj);
      break;
  }
  surface_to_world(pr, *sf);
  return sf->p;
}

// World distance of a hit as SurfaceIntersection3F.transform (geometry/
// SurfaceIntersection3F.java:389) forms it: from the object ray's origin mapped
// back to world space to the world hit point.
DFC_D float world_t(const DPrim& pr, V3 o, const Surface& sf) {
  if (pr.identity) return len(sf.p - o);
  return len(sf.p - xf_point(pr.o2w, xf_point(pr.w2o, o)));
}

// Area-light pdf for a direction (Shape3F.evaluateProbabilityDensityFunction and
// the Sphere3F override), in the light's object space.
DFC_D float area_light_pdf(const SceneView& S, const DLight& lt, V3 p, V3 wi) {
  V3 ref = xf_point(lt.w2o, p);
  V3 w = normalize(xf_vec(lt.w2o, wi));
  if (lt.shape == kShapeTriangle) {
    const float* q = S.tri_attr + (size_t)lt.shape_data * 24;
    float t = tri_t(ld3(q), ld3(q + 3), ld3(q + 6), ref, w, 0.001f, kFltMax);
    if (!(t > 0.0f)) return 0.0f;
    Surface s = triangle_surface(q, ref, w, t);
    V3 dp = s.p - ref;
    float pd = dot(dp, dp) / (fabsf(dot(normalize(s.s.w), -w)) * lt.area);
    return (isinf(pd) || isnan(pd)) ? 0.0f : pd;
  }
  if (lt.shape == kShapeSphere) {
    float t = sphere_t(ref, w, 0.001f, kFltMax);
    if (!(t > 0.0f)) return 0.0f;
    Surface s = sphere_surface(ref, w, t);
    V3 dp = s.p - ref;
    float pd = dot(dp, dp) / fabsf(dot(s.s.w, -w)) * (4.0f * kPi);
    return (isinf(pd) || isnan(pd)) ? 0.0f : pd;
  }
  return 0.0f;
}

DFC_D void film_add_to(float4* film_sum, float4* film_sq, unsigned pix, V3 L) {
  if (!(isfinite(L.x) && isfinite(L.y) && isfinite(L.z))) return;  // AbstractCPURenderer.java:231
  if (luminance(L) < -1.0e-5f) return;
  float* f = reinterpret_cast<float*>(film_sum + pix);
  atomicAdd(f + 0, L.x); atomicAdd(f + 1, L.y); atomicAdd(f + 2, L.z); atomicAdd(f + 3, 1.0f);
  float* g = reinterpret_cast<float*>(film_sq + pix);
  atomicAdd(g + 0, L.x * L.x); atomicAdd(g + 1, L.y * L.y); atomicAdd(g + 2, L.z * L.z);
}
// image/PixelImageF.java:569 filmAddColorXYZ (GaussianFilter2F(2, 2, 2) table):
// the sample at film position (x + jitter x, y + jitter y) adds its XYZ, weighted
// by the filter table entry, and the weight to every pixel within radius 2.
DFC_D void film_splat(const ShadeArgs& a, unsigned pix, uint32_t key, V3 L) {
  if (!(isfinite(L.x) && isfinite(L.y) && isfinite(L.z))) return;  // AbstractCPURenderer.java:231
  if (luminance(L) < -1.0e-5f) return;
  const float* T = a.pixel_film;
  const float* m = T + kFilmTable * kFilmTable;  // column-major sRGB -> XYZ (ColorSpaceF)
  const V3 X = {m[0] * L.x + m[3] * L.y + m[6] * L.z, m[1] * L.x + m[4] * L.y + m[7] * L.z, m[2] * L.x + m[5] * L.y + m[8] * L.z};
  const unsigned W = a.width, H = a.height;
  const float dx = (float)(pix % W) + rng_uniform(key, kDimPixelX) - 0.5f;
  const float dy = (float)(pix / W) + rng_uniform(key, kDimPixelY) - 0.5f;
  const int x0 = (int)fmaxf(ceilf(dx - 2.0f), 0.0f), x1 = (int)fminf(floorf(dx + 2.0f), (float)(W - 1));
  const int y0 = (int)fmaxf(ceilf(dy - 2.0f), 0.0f), y1 = (int)fminf(floorf(dy + 2.0f), (float)(H - 1));
  for (int fy = y0; fy <= y1; ++fy) {
    const int oy = min((int)floorf(fabsf((fy - dy) * 0.5f * 16.0f)), kFilmTable - 1);
    for (int fx = x0; fx <= x1; ++fx) {
      const int ox = min((int)floorf(fabsf((fx - dx) * 0.5f * 16.0f)), kFilmTable - 1);
      const float w = T[oy * kFilmTable + ox];
      float* f = reinterpret_cast<float*>(a.film_sum + (size_t)fy * W + fx);
      atomicAdd(f + 0, X.x * w); atomicAdd(f + 1, X.y * w); atomicAdd(f + 2, X.z * w); atomicAdd(f + 3, w);
    }
  }
}
DFC_D void film_add(const ShadeArgs& a, unsigned pix, uint32_t key, V3 L) {
  if (a.pixel_film) film_splat(a, pix, key, L);
  else film_add_to(a.film_sum, a.film_sq, pix, L);
}

// One shade step of the path tracer for every path on the work list.  In
// the batch engine (kMulti) the scene, film and bounce limits come from the
// path's job, a path ends at its own step max_bounce + 3 (the step count of
// a render pass of the per-job renderer), and a retired path's slot goes back
// on the free stack.
template <bool kRecords, bool kMulti, bool kTextured = false>
__device__ __forceinline__ void shade_path(const ShadeArgs& a) {
  const unsigned n = *a.work_count;
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const unsigned i = base + threadIdx.x;
    bool spawn_ext = false, spawn_shadow = false, spawn_mis = false, keep = false, shadow_any = false, retire = false;
    unsigned p = 0, job = 0;
    if (i < n) {
      p = a.work_list[i];
      const DJob* J = nullptr;
      if constexpr (kMulti) { job = a.slot_job[p]; J = a.jobs + job; }
      const SceneView& S = scene_at<kMulti>(a, kMulti ? J->scene : 0);
      const int max_bounce = kMulti ? J->max_bounce : a.max_bounce;
      const int min_rr = kMulti ? J->min_rr : a.min_rr;
      uint4 meta = a.meta[p];
      float4 b4 = a.beta[p];
      float4 l4 = a.radiance[p];
      V3 beta = {b4.x, b4.y, b4.z}, L = {l4.x, l4.y, l4.z};
      float eta_scale = b4.w;
      unsigned flags = meta.w;
      int bounce = (int)(meta.z & 0xffffu), dimb = (int)(meta.z >> 16);
      const uint32_t key = meta.y;
      const size_t P = a.paths;
      // 1. fold in the light rays of the previous step
      if (flags & kPendShadow) {
        const float4 hs = a.hits[P + p];
        const float4 c = a.pend_shadow[p];
        const int hp = __float_as_int(hs.y);
        bool vis;
        if (flags & kShadowAny) vis = hp < 0;
        else vis = hp >= 0 && S.prims[hp].light == __float_as_int(c.w);
        if (vis) L = L + V3{c.x, c.y, c.z};
      }
      if (flags & kPendMis) {
        const float4 hm = a.hits[2 * P + p];
        const float4 c = a.pend_mis[p];
        const int li = __float_as_int(c.w);
        const int hp = __float_as_int(hm.y);
        const float4 md = a.ray_d[2 * P + p];
        const V3 wi = {md.x, md.y, md.z};
        if (hp >= 0) {
          const DPrim& hpr = S.prims[hp];
          if (hpr.light == li) {
            const DLight& lt = S.lights[li];
            const float4 mo = a.ray_o[2 * P + p];
            Surface s;
            surface_of<kRecords>(S, hpr, __float_as_int(hm.z), V3{mo.x, mo.y, mo.z}, wi, hm.w, &s);
            if (lt.two_sided || dot(s.s.w, -wi) > 0.0f) L = L + mul(V3{c.x, c.y, c.z}, ld3(lt.radiance));
          }
        } else {
          V3 Le = light_Le_miss(S, S.lights[li], wi);
          L = L + mul(V3{c.x, c.y, c.z}, Le);
        }
      }
      flags &= ~(kPendShadow | kPendMis | kShadowAny);
      bool alive = (flags & kAlive) != 0u;
      const int step = (int)l4.w;  // shade steps this path has had
      const bool last_step = kMulti ? step >= max_bounce + 3 : a.last_step != 0;
      if (alive) {
        const float4 h = a.hits[p];
        const float4 ro = a.ray_o[p], rd = a.ray_d[p];
        const V3 ray_o = {ro.x, ro.y, ro.z}, ray_d = {rd.x, rd.y, rd.z};
        const int hp = __float_as_int(h.y);
        const bool spec = (flags & kFlagSpecular) != 0u;
        const bool rec = !kMulti && a.record_primary && bounce == 0 && dimb == 0 && p < a.pixels;
        if (rec && hp < 0) { a.primary_prim[p] = -1; a.primary_t[p] = __int_as_float(0x7fc00000); }
        if (kMulti && J->kind != kJobPathTracing) {
          // ray-casting and depth-camera jobs of the engine end at their camera ray, shaded as k_shade_primary does
          if (hp < 0) {
            if (J->kind == kJobRayCasting)
              for (int k = 0; k < S.light_count; ++k) L = L + light_Le_miss(S, S.lights[k], ray_d);  // Scene.java:675
          } else {
            Surface sf;
            surface_of<kRecords>(S, S.prims[hp], __float_as_int(h.z), ray_o, ray_d, h.w, &sf);
            if (J->kind == kJobRayCasting) {
              const float c = fabsf(dot(sf.s.w, ray_d)) * 0.5f;
              L = V3{c, c, c};
            } else {  // Scene.java:327 radianceDepthCamera
              const V3 dd = sf.p - ray_o;
              const float in = clampf(1.0f / (dot(dd, dd) * 0.5f), 0.0f, 1.0f);
              L = V3{in, in, in};
            }
          }
          alive = false;
        } else if (hp < 0) {
          if (bounce == 0 && !kMulti && a.preview) L = {1, 1, 1};
          else if (bounce == 0 || spec) {
            for (int k = 0; k < S.light_count; ++k) L = L + mul(beta, light_Le_miss(S, S.lights[k], ray_d));
          }
          alive = false;
        } else {
          const DPrim& pr = S.prims[hp];
          Surface sf;
          surface_of<kRecords>(S, pr, __float_as_int(h.z), ray_o, ray_d, h.w, &sf);
          // SurfaceIntersection3F.transform: t = |origin - world point|
          if (rec) { a.primary_prim[p] = hp; a.primary_t[p] = world_t(pr, ray_o, sf); }
          const V3 wo = -ray_d;
          if (bounce == 0 || spec) {
            V3 Le;
            if (pr.light >= 0) {
              const DLight& lt = S.lights[pr.light];
              Le = (lt.two_sided || dot(sf.s.w, wo) > 0.0f) ? ld3(lt.radiance) : V3{0, 0, 0};
            } else if constexpr (kTextured) {
              Le = material_Le(S, pr, ray_d, sf);
            } else {
              Le = ld3(S.materials[pr.material].emission);
            }
            L = L + mul(beta, Le);
          }
          if (bounce >= max_bounce) {
            alive = false;
          } else {
            const DMaterial& m = S.materials[pr.material];
            const float u_mat = rng_uniform(key, bounce_dim(dimb, kDimMaterial));
            Bsdf B;
            bool built;
            // textured and composite materials only occur in scenes shaded by the kTextured variants
            if constexpr (kTextured) built = m.kind < kMatTextured ? build_bsdf(m, sf, ray_d, u_mat, &B) : textured_bsdf(S, pr, ray_d, u_mat, true, &sf, &B);
            else built = build_bsdf(m, sf, ray_d, u_mat, &B);
            if (!built) {
              // Scene.java:494: no BSDF, continue straight through without counting a bounce
              a.ray_o[p] = make_float4(sf.p.x, sf.p.y, sf.p.z, kTMin);
              a.ray_d[p] = make_float4(ray_d.x, ray_d.y, ray_d.z, kFltMax);
              spawn_ext = true;
              ++dimb;
            } else {
              const V3 ns = sf.s.w;
              if (bsdf_nonspec(B) > 0 && S.light_count > 0) {
                const int nl = S.light_count;
                const int li = min((int)(rng_uniform(key, bounce_dim(dimb, kDimLightPick)) * nl), nl - 1);
                const DLight& lt = S.lights[li];
                const float lscale = (float)nl;  // Color3F.divide(x, 1 / lightCount)
                LightS ls;
                const bool have = light_sample(S, lt, sf, rng_uniform(key, bounce_dim(dimb, kDimLightSampleU)),
                                               rng_uniform(key, bounce_dim(dimb, kDimLightSampleV)),
                                               rng_uniform(key, bounce_dim(dimb, kDimSunPick)), &ls);
                const bool delta = light_is_delta(lt.type);
                if (have && !is_black(ls.L) && ls.pdf > 0.0f) {
                  V3 f = bsdf_f(B, kAllButSpecular, ls.wi) * fabsf(dot(ls.wi, ns));
                  if (!is_black(f)) {
                    float w = 1.0f;
                    if (!delta) w = (ls.pdf * ls.pdf) / (ls.pdf * ls.pdf + bsdf_pdf(B, kAllButSpecular, ls.wi) * bsdf_pdf(B, kAllButSpecular, ls.wi));
                    V3 c = mul(beta, mul(f, ls.L) * (w / ls.pdf)) * lscale;
                    V3 toL = ls.p - sf.p;
                    float dist = len(toL);
                    V3 sd = normalize(toL);
                    a.ray_o[P + p] = make_float4(sf.p.x, sf.p.y, sf.p.z, kTMin);
                    a.ray_d[P + p] = make_float4(sd.x, sd.y, sd.z, fabsf(dist) + 0.001f);
                    a.pend_shadow[p] = make_float4(c.x, c.y, c.z, __int_as_float(li));
                    shadow_any = lt.type != kLightDiffuseArea;
                    flags |= kPendShadow | (shadow_any ? kShadowAny : 0u);
                    spawn_shadow = true;
                  }
                }
                if (!delta) {
                  BSample bs;
                  if (bsdf_sample(B, kAllButSpecular, rng_uniform(key, bounce_dim(dimb, kDimMisSampleU)),
                                  rng_uniform(key, bounce_dim(dimb, kDimMisSampleV)), &bs)) {
                    V3 f = bs.f * fabsf(dot(bs.wi, ns));
                    if (!is_black(f) && bs.pdf > 0.0f) {
                      float w = 1.0f;
                      bool ok = true;
                      if (!is_spec(bs.type)) {
                        float lp = lt.type == kLightDiffuseArea ? area_light_pdf(S, lt, sf.p, bs.wi) : ((lt.type == kLightPerez || lt.type == kLightImage) ? sky_pdf(S, lt, bs.wi) : 0.0f);
                        if (lp == 0.0f) ok = false;
                        else w = (bs.pdf * bs.pdf) / (bs.pdf * bs.pdf + lp * lp);
                      }
                      if (ok) {
                        V3 c = mul(beta, f * (w / bs.pdf)) * lscale;
                        a.ray_o[2 * P + p] = make_float4(sf.p.x, sf.p.y, sf.p.z, kTMin);
                        a.ray_d[2 * P + p] = make_float4(bs.wi.x, bs.wi.y, bs.wi.z, kFltMax);
                        a.pend_mis[p] = make_float4(c.x, c.y, c.z, __int_as_float(li));
                        flags |= kPendMis;
                        spawn_mis = true;
                      }
                    }
                  }
                }
              }
              BSample bs;
              bool cont = bsdf_sample(B, kAll, rng_uniform(key, bounce_dim(dimb, kDimBsdfU)), rng_uniform(key, bounce_dim(dimb, kDimBsdfV)), &bs);
              if (cont && (is_black(bs.f) || bs.pdf == 0.0f)) cont = false;
              if (cont) {
                beta = mul(beta, bs.f * (fabsf(dot(bs.wi, ns)) / bs.pdf));
                const bool sp2 = is_spec(bs.type);
                flags = sp2 ? (flags | kFlagSpecular) : (flags & ~kFlagSpecular);
                if ((bs.type & kTrans) && sp2) eta_scale *= dot(wo, sf.g.w) > 0.0f ? B.eta * B.eta : 1.0f / (B.eta * B.eta);
                a.ray_o[p] = make_float4(sf.p.x, sf.p.y, sf.p.z, kTMin);
                a.ray_d[p] = make_float4(bs.wi.x, bs.wi.y, bs.wi.z, kFltMax);
                V3 rr = beta * eta_scale;
                float mx = fmaxf(rr.x, fmaxf(rr.y, rr.z));
                if (mx < 1.0f && bounce >= min_rr) {
                  float q = fmaxf(0.05f, 1.0f - mx);
                  if (rng_uniform(key, bounce_dim(dimb, kDimRoulette)) < q) cont = false;
                  else beta = beta * (1.0f / (1.0f - q));
                }
              }
              if (cont) { spawn_ext = true; ++bounce; ++dimb; }
              else alive = false;
            }
          }
        }
      }
      if (alive && !spawn_ext) alive = false;
      if (last_step && alive) { alive = false; spawn_ext = false; }
      flags = alive ? (flags | kAlive) : (flags & ~kAlive);
      keep = alive || spawn_shadow || spawn_mis;
      if (last_step) { keep = false; spawn_shadow = spawn_mis = false; }
      if (!keep && !(flags & kNoSample)) {
        if constexpr (kMulti) film_add_to(J->film_sum, J->film_sq, meta.x, L);
        else film_add(a, meta.x, meta.y, L);
      }
      retire = kMulti && !keep;
      a.beta[p] = make_float4(beta.x, beta.y, beta.z, eta_scale);
      a.radiance[p] = make_float4(L.x, L.y, L.z, (float)(step + 1));
      a.meta[p] = make_uint4(meta.x, meta.y, ((unsigned)bounce & 0xffffu) | ((unsigned)dimb << 16), flags);
    }
    // appends (all lanes of the warp take part)
    if (!kMulti && a.ray_mask) {
      // rays listed later in path order (k_ray_list_ordered): pixel-coherent traversal batches
      if (i < n) a.ray_mask[p] = (unsigned char)((spawn_ext ? 1u : 0u) | (spawn_shadow ? 2u : 0u) | (spawn_mis ? 4u : 0u) | (shadow_any ? 8u : 0u));
    } else {
      const unsigned r0 = warp_append(a.next_ray_count, spawn_ext);
      if (spawn_ext) a.next_ray_list[r0] = p << 3;
      const unsigned r1 = warp_append(a.next_ray_count, spawn_shadow);
      if (spawn_shadow) a.next_ray_list[r1] = (p << 3) | (shadow_any ? 4u : 0u) | 1u;
      const unsigned r2 = warp_append(a.next_ray_count, spawn_mis);
      if (spawn_mis) a.next_ray_list[r2] = (p << 3) | 2u;
    }
    const unsigned w = warp_append(a.next_work_count, keep);
    if (keep) a.next_work_list[w] = p;
    if constexpr (kMulti) {
      // retired slots back on the free stack; per-job retire counts, one atomic per job in the warp
      const unsigned f = warp_append(a.free_top, retire);
      if (retire) a.free_stack[f] = p;
      const unsigned peers = __match_any_sync(0xffffffffu, retire ? job : 0xffffffffu);
      const unsigned lane = threadIdx.x & 31u;
      if (retire && (int)lane == __ffs(peers) - 1) atomicAdd(a.job_done + job, (unsigned long long)__popc(peers));
      const unsigned rmask = __ballot_sync(0xffffffffu, retire);
      if (lane == 0 && rmask) atomicAdd(&a.state->retired, (unsigned long long)__popc(rmask));
    }
  }
}

// One block per kRayListBlock consecutive paths: each thread counts its
// path's rays, a block scan places them, one atomic reserves the block's run.
// Within a run the rays are in path (pixel) order, so the traversal's warps
// fetch neighbouring pixels' rays together.
__global__ void __launch_bounds__(kRayListBlock) k_ray_list_ordered(const unsigned char* ray_mask, unsigned paths, unsigned* ray_list,
                                                                     unsigned* ray_count) {
  __shared__ unsigned warp_sum[kRayListBlock / 32];
  __shared__ unsigned block_base;
  const unsigned p = blockIdx.x * kRayListBlock + threadIdx.x;
  const unsigned m = p < paths ? (unsigned)ray_mask[p] : 0u;
  const unsigned c = __popc(m & 7u);
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned incl = c;  // inclusive warp scan
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
    if ((int)lane >= o) incl += v;
  }
  if (lane == 31u) warp_sum[warp] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int w = 0; w < kRayListBlock / 32; ++w) { const unsigned t = warp_sum[w]; warp_sum[w] = acc; acc += t; }
    block_base = acc ? atomicAdd(ray_count, acc) : 0u;
  }
  __syncthreads();
  unsigned at = block_base + warp_sum[warp] + incl - c;
  if (m & 1u) ray_list[at++] = p << 3;
  if (m & 2u) ray_list[at++] = (p << 3) | ((m & 8u) ? 4u : 0u) | 1u;
  if (m & 4u) ray_list[at] = (p << 3) | 2u;
}

// At most 256 threads a block, two blocks per SM: the shading kernels fit in
// 128 registers (the general BSDF asks for ~156, which left one 256-thread
// block per SM); the batch and textured variants spill at most 44 bytes.
constexpr int kShadeMinBlocks = 2;
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path(ShadeArgs a) { shade_path<false, false>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_records(ShadeArgs a) { shade_path<true, false>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_batch(ShadeArgs a) { shade_path<false, true>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_batch_records(ShadeArgs a) { shade_path<true, true>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_textured(ShadeArgs a) { shade_path<true, false, true>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_batch_textured(ShadeArgs a) { shade_path<true, true, true>(a); }

// ---- material sort of the shade work list -----------------------------------
// Shading diverges badly when one warp holds paths on different materials (each
// material is a different BSDF routine), so the work list of every step is
// counting-sorted by material kind before shading.
template <bool kMulti>
__device__ __forceinline__ void sort_count(const SortArgs& a) {
  __shared__ unsigned cnt[kSortBins];
  if (threadIdx.x < kSortBins) cnt[threadIdx.x] = 0;
  __syncthreads();
  const unsigned n = *a.work_count;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned p = a.work_list[i];
    int key = kMatKinds + 1;
    if (a.meta[p].w & kFlagAlive) {
      const int hp = __float_as_int(a.hits[p].y);
      const SceneView& S = scene_at<kMulti>(a, kMulti ? a.jobs[a.slot_job[p]].scene : 0);
      key = hp < 0 ? kMatKinds : S.materials[S.prims[hp].material].kind;
    }
    a.keys[i] = (unsigned char)key;
    atomicAdd(&cnt[key], 1u);
  }
  __syncthreads();
  if (threadIdx.x < kSortBins && cnt[threadIdx.x]) atomicAdd(&a.bins[threadIdx.x], cnt[threadIdx.x]);
}
__global__ void k_sort_count(SortArgs a) { sort_count<false>(a); }
__global__ void k_sort_count_batch(SortArgs a) { sort_count<true>(a); }

__global__ void k_sort_scatter(SortArgs a) {
  __shared__ unsigned start[kSortBins];
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int k = 0; k < kSortBins; ++k) { start[k] = acc; acc += a.bins[k]; }
  }
  __syncthreads();
  const unsigned n = *a.work_count;
  const unsigned lane = threadIdx.x & 31u;
  for (unsigned base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const unsigned i = base + threadIdx.x;
    const bool valid = i < n;
    const int key = valid ? (int)a.keys[i] : -1;
    // one atomic per distinct key in the warp
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    unsigned pos = 0;
    if (valid && (int)lane == leader) pos = atomicAdd(&a.bins[kSortBins + key], (unsigned)__popc(peers));
    pos = __shfl_sync(0xffffffffu, pos, leader);
    if (valid) a.sorted[start[key] + pos + (unsigned)__popc(peers & ((1u << lane) - 1u))] = a.work_list[i];
  }
}

// RAY_CASTING (Scene.java:675) and DEPTH_CAMERA (Scene.java:327) on the
// primary hits; AO spawns its occlusion rays (Scene.java:272).
__global__ void k_shade_primary(ShadeArgs a, int algorithm) {
  const unsigned n = *a.work_count;
  const unsigned stride = gridDim.x * blockDim.x;
  const SceneView& S = a.scene;
  for (unsigned base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const unsigned i = base + threadIdx.x;
    if (i >= n) continue;
    const unsigned p = a.work_list[i];
    const uint4 meta = a.meta[p];
    if (!(meta.w & kAlive)) { if (algorithm == DFC_ALGO_AO) a.radiance[p] = make_float4(0, 0, 0, -2.0f); continue; }
    const float4 h = a.hits[p];
    const float4 ro = a.ray_o[p], rd = a.ray_d[p];
    const V3 ray_o = {ro.x, ro.y, ro.z}, ray_d = {rd.x, rd.y, rd.z};
    const int hp = __float_as_int(h.y);
    if (a.record_primary && p < a.pixels && hp < 0) { a.primary_prim[p] = -1; a.primary_t[p] = __int_as_float(0x7fc00000); }
    V3 L = {0, 0, 0};
    if (hp < 0) {
      if (a.preview) L = {1, 1, 1};
      else if (algorithm == DFC_ALGO_RAY_CASTING) for (int k = 0; k < S.light_count; ++k) L = L + light_Le_miss(S, S.lights[k], ray_d);
      if (algorithm == DFC_ALGO_AO) { a.radiance[p] = make_float4(L.x, L.y, L.z, -1.0f); continue; }
      film_add(a, meta.x, meta.y, L);
      continue;
    }
    const DPrim& pr = S.prims[hp];
    Surface sf;
    surface_of<true>(S, pr, __float_as_int(h.z), ray_o, ray_d, h.w, &sf);
    if (a.record_primary && p < a.pixels) { a.primary_prim[p] = hp; a.primary_t[p] = world_t(pr, ray_o, sf); }
    if (algorithm == DFC_ALGO_RAY_CASTING) {
      float c = fabsf(dot(sf.s.w, ray_d)) * 0.5f;
      film_add(a, meta.x, meta.y, V3{c, c, c});
    } else if (algorithm == DFC_ALGO_DEPTH) {
      V3 dd = sf.p - ray_o;
      float in = clampf(1.0f / (dot(dd, dd) * 0.5f), 0.0f, 1.0f);
      film_add(a, meta.x, meta.y, V3{in, in, in});
    } else {
      // AO: store the geometric basis' hit point and spawn samples into the AO ray pool
      a.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      for (int s = 0; s < a.ao_samples; ++s) {
        V3 dl = uniform_hemisphere(rng_uniform(meta.y, kDimBounceBase + 2 * s), rng_uniform(meta.y, kDimBounceBase + 2 * s + 1));
        V3 dw = normalize(to_world(dl, ONB{normalize(sf.g.u), normalize(sf.g.v), sf.g.w}));
        size_t slot = (size_t)p * a.ao_samples + s;
        a.ao_o[slot] = make_float4(sf.p.x, sf.p.y, sf.p.z, kTMin);
        a.ao_d[slot] = make_float4(dw.x, dw.y, dw.z, kFltMax);
      }
    }
  }
}

__global__ void __launch_bounds__(kTraceBlock) k_trace_ao(AoArgs a) {
  __shared__ int stack_smem[kStack * kTraceBlock];
  int* stack = stack_smem + threadIdx.x;
  const size_t n = (size_t)a.paths * a.samples;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t base = (size_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const size_t i = base + threadIdx.x;
    if (i >= n) continue;
    const unsigned p = (unsigned)(i / a.samples);
    if (a.radiance[p].w < 0.0f) continue;  // primary miss
    const float4 ro = a.ao_o[i], rd = a.ao_d[i];
    Hit h = {0.0f, -1, -1, 0.0f};
    float v;
    if (a.max_distance > 0.0f) {
      bool hit = trace_ray<true>(a.scene, V3{ro.x, ro.y, ro.z}, V3{rd.x, rd.y, rd.z}, kFltMax, false, &h, stack, a.overflow);
      v = hit ? clampf(h.t, 0.0f, a.max_distance) / a.max_distance : 1.0f;
    } else {
      bool hit = trace_ray<true>(a.scene, V3{ro.x, ro.y, ro.z}, V3{rd.x, rd.y, rd.z}, kFltMax, true, &h, stack, a.overflow);
      v = hit ? 0.0f : 1.0f;
    }
    a.ao_value[i] = v;
  }
}

// ---- RAY_TRACING --------------------------------------------------------------
// scene/Scene.java:786 doRadianceRayTracer: at each hit its emission, every
// light sampled once (checkLightVisibility: closest hit on the light for area
// lights, occlusion otherwise, t in (0.001, distance + 0.001)), then below the
// bounce limit the BSDF's specular reflection and specular transmission
// samples recursively; no BSDF: the ray passes through.  The recursion is a
// depth-first walk over an explicit per-thread stack; each node's weight is the
// product of f |cos| / pdf along its branch.  Random numbers per node n (root
// 0; reflection, transmission, pass-through children 3n+1, 3n+2, 3n+3): key
// rng_path_key(sample key, n, kRtSalt), dims 0-1 reflection, 2-3
// transmission, 4 the material draw, 8+3k.. light k (as the oracle).
constexpr uint32_t kRtSalt = 0x52545243u;
constexpr int kRtMaxNodes = 4096;  // nodes per sample; beyond it the tree is cut and counted
constexpr int kRtStack = 24;
struct RtEntry { V3 o, d, w; int bounce; uint32_t nid; };

__global__ void __launch_bounds__(kTraceBlock) k_ray_trace(ShadeArgs a, unsigned* overflow, unsigned long long* rays) {
  __shared__ int stack_smem[kStack * kTraceBlock];
  int* tstack = stack_smem + threadIdx.x;
  const SceneView& S = a.scene;
  const unsigned stride = gridDim.x * blockDim.x;
  unsigned long long nrays = 0;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < a.paths; p += stride) {
    const uint4 meta = a.meta[p];
    if (!(meta.w & kAlive)) continue;  // no camera ray: no sample (AbstractCPURenderer.java:221)
    const uint32_t key = meta.y;
    const float4 ro = a.ray_o[p], rd = a.ray_d[p];
    RtEntry st[kRtStack];
    int sp = 0, nodes = 0;
    st[sp++] = RtEntry{V3{ro.x, ro.y, ro.z}, V3{rd.x, rd.y, rd.z}, V3{1, 1, 1}, 0, 0u};
    V3 L = {0, 0, 0};
    const bool rec = a.record_primary && p < a.pixels;
    while (sp > 0) {
      const RtEntry e = st[--sp];
      if (++nodes > kRtMaxNodes) { atomicAdd(overflow, 1u); break; }
      const uint32_t nk = rng_path_key(key, e.nid, kRtSalt);
      Hit h = {0.0f, -1, -1, 0.0f};
      ++nrays;
      const bool found = trace_ray<true>(S, e.o, e.d, kFltMax, false, &h, tstack, overflow);
      if (!found) {
        if (rec && e.nid == 0u) { a.primary_prim[p] = -1; a.primary_t[p] = __int_as_float(0x7fc00000); }
        V3 Le = {0, 0, 0};
        for (int k = 0; k < S.light_count; ++k) Le = Le + light_Le_miss(S, S.lights[k], e.d);
        L = L + mul(e.w, Le);
        continue;
      }
      const DPrim& pr = S.prims[h.prim];
      Surface sf;
      surface_of<true>(S, pr, h.aux, e.o, e.d, h.t_obj, &sf);
      if (rec && e.nid == 0u) { a.primary_prim[p] = h.prim; a.primary_t[p] = world_t(pr, e.o, sf); }
      Bsdf B;
      const DMaterial& m = S.materials[pr.material];
      if (m.kind < kMatTextured ? !build_bsdf(m, sf, e.d, rng_uniform(nk, 4), &B, false)
                                : !textured_bsdf(S, pr, e.d, rng_uniform(nk, 4), false, &sf, &B)) {
        if (sp < kRtStack) st[sp++] = RtEntry{sf.p, e.d, e.w, e.bounce, e.nid * 3u + 3u};
        else atomicAdd(overflow, 1u);
        continue;
      }
      const V3 n = sf.s.w, wo = -e.d;
      V3 Ln;
      if (pr.light >= 0) {
        const DLight& lt = S.lights[pr.light];
        Ln = (lt.two_sided || dot(n, wo) > 0.0f) ? ld3(lt.radiance) : V3{0, 0, 0};
      } else {
        Ln = material_Le(S, pr, e.d, sf);  // after the BSDF, as Scene.doRadianceRayTracer: on the modified hit
      }
      for (int k = 0; k < S.light_count; ++k) {
        const DLight& lt = S.lights[k];
        LightS ls;
        if (!light_sample(S, lt, sf, rng_uniform(nk, 8 + 3 * k), rng_uniform(nk, 9 + 3 * k), rng_uniform(nk, 10 + 3 * k), &ls)) continue;
        if (is_black(ls.L) || !(ls.pdf > 0.0f)) continue;
        const V3 f = bsdf_f(B, kAll, ls.wi);
        if (is_black(f)) continue;
        const V3 toL = ls.p - sf.p;
        const float dist = fabsf(len(toL)) + 0.001f;
        Hit sh = {0.0f, -1, -1, 0.0f};
        ++nrays;
        bool vis;
        if (lt.type == kLightDiffuseArea) {
          vis = trace_ray<true>(S, sf.p, normalize(toL), dist, false, &sh, tstack, overflow) && S.prims[sh.prim].light == k;
        } else {
          vis = !trace_ray<true>(S, sf.p, normalize(toL), dist, true, &sh, tstack, overflow);
        }
        if (vis) Ln = Ln + mul(f, ls.L) * (fabsf(dot(ls.wi, n)) * (1.0f / ls.pdf));
      }
      L = L + mul(e.w, Ln);
      if (e.bounce + 1 < a.max_bounce) {
#pragma unroll 1
        for (int b = 0; b < 2; ++b) {
          BSample bs;
          if (!bsdf_sample(B, b == 0 ? (kSpecular | kRefl) : (kSpecular | kTrans), rng_uniform(nk, 2 * b), rng_uniform(nk, 2 * b + 1), &bs)) continue;
          const float c = fabsf(dot(bs.wi, n));
          if (is_black(bs.f) || !(bs.pdf > 0.0f) || !(c > 0.0f)) continue;
          if (sp < kRtStack) st[sp++] = RtEntry{sf.p, bs.wi, mul(e.w, bs.f * (c / bs.pdf)), e.bounce + 1, e.nid * 3u + 1u + (uint32_t)b};
          else atomicAdd(overflow, 1u);
        }
      }
    }
    film_add(a, meta.x, key, L);
  }
  // rays traced by this block's threads, one atomic per warp
  for (int off = 16; off > 0; off >>= 1) nrays += __shfl_down_sync(0xffffffffu, nrays, off);
  if ((threadIdx.x & 31u) == 0u && nrays) atomicAdd(rays, nrays);
}

__global__ void k_ao_resolve(ShadeArgs a, const float* ao_value, int samples) {
  const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.paths) return;
  const uint4 meta = a.meta[p];
  const float4 r = a.radiance[p];
  V3 L;
  if (r.w < -1.5f) return;  // no camera ray: no sample (AbstractCPURenderer.java:221)
  if (r.w < 0.0f) L = {r.x, r.y, r.z};
  else {
    float acc = 0.0f;
    for (int s = 0; s < samples; ++s) acc += ao_value[(size_t)p * samples + s];
    float v = acc * (kPi / samples);
    v = v / kPi;
    L = {v, v, v};
  }
  film_add(a, meta.x, meta.y, L);
}

// Film resolve: mean radiance -> tone mapper -> sRGB -> RGBA8
// (renderer/gpu/AbstractImageKernel.java:1104-1160, 1189-1325).
__global__ void k_resolve_rgba8(const float4* film_sum, int pixels, int tone_mapper, float exposure, uchar4* out, const float* film_consts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const float4 s = film_sum[i];
  V3 c;
  if (film_consts) {  // PixelImageF.filmRender: XYZ -> RGB, multiplyAndSaturateNegative(1 / weight sum)
    const float* m = film_consts + kFilmTable * kFilmTable + 9;
    c = V3{m[0] * s.x + m[1] * s.y + m[2] * s.z, m[3] * s.x + m[4] * s.y + m[5] * s.z, m[6] * s.x + m[7] * s.y + m[8] * s.z};
    if (s.w != 0.0f) {
      const float r = 1.0f / s.w;
      c = V3{fmaxf(c.x * r, 0.0f), fmaxf(c.y * r, 0.0f), fmaxf(c.z * r, 0.0f)};
    }
    tone_mapper = 1;  // no tone mapper on this film
  } else {
    c = s.w > 0.0f ? V3{s.x / s.w, s.y / s.w, s.z / s.w} : V3{0, 0, 0};
  }
  // renderer/gpu/AbstractImageKernel.java:1189-1325 (exposure e)
  auto tm = [&](float x) {
    const float b = x * exposure;
    switch (tone_mapper) {
      case 0: {  // imageToneMapFilmicCurveACESModifiedVersion1: filmic curve (2.51, 0.03, 2.43, 0.59, 0.14)
        const float v = fmaxf(b - 0.0f, -3.4028235e38f);
        return clampf((v * (2.51f * v + 0.03f)) / (v * (2.43f * v + 0.59f) + 0.14f), 0.0f, 1.0f);
      }
      case 2: return b / (1.0f + b);                                     // imageToneMapReinhard
      case 3: return b * (1.0f + b / (4.0f * 4.0f)) / (1.0f + b);         // ...ReinhardModifiedVersion1, L_white 4
      case 4: return 1.0f - expf(-b * exposure);                          // ...ReinhardModifiedVersion2
      case 5: return b / (b + 0.155f) * 1.019f;                           // imageToneMapUnreal3
      default: return x;                                                  // NONE
    }
  };
  c = V3{tm(c.x), tm(c.y), tm(c.z)};
  auto enc = [](float v) {
    v = clampf(v, 0.0f, 1.0f);
    // sRGB redo-gamma with the ColorSpaceF parameters (break point 0.00304, gamma 2.4)
    const float slope = 12.923210180787857f, slope_match = 1.0553409f, offset = 0.0553409f;
    v = v <= 0.00304f ? v * slope : slope_match * powf(v, 1.0f / 2.4f) - offset;
    return (unsigned char)(clampf(v, 0.0f, 1.0f) * 255.0f + 0.5f);
  };
  out[i] = make_uchar4(enc(c.x), enc(c.y), enc(c.z), 255);
}

// ---- batch engine: path slots refilled every iteration ------------------------
// The engine keeps `capacity` path slots.  Retired slots go on a free stack
// (shade pushes them); each iteration's plan takes as many as there are
// unstarted paths of admitted jobs, and regen starts those paths in them, so
// new jobs join the running wavefront at every bounce iteration.

__global__ void k_batch_init(BatchArgs a) {
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < a.capacity; i += stride) a.free_stack[i] = a.capacity - 1u - i;
  if (blockIdx.x == 0 && threadIdx.x == 0) a.state->free_top = a.capacity;
}

// Segment ring index of the appended segment that holds global path index g.
DFC_D unsigned seg_of(const BatchArgs& a, unsigned long long g) {
  unsigned lo = a.ctl->seg_lo, hi = a.ctl->seg_hi;
  while (hi - lo > 1u) {
    const unsigned mid = lo + (hi - lo) / 2u;
    if (a.segs[mid & a.seg_mask].start <= g) lo = mid;
    else hi = mid;
  }
  return lo & a.seg_mask;
}

// One thread: the previous iteration's counters are final (its rays are
// added up, then they are zeroed for the lists this iteration's shade fills),
// the unstarted paths of cancelled jobs at the cursor are skipped (counted as
// done), and the number of paths to start is fixed for regen.
__global__ void k_batch_plan(BatchArgs a) {
  for (unsigned i = threadIdx.x; i < 2u * kSortBins; i += blockDim.x) a.sort_bins[i] = 0u;
  if (threadIdx.x != 0) return;
  BatchState* st = a.state;
  st->rays += a.counts_next[0];
  a.counts_next[0] = 0u;
  a.counts_next[1] = 0u;
  a.counts_next[2] = 0u;
  const unsigned long long admitted = a.ctl->admitted;
  for (int guard = 0; guard < 64 && st->cursor < admitted; ++guard) {
    const DSegment& S = a.segs[seg_of(a, st->cursor)];
    if (!a.jobs[S.job].cancelled) break;
    const unsigned long long end = S.start + S.count;
    a.job_done[S.job] += end - st->cursor;
    st->cursor = end;
  }
  const unsigned long long rem = admitted - st->cursor;
  const unsigned top = st->free_top;
  const unsigned k = rem < (unsigned long long)top ? (unsigned)rem : top;
  st->regen_k = k;
  st->regen_base = top - k;
  st->regen_cursor = st->cursor;
  st->free_top = top - k;
  st->cursor += k;
  st->iterations += 1u;
}

// Starts the planned paths: global path index -> segment (binary search over
// the appended window by first path index) -> job path -> pixel and sample ->
// camera ray, in
// the same form as k_raygen so that a job's samples are those the per-job
// renderer draws for the same seed.
__global__ void k_batch_regen(BatchArgs a) {
  const BatchState* st = a.state;
  const unsigned k = st->regen_k, sbase = st->regen_base;
  const unsigned long long g0 = st->regen_cursor;
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = blockIdx.x * blockDim.x; base < k; base += stride) {
    const unsigned i = base + threadIdx.x;
    bool ok = false, valid = i < k;
    unsigned slot = 0;
    if (valid) {
      slot = a.free_stack[sbase + i];
      const unsigned long long g = g0 + i;
      const DSegment& S = a.segs[seg_of(a, g)];
      const unsigned jr = S.job;
      const DJob& J = a.jobs[jr];
      const unsigned long long q = S.q0 + (g - S.start);
      const unsigned pix = (unsigned)(q % J.pixels);
      const unsigned sample = (unsigned)(q / J.pixels);
      const unsigned x = pix % J.width, y = pix / J.width;
      const uint32_t key = rng_path_key(J.seed, pix, sample);
      V3 o = {0, 0, 0}, d = {0, 0, 1};
      if (!J.cancelled)
        ok = camera_ray(J.camera, (float)x, (float)y, rng_uniform(key, kDimPixelX), rng_uniform(key, kDimPixelY),
                        rng_uniform(key, kDimLensU), rng_uniform(key, kDimLensV), &o, &d);
      a.slot_job[slot] = jr;
      a.beta[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
      a.radiance[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      a.meta[slot] = make_uint4(pix, key, 0u, ok ? kAlive : kNoSample);
      a.ray_o[slot] = make_float4(o.x, o.y, o.z, kTMin);
      a.ray_d[slot] = make_float4(d.x, d.y, d.z, kFltMax);
    }
    const unsigned r = warp_append(a.counts_cur + 0, ok);
    if (ok) a.ray_list[r] = slot << 3;
    const unsigned w = warp_append(a.counts_cur + 1, valid);
    if (valid) a.work_list[w] = slot;
  }
}

}  // namespace dfc
