// AMBIENT_OCCLUSION rays and the RAY_TRACING kernel (one thread per camera
// sample, traced depth first).
#include "dfc_shade.cuh"

namespace dfc {

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

// One camera sample of the ray tracer: the radiance of the ray tree rooted at
// (o, d).  *prim0, *t0 receive the camera ray's hit (-1, NaN for a miss);
// *nrays counts the rays traced; a tree cut at kRtMaxNodes or a full stack is
// counted in *overflow.
DFC_D V3 rt_sample(const SceneView& S, V3 o, V3 d, uint32_t key, int max_bounce, int* tstack, unsigned* overflow,
                   unsigned long long* nrays, int* prim0, float* t0) {
  RtEntry st[kRtStack];
  int sp = 0, nodes = 0;
  st[sp++] = RtEntry{o, d, V3{1, 1, 1}, 0, 0u};
  V3 L = {0, 0, 0};
  *prim0 = -1;
  *t0 = __int_as_float(0x7fc00000);
  while (sp > 0) {
    const RtEntry e = st[--sp];
    if (++nodes > kRtMaxNodes) { atomicAdd(overflow, 1u); break; }
    const uint32_t nk = rng_path_key(key, e.nid, kRtSalt);
    Hit h = {0.0f, -1, -1, 0.0f};
    ++*nrays;
    const bool found = trace_ray<true>(S, e.o, e.d, kFltMax, false, &h, tstack, overflow);
    if (!found) {
      V3 Le = {0, 0, 0};
      for (int k = 0; k < S.light_count; ++k) Le = Le + light_Le_miss(S, S.lights[k], e.d);
      L = L + mul(e.w, Le);
      continue;
    }
    const DPrim& pr = S.prims[h.prim];
    Surface sf;
    surface_of<true>(S, pr, h.aux, e.o, e.d, h.t_obj, &sf);
    if (e.nid == 0u) { *prim0 = h.prim; *t0 = world_t(pr, e.o, sf); }
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
      ++*nrays;
      bool vis;
      if (lt.type == kLightDiffuseArea) {
        vis = trace_ray<true>(S, sf.p, normalize(toL), dist, false, &sh, tstack, overflow) && S.prims[sh.prim].light == k;
      } else {
        vis = !trace_ray<true>(S, sf.p, normalize(toL), dist, true, &sh, tstack, overflow);
      }
      if (vis) Ln = Ln + mul(f, ls.L) * (fabsf(dot(ls.wi, n)) * (1.0f / ls.pdf));
    }
    L = L + mul(e.w, Ln);
    if (e.bounce + 1 < max_bounce) {
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
  return L;
}

__global__ void __launch_bounds__(kTraceBlock) k_ray_trace(ShadeArgs a, unsigned* overflow, unsigned long long* rays) {
  __shared__ int stack_smem[kStack * kTraceBlock];
  int* tstack = stack_smem + threadIdx.x;
  const SceneView& S = a.scene;
  const unsigned stride = gridDim.x * blockDim.x;
  unsigned long long nrays = 0;
  for (unsigned p = blockIdx.x * blockDim.x + threadIdx.x; p < a.paths; p += stride) {
    const uint4 meta = a.meta[p];
    if (!(meta.w & kAlive)) continue;  // no camera ray: no sample (AbstractCPURenderer.java:221)
    const float4 ro = a.ray_o[p], rd = a.ray_d[p];
    int prim0;
    float t0;
    const V3 L = rt_sample(S, V3{ro.x, ro.y, ro.z}, V3{rd.x, rd.y, rd.z}, meta.y, a.max_bounce, tstack, overflow, &nrays, &prim0, &t0);
    if (a.record_primary && p < a.pixels) { a.primary_prim[p] = prim0; a.primary_t[p] = t0; }
    film_add(a, meta.x, meta.y, L);
  }
  // rays traced by this block's threads, one atomic per warp
  for (int off = 16; off > 0; off >>= 1) nrays += __shfl_down_sync(0xffffffffu, nrays, off);
  if ((threadIdx.x & 31u) == 0u && nrays) atomicAdd(rays, nrays);
}

// AMBIENT_OCCLUSION (Scene.java:272) of one camera sample with a known
// primary hit, as k_shade_primary + k_trace_ao + k_ao_resolve compute it:
// `samples` rays over the hemisphere of the geometric basis, weighted by
// their hit distance up to max_distance (occlusion alone when it is <= 0).
DFC_D V3 ao_sample(const SceneView& S, const DPrim& pr, int aux, V3 ray_o, V3 ray_d, float t_obj, uint32_t key, int samples,
                   float max_distance, int* tstack, unsigned* overflow, unsigned long long* nrays) {
  Surface sf;
  surface_of<true>(S, pr, aux, ray_o, ray_d, t_obj, &sf);
  const ONB g = ONB{normalize(sf.g.u), normalize(sf.g.v), sf.g.w};
  float acc = 0.0f;
  for (int s = 0; s < samples; ++s) {
    const V3 dl = uniform_hemisphere(rng_uniform(key, kDimBounceBase + 2 * s), rng_uniform(key, kDimBounceBase + 2 * s + 1));
    const V3 dw = normalize(to_world(dl, g));
    Hit h = {0.0f, -1, -1, 0.0f};
    ++*nrays;
    float v;
    if (max_distance > 0.0f) {
      const bool hit = trace_ray<true>(S, sf.p, dw, kFltMax, false, &h, tstack, overflow);
      v = hit ? clampf(h.t, 0.0f, max_distance) / max_distance : 1.0f;
    } else {
      v = trace_ray<true>(S, sf.p, dw, kFltMax, true, &h, tstack, overflow) ? 0.0f : 1.0f;
    }
    acc += v;
  }
  float v = acc * (kPi / samples);
  v = v / kPi;
  return V3{v, v, v};
}

// Batch engine: the AMBIENT_OCCLUSION and RAY_TRACING jobs' paths (sort key
// kKeyInline, after their camera ray was traced in the wavefront) finish in
// this one step: the occlusion rays or the ray tree are traced here, depth
// first on the path's thread, the sample goes to the job's film and the slot
// back on the free stack.
__global__ void __launch_bounds__(kTraceBlock) k_shade_inline_batch(ShadeArgs a) {
  __shared__ int stack_smem[kStack * kTraceBlock];
  int* tstack = stack_smem + threadIdx.x;
  unsigned begin = 0u, n = 0u;
  for (int k = 0; k < a.range_hi; ++k) {
    const unsigned c = a.range_bins[k];
    if (k < a.range_lo) begin += c;
    n += c;
  }
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long nrays = 0;
  // the loop bound is the same for every thread of a block, so the warp votes below see all 32 lanes
  for (unsigned base = begin + blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const unsigned i = base + threadIdx.x;
    const bool valid = i < n;
    unsigned p = 0, job = 0;
    if (valid) {
      p = a.work_list[i];
      job = a.slot_job[p];
      const DJob& J = a.jobs[job];
      const SceneView& S = a.scenes[J.scene];
      const uint4 meta = a.meta[p];
      const float4 ro = a.ray_o[p], rd = a.ray_d[p];
      const V3 o = {ro.x, ro.y, ro.z}, d = {rd.x, rd.y, rd.z};
      V3 L = {0, 0, 0};
      if (J.kind == kJobRayTracing) {
        int prim0;
        float t0;
        L = rt_sample(S, o, d, meta.y, J.max_bounce, tstack, a.overflow, &nrays, &prim0, &t0);
        --nrays;  // its camera ray was traced (and counted) in the wavefront
      } else {  // ambient occlusion from the camera ray's hit in the wavefront's hit record
        const float4 h = a.hits[p];
        const int hp = __float_as_int(h.y);
        if (hp >= 0) L = ao_sample(S, S.prims[hp], __float_as_int(h.z), o, d, h.w, meta.y, J.ao_samples, J.ao_distance, tstack, a.overflow, &nrays);
      }
      film_add_to(J.film_sum, J.film_sq, meta.x, L);
    }
    // every path here is done: its slot goes back on the free stack, one retire atomic per job in the warp
    const unsigned f = warp_append(a.free_top, valid);
    if (valid) a.free_stack[f] = p;
    const unsigned peers = __match_any_sync(0xffffffffu, valid ? job : 0xffffffffu);
    if (valid && (int)lane == __ffs(peers) - 1) atomicAdd(a.job_done + job, (unsigned long long)__popc(peers));
    const unsigned rmask = __ballot_sync(0xffffffffu, valid);
    if (lane == 0u && rmask) atomicAdd(&a.state->retired, (unsigned long long)__popc(rmask));
  }
  for (int off = 16; off > 0; off >>= 1) nrays += __shfl_down_sync(0xffffffffu, nrays, off);
  if (lane == 0u && nrays) atomicAdd(&a.state->rays, nrays);
}

}  // namespace dfc
