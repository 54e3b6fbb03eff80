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
//
// This file holds ray generation, the path-ordered ray lists, the material
// sort, primary-hit shading, film resolve and the batch engine's kernels;
// traversal is in dfc_trace.cu, shading in dfc_shade.cu and
// dfc_shade_simple.cu, ambient occlusion and ray tracing in dfc_raytrace.cu.
#include "dfc_shade.cuh"


namespace dfc {

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

// One block per kRayListBlock consecutive paths: each thread counts its
// path's rays (and, with a work list, whether the path is shaded again), a
// block scan places them, one atomic per list reserves the block's run.
// Within a run the entries are in path (pixel) order, so the traversal's
// warps fetch neighbouring pixels' rays together and the shading kernel reads
// neighbouring paths' state.
__global__ void __launch_bounds__(kRayListBlock) k_ray_list_ordered(const unsigned char* ray_mask, unsigned paths, unsigned* ray_list,
                                                                     unsigned* ray_count, unsigned* work_list, unsigned* work_count) {
  static_assert(kRayListBlock * 3 < 65536, "ray and work counts are packed in 16-bit fields");
  __shared__ unsigned warp_sum[kRayListBlock / 32];
  __shared__ unsigned block_base, work_base;
  const unsigned p = blockIdx.x * kRayListBlock + threadIdx.x;
  const unsigned m = p < paths ? (unsigned)ray_mask[p] : 0u;
  const unsigned keep = work_list != nullptr && (m & kMaskKeep) ? 1u : 0u;
  const unsigned c = __popc(m & 7u) | (keep << 16);  // rays, work entries (packed)
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
    const unsigned rays = acc & 0xffffu, works = acc >> 16;
    block_base = rays ? atomicAdd(ray_count, rays) : 0u;
    work_base = works ? atomicAdd(work_count, works) : 0u;
  }
  __syncthreads();
  const unsigned excl = warp_sum[warp] + incl - c;
  unsigned at = block_base + (excl & 0xffffu);
  if (m & 1u) ray_list[at++] = p << 3;
  if (m & 2u) ray_list[at++] = (p << 3) | ((m & 8u) ? 4u : 0u) | 1u;
  if (m & 4u) ray_list[at] = (p << 3) | 2u;
  if (keep) work_list[work_base + (excl >> 16)] = p;
}

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
    int key = kKeyNothing;
    if (a.meta[p].w & kFlagAlive) {
      const int hp = __float_as_int(a.hits[p].y);
      const DJob* J = kMulti ? a.jobs + a.slot_job[p] : nullptr;
      const SceneView& S = scene_at<kMulti>(a, kMulti ? J->scene : 0);
      if (kMulti && (J->kind == kJobAmbientOcclusion || J->kind == kJobRayTracing)) key = kKeyInline;
      else key = hp < 0 ? kKeyMiss : material_sort_key(S.materials[S.prims[hp].material].kind);
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
  if (threadIdx.x < 32) {  // exclusive scan of the bin counts by the first warp (one load per lane)
    const unsigned lane = threadIdx.x;
    const unsigned c = lane < (unsigned)kSortBins ? a.bins[lane] : 0u;
    unsigned incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if ((int)lane >= o) incl += v;
    }
    if (lane < (unsigned)kSortBins) start[lane] = incl - c;
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
