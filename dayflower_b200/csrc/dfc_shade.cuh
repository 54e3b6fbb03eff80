// Path-tracing shade step and the surface, light and film helpers it shares
// with the primary-hit, ambient-occlusion and ray-tracing kernels.
#pragma once

#include "dfc_texture.cuh"
#include "dfc_trav.cuh"

namespace dfc {

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
DFC_LIGHT_FN float area_light_pdf_t(const float* tri_attr, const DLight& lt, V3 p, V3 wi) {
  V3 ref = xf_point(lt.w2o, p);
  V3 w = normalize(xf_vec(lt.w2o, wi));
  if (lt.shape == kShapeTriangle) {
    const float* q = tri_attr + (size_t)lt.shape_data * 24;
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
DFC_D float area_light_pdf(const SceneView& S, const DLight& lt, V3 p, V3 wi) { return area_light_pdf_t(S.tri_attr, lt, p, wi); }

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
// The per-job renderer's box film.  A render pass has one path per pixel and
// its kernels run one after another on the renderer's stream, so every pixel
// has a single writer per pass: the sums take a plain read-add-write (two
// 16-byte loads and stores instead of seven atomics), in pass order, and a
// render is bitwise the same on every run.  The batch engine, whose wavefront
// can hold several samples of one pixel at once, adds with film_add_to.
DFC_D void film_add_owned(float4* film_sum, float4* film_sq, unsigned pix, V3 L) {
  if (!(isfinite(L.x) && isfinite(L.y) && isfinite(L.z))) return;  // AbstractCPURenderer.java:231
  if (luminance(L) < -1.0e-5f) return;
  float4 s = film_sum[pix];
  s.x += L.x; s.y += L.y; s.z += L.z; s.w += 1.0f;
  film_sum[pix] = s;
  float4 q = film_sq[pix];
  q.x += L.x * L.x; q.y += L.y * L.y; q.z += L.z * L.z;
  film_sq[pix] = q;
}
DFC_D void film_add(const ShadeArgs& a, unsigned pix, uint32_t key, V3 L) {
  if (a.pixel_film) film_splat(a, pix, key, L);
  else film_add_owned(a.film_sum, a.film_sq, pix, L);
}

// One shade step of the path tracer for every path on the work list.  In
// the batch engine (kMulti) the scene, film and bounce limits come from the
// path's job, a path ends at its own step max_bounce + 3 (the step count of
// a render pass of the per-job renderer), and a retired path's slot goes back
// on the free stack.
template <bool kRecords, bool kMulti, bool kTextured = false, int kLobes = kMaxLobes>
__device__ __forceinline__ void shade_path(const ShadeArgs& a) {
  unsigned begin = 0u, n = *a.work_count;
  if (a.range_bins) {  // this kernel's range of the sorted work list
    unsigned lo = 0u, hi = 0u;
    for (int k = 0; k < a.range_hi; ++k) {
      const unsigned c = a.range_bins[k];
      if (k < a.range_lo) lo += c;
      hi += c;
    }
    begin = lo;
    n = hi;
  }
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned base = begin + blockIdx.x * blockDim.x; base < n; base += stride) {
    const unsigned i = base + threadIdx.x;
    bool spawn_ext = false, spawn_shadow = false, spawn_mis = false, keep = false, shadow_any = false, retire = false;
    unsigned p = 0, job = 0;
    const bool valid = i < n;
    if (valid) {
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
            BsdfN<kLobes> B;
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
      if (valid)
        a.ray_mask[p] = (unsigned char)((spawn_ext ? 1u : 0u) | (spawn_shadow ? 2u : 0u) | (spawn_mis ? 4u : 0u) | (shadow_any ? 8u : 0u) |
                                        (keep && a.ordered_work ? kMaskKeep : 0u));
    } else {
      const unsigned r0 = warp_append(a.next_ray_count, spawn_ext);
      if (spawn_ext) a.next_ray_list[r0] = p << 3;
      const unsigned r1 = warp_append(a.next_ray_count, spawn_shadow);
      if (spawn_shadow) a.next_ray_list[r1] = (p << 3) | (shadow_any ? 4u : 0u) | 1u;
      const unsigned r2 = warp_append(a.next_ray_count, spawn_mis);
      if (spawn_mis) a.next_ray_list[r2] = (p << 3) | 2u;
    }
    if (kMulti || !a.ordered_work) {
      const unsigned w = warp_append(a.next_work_count, keep);
      if (keep) a.next_work_list[w] = p;
    }
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

}  // namespace dfc
