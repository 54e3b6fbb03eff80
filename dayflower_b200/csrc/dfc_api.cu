// C-ABI of libdayflower_cuda: the handle that stands in for Dayflower's
// GPURenderer (renderer/gpu/GPURenderer.java, AbstractGPURenderer.java).
//
// A handle owns one CUDA stream, the device scene, the film and the
// wavefront buffers.  dfc_render() runs render passes of one sample per pixel
// (AbstractGPURenderer.java:231-297); each pass is the kernel sequence in
// dfc_kernels.cu enqueued on the handle's stream, with no host synchronisation
// between the bounce steps.
#include <cuda_runtime.h>

#include <chrono>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dayflower_cuda.h"
#include "dfc_devscene.h"
#include "dfc_ingest.h"
#include "dfc_kernels.h"

using namespace dfc;

struct dfc_renderer {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::mutex mu;
  std::atomic<bool> stop{false};
  std::string err;
  // settings (AbstractGPURenderer.java:148-158)
  int width = 800, height = 800;
  int image_from_camera = 0;
  int algorithm = DFC_PATH_TRACING;
  int max_bounce = 20, min_rr = 5, ao_samples = 10, tone_mapper = DFC_TONE_MAPPER_NONE, preview = 0;
  float max_distance = 20.0f;
  uint32_t seed = 0x5eed1234u;
  // scene
  Staged staged;
  bool have_scene = false;
  DeviceScene scene;
  // film and wavefront
  bool set_up = false;
  unsigned pixels = 0, paths = 0;
  int steps = 0;
  DevBuf d_film_sum, d_film_sq, d_primary_prim, d_primary_t, d_rgba;
  int film_filter = 0;   // 0: per-pixel box film; 1: the CPU renderer's Gaussian XYZ film (PixelImageF)
  int bvh_builder = DFC_BVH_DEVICE;  // mesh hierarchies of later commits: device builder (default) or host SAH
  DevBuf d_film_consts;  // Gaussian film: filter table, sRGB -> XYZ, XYZ -> sRGB
  DevBuf d_beta, d_rad, d_meta, d_ray_o, d_ray_d, d_hits, d_pend_s, d_pend_m;
  DevBuf d_ray_list[2], d_work_list[2], d_counts, d_overflow, d_ray_total;
  DevBuf d_ray_mask;  // path tracing: each path's new rays of the last shading step (k_ray_list_ordered)
  DevBuf d_sort_keys, d_sort_bins, d_sorted;
  DevBuf d_ao_o, d_ao_d, d_ao_v;
  int64_t pass = 0, total_paths = 0, launches = 0;
  // device milliseconds and launches of the last render call: [0] whole call, then per kernel kind
  // (DFC_KERNEL_*; filled while stage timing is on)
  float last_ms[DFC_KERNEL_KINDS] = {};
  int64_t last_launches[DFC_KERNEL_KINDS] = {};
  // observed renders: pinned host copy of the RGBA8 image handed to the observer
  uint8_t* h_rgba = nullptr;
  size_t h_rgba_bytes = 0;
  float commit_ms[4] = {0, 0, 0, 0};  // last dfc_scene_commit: ingest, of which BLAS, TLAS builds; upload
  // optional per-stage timing: event pairs around every launch of a render call
  int stage_timing = 0;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_marks;  // (stage, index of the start event)
  int sm_count = 148;
  bool full_bsdf = false;  // the committed scene has materials of more than two lobes (or evaluated per hit)
  int trace_blocks = 6, ao_blocks = 5, rt_blocks = 4;  // resident blocks per SM of k_trace / k_trace_ao / k_ray_trace
};

namespace {

int fail(dfc_renderer* r, int code, const std::string& msg) {
  if (r) r->err = msg;
  return code;
}

// The handle whose render observer this thread is running (dfc_render_observed
// holds the handle's lock during the callback, so a call back into the same
// handle is refused instead of deadlocking).
thread_local const dfc_renderer* t_observing = nullptr;
int cuda_fail(dfc_renderer* r, cudaError_t e, const char* what) {
  int code = (e == cudaErrorMemoryAllocation) ? DFC_E_OOM : DFC_E_CUDA;
  return fail(r, code, std::string(what) + ": " + cudaGetErrorString(e));
}
// Entry points that take the handle's lock.  A call from inside the handle's
// own render observer (same thread, lock held) is refused.
#define DFC_LOCK(r)                                                                                       \
  if (t_observing == (r)) return fail((r), DFC_E_STATE, "called from inside the handle's render observer"); \
  std::lock_guard<std::mutex> lk((r)->mu)

#define DFC_CK(expr, what)                             \
  do {                                                 \
    cudaError_t e_ = (expr);                           \
    if (e_ != cudaSuccess) return cuda_fail(r, e_, what); \
  } while (0)

// Per-pass totals: [0] rays traced, [1] shade work items, [2] camera rays (the rays of step 0).
__global__ void k_sum_counts(const unsigned* counts, int steps, unsigned long long* total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    unsigned long long s = 0, w = 0;
    for (int i = 0; i < steps; ++i) { s += counts[4 * i]; w += counts[4 * i + 1]; }
    total[0] += s;
    total[1] += w;
    total[2] += counts[0];
  }
}

// Stage ids are the DFC_KERNEL_* kinds.
int stage_begin(dfc_renderer* r, int stage) {
  if (!r->stage_timing) return -1;
  const size_t need = r->ev_marks.size() * 2 + 2;
  while (r->ev_pool.size() < need) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
    r->ev_pool.push_back(e);
  }
  const int i = (int)r->ev_marks.size() * 2;
  cudaEventRecord(r->ev_pool[i], r->stream);
  r->ev_marks.push_back({stage, i});
  return i;
}
void stage_end(dfc_renderer* r, int i) {
  if (i >= 0) cudaEventRecord(r->ev_pool[i + 1], r->stream);
}
void collect_stages(dfc_renderer* r) {
  for (int k = 1; k < DFC_KERNEL_KINDS; ++k) { r->last_ms[k] = 0.0f; r->last_launches[k] = 0; }
  for (auto& m : r->ev_marks) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, r->ev_pool[m.second], r->ev_pool[m.second + 1]) == cudaSuccess) r->last_ms[m.first] += ms;
    r->last_launches[m.first] += 1;
  }
  r->ev_marks.clear();
}

// The CPU renderer's film constants: the 16x16 table of GaussianFilter2F(2, 2, 2)
// (filter/Filter2F.java:119, GaussianFilter2F.java:117) and the sRGB matrices of
// ColorSpaceF (color/ColorSpaceF.java:85, derived from the primaries and white
// point), laid out as k_resolve_rgba8 and film_splat read them.
std::vector<float> pixel_film_constants() {
  std::vector<float> c(kFilmTable * kFilmTable + 18);
  auto gauss = [](float d) {
    const float e = std::exp(-2.0f * 2.0f * 2.0f);
    return std::fmax(0.0f, std::exp(-2.0f * d * d) - e);
  };
  for (int y = 0; y < kFilmTable; ++y)
    for (int x = 0; x < kFilmTable; ++x)
      c[y * kFilmTable + x] = gauss((x + 0.5f) * 2.0f * (1.0f / kFilmTable)) * gauss((y + 0.5f) * 2.0f * (1.0f / kFilmTable));
  const float xR = 0.64f, yR = 0.33f, xG = 0.3f, yG = 0.6f, xB = 0.15f, yB = 0.06f, xW = 0.31271f, yW = 0.32902f;
  const float zR = 1.0f - (xR + yR), zG = 1.0f - (xG + yG), zB = 1.0f - (xB + yB), zW = 1.0f - (xW + yW);
  const float rX = (yG * zB) - (yB * zG), rY = (xB * zG) - (xG * zB), rZ = (xG * yB) - (xB * yG);
  const float rW = ((rX * xW) + (rY * yW) + (rZ * zW)) / yW;
  const float gX = (yB * zR) - (yR * zB), gY = (xR * zB) - (xB * zR), gZ = (xB * yR) - (xR * yB);
  const float gW = ((gX * xW) + (gY * yW) + (gZ * zW)) / yW;
  const float bX = (yR * zG) - (yG * zR), bY = (xG * zR) - (xR * zG), bZ = (xR * yG) - (xG * yR);
  const float bW = ((bX * xW) + (bY * yW) + (bZ * zW)) / yW;
  const float m[9] = {rX / rW, rY / rW, rZ / rW, gX / gW, gY / gW, gZ / gW, bX / bW, bY / bW, bZ / bW};  // XYZ -> RGB rows
  const float a = m[0] * (m[4] * m[8] - m[7] * m[5]), b = m[1] * (m[3] * m[8] - m[6] * m[5]), cc = m[2] * (m[3] * m[7] - m[6] * m[4]);
  const float sd = 1.0f / (a - b + cc);
  const float inv[9] = {sd * (m[4] * m[8] - m[5] * m[7]), sd * (m[5] * m[6] - m[3] * m[8]), sd * (m[3] * m[7] - m[4] * m[6]),
                        sd * (m[2] * m[7] - m[1] * m[8]), sd * (m[0] * m[8] - m[2] * m[6]), sd * (m[1] * m[6] - m[0] * m[7]),
                        sd * (m[1] * m[5] - m[2] * m[4]), sd * (m[2] * m[3] - m[0] * m[5]), sd * (m[0] * m[4] - m[1] * m[3])};
  std::memcpy(c.data() + kFilmTable * kFilmTable, inv, sizeof inv);  // RGB -> XYZ, column-major
  std::memcpy(c.data() + kFilmTable * kFilmTable + 9, m, sizeof m);
  return c;
}

int alloc_wavefront(dfc_renderer* r) {
  const unsigned W = (unsigned)r->width, H = (unsigned)r->height;
  r->pixels = W * H;
  r->paths = r->pixels;
  const size_t P = r->paths;
  DFC_CK(r->d_film_sum.ensure(P * 16), "film");
  DFC_CK(r->d_film_sq.ensure(P * 16), "film");
  DFC_CK(r->d_primary_prim.ensure(P * 4), "primary hits");
  DFC_CK(r->d_primary_t.ensure(P * 4), "primary hits");
  DFC_CK(r->d_rgba.ensure(P * 4), "image");
  DFC_CK(r->d_beta.ensure(P * 16), "path state");
  DFC_CK(r->d_rad.ensure(P * 16), "path state");
  DFC_CK(r->d_meta.ensure(P * 16), "path state");
  DFC_CK(r->d_ray_o.ensure(3 * P * 16), "rays");
  DFC_CK(r->d_ray_d.ensure(3 * P * 16), "rays");
  DFC_CK(r->d_hits.ensure(3 * P * 16), "hits");
  DFC_CK(r->d_pend_s.ensure(P * 16), "pending");
  DFC_CK(r->d_pend_m.ensure(P * 16), "pending");
  for (int k = 0; k < 2; ++k) {
    DFC_CK(r->d_ray_list[k].ensure(3 * P * 4), "ray list");
    DFC_CK(r->d_work_list[k].ensure(P * 4), "work list");
  }
  DFC_CK(r->d_overflow.ensure(16), "counters");
  DFC_CK(r->d_ray_total.ensure(32), "counters");
  DFC_CK(r->d_sort_keys.ensure(P), "sort");
  DFC_CK(r->d_sorted.ensure(P * 4), "sort");
  DFC_CK(r->d_ray_mask.ensure(P), "ray mask");
  DFC_CK(cudaMemsetAsync(r->d_ray_mask.p, 0, P, r->stream), "ray mask");
  if (r->film_filter == 1) {
    const std::vector<float> c = pixel_film_constants();
    DFC_CK(r->d_film_consts.ensure(c.size() * sizeof(float)), "film");
    DFC_CK(cudaMemcpy(r->d_film_consts.p, c.data(), c.size() * sizeof(float), cudaMemcpyHostToDevice), "film");
  }
  return DFC_OK;
}

int clear_film(dfc_renderer* r) {
  const size_t P = r->pixels;
  DFC_CK(cudaMemsetAsync(r->d_film_sum.p, 0, P * 16, r->stream), "clear");
  DFC_CK(cudaMemsetAsync(r->d_film_sq.p, 0, P * 16, r->stream), "clear");
  DFC_CK(cudaMemsetAsync(r->d_primary_prim.p, 0xff, P * 4, r->stream), "clear");
  DFC_CK(cudaMemsetAsync(r->d_primary_t.p, 0, P * 4, r->stream), "clear");
  DFC_CK(cudaMemsetAsync(r->d_overflow.p, 0, 16, r->stream), "clear");
  DFC_CK(cudaMemsetAsync(r->d_ray_total.p, 0, 32, r->stream), "clear");
  r->pass = 0;
  r->total_paths = 0;
  r->launches = 0;
  return DFC_OK;
}

ShadeArgs shade_args(dfc_renderer* r, int step) {
  ShadeArgs a{};
  a.scene = r->scene.view;
  a.pixel_film = r->film_filter == 1 ? r->d_film_consts.as<float>() : nullptr;
  a.width = (unsigned)r->width;
  a.height = (unsigned)r->height;
  a.paths = r->paths;
  a.pixels = r->pixels;
  a.max_bounce = r->max_bounce;
  a.min_rr = r->min_rr;
  a.preview = r->preview;
  a.last_step = 0;
  a.record_primary = r->pass == 0;
  a.ao_samples = r->ao_samples;
  unsigned* counts = r->d_counts.as<unsigned>();
  a.work_list = r->d_work_list[step & 1].as<unsigned>();
  a.work_count = counts + 4 * step + 1;
  a.next_work_list = r->d_work_list[(step + 1) & 1].as<unsigned>();
  a.next_work_count = counts + 4 * (step + 1) + 1;
  a.next_ray_list = r->d_ray_list[(step + 1) & 1].as<unsigned>();
  a.next_ray_count = counts + 4 * (step + 1);
  a.beta = r->d_beta.as<float4>();
  a.radiance = r->d_rad.as<float4>();
  a.meta = r->d_meta.as<uint4>();
  a.ray_o = r->d_ray_o.as<float4>();
  a.ray_d = r->d_ray_d.as<float4>();
  a.hits = r->d_hits.as<float4>();
  a.pend_shadow = r->d_pend_s.as<float4>();
  a.pend_mis = r->d_pend_m.as<float4>();
  a.film_sum = r->d_film_sum.as<float4>();
  a.film_sq = r->d_film_sq.as<float4>();
  a.primary_prim = r->d_primary_prim.as<int>();
  a.primary_t = r->d_primary_t.as<float>();
  a.ao_o = r->d_ao_o.as<float4>();
  a.ao_d = r->d_ao_d.as<float4>();
  return a;
}

// The traversal kernel for the committed scene: the one with the disk ... torus
// tests only when the scene has such primitives.
// Passes with at least this many paths list each step's rays in path order (k_ray_list_ordered).
constexpr unsigned kOrderedRayListMinPaths = 1u << 18;

using TraceKernel = void (*)(TraceArgs);
TraceKernel trace_kernel(const dfc_renderer* r) { return r->scene.host.record_shapes ? k_trace_records : k_trace; }

TraceArgs trace_args(dfc_renderer* r, int step) {
  TraceArgs t{};
  t.scene = r->scene.view;
  unsigned* counts = r->d_counts.as<unsigned>();
  t.ray_list = r->d_ray_list[step & 1].as<unsigned>();
  t.ray_count = counts + 4 * step;
  t.fetch = counts + 4 * step + 2;
  t.ray_o = r->d_ray_o.as<float4>();
  t.ray_d = r->d_ray_d.as<float4>();
  t.hits = r->d_hits.as<float4>();
  t.paths = r->paths;
  t.overflow = r->d_overflow.as<unsigned>();
  return t;
}

// Enqueues one render pass (one sample per pixel) on the handle's stream.
int enqueue_pass(dfc_renderer* r) {
  const int algo = r->algorithm;
  const int steps = algo == DFC_PATH_TRACING ? r->max_bounce + 4 : 1;
  const size_t counts_bytes = (size_t)(steps + 2) * 4 * sizeof(unsigned);
  DFC_CK(r->d_counts.ensure(counts_bytes), "counters");
  DFC_CK(cudaMemsetAsync(r->d_counts.p, 0, counts_bytes, r->stream), "counters");
  unsigned* counts = r->d_counts.as<unsigned>();
  RaygenArgs g{};
  g.scene = r->scene.view;
  g.paths = r->paths;
  g.pixels = r->pixels;
  g.width = (unsigned)r->width;
  g.sample_base = (unsigned)r->pass;
  g.seed = r->seed;
  g.beta = r->d_beta.as<float4>();
  g.radiance = r->d_rad.as<float4>();
  g.meta = r->d_meta.as<uint4>();
  g.ray_o = r->d_ray_o.as<float4>();
  g.ray_d = r->d_ray_d.as<float4>();
  g.ray_list = r->d_ray_list[0].as<unsigned>();
  g.ray_count = counts;
  g.work_list = r->d_work_list[0].as<unsigned>();
  g.work_count = counts + 1;
  int ev = stage_begin(r, DFC_KERNEL_RAYGEN);
  k_raygen<<<(r->paths + 255) / 256, 256, 0, r->stream>>>(g);
  stage_end(r, ev);
  r->launches++;
  const int trace_grid = r->sm_count * r->trace_blocks;
  // Shading: one block per 256 paths (a block shades at most one run of the work list), so the
  // hardware's block scheduler balances SMs whose runs cost more (materials differ in cost along
  // the material-sorted list).  Measured on the benchmark scene against grid-stride loops over
  // 4, 8, 16, 32 blocks per SM: shading 699, 714, 680, 658 ms per 64-spp render; one block per
  // run 640 ms.
  const int shade_grid = std::max(r->sm_count * 8, (int)((r->paths + 255) / 256));
  const int count_grid = r->sm_count * 8;  // the sort's count: one block-local histogram per block
  const int sort_grid = r->sm_count * 4;  // the scatter: fewer blocks, fewer bin scans and cursor atomics per launch
  if (algo == DFC_PATH_TRACING) {
    const size_t bins_bytes = (size_t)steps * 2 * kSortBins * sizeof(unsigned);
    DFC_CK(r->d_sort_bins.ensure(bins_bytes), "sort");
    DFC_CK(cudaMemsetAsync(r->d_sort_bins.p, 0, bins_bytes, r->stream), "sort");
    for (int s = 0; s < steps; ++s) {
      ev = stage_begin(r, DFC_KERNEL_TRACE);
      trace_kernel(r)<<<trace_grid, kTraceThreads, 0, r->stream>>>(trace_args(r, s));
      stage_end(r, ev);
      ShadeArgs a = shade_args(r, s);
      a.last_step = s == steps - 1;
      SortArgs so{};
      so.scene = r->scene.view;
      so.paths = r->paths;
      so.work_list = a.work_list;
      so.work_count = a.work_count;
      so.meta = a.meta;
      so.hits = a.hits;
      so.keys = r->d_sort_keys.as<unsigned char>();
      so.bins = r->d_sort_bins.as<unsigned>() + (size_t)s * 2 * kSortBins;
      so.sorted = r->d_sorted.as<unsigned>();
      // path-ordered ray lists pay for their extra launch only on large passes; small ones stay launch-bound
      a.ray_mask = r->paths >= kOrderedRayListMinPaths ? r->d_ray_mask.as<unsigned char>() : nullptr;
      // the next work list also in path order (the material sort below keeps that order within
      // each warp's run, so neighbouring lanes read neighbouring paths' state)
      a.ordered_work = a.ray_mask != nullptr;
      ev = stage_begin(r, DFC_KERNEL_SORT_COUNT);
      k_sort_count<<<count_grid, 256, 0, r->stream>>>(so);
      stage_end(r, ev);
      ev = stage_begin(r, DFC_KERNEL_SORT_SCATTER);
      k_sort_scatter<<<sort_grid, 256, 0, r->stream>>>(so);
      stage_end(r, ev);
      a.work_list = so.sorted;
      // the two-lobe kernel shades the matte ... plastic hits, misses and light-ray-only paths; the general
      // kernel the other materials, when the scene has any
      ShadeArgs simple = a;
      if (r->full_bsdf) {
        simple.range_bins = so.bins;
        simple.range_lo = 0;
        simple.range_hi = kSimpleBins;
      }
      ev = stage_begin(r, DFC_KERNEL_SHADE);
      (r->scene.host.record_shapes ? k_shade_path_simple_records : k_shade_path_simple)<<<shade_grid, 256, 0, r->stream>>>(simple);
      if (r->full_bsdf) {
        a.range_bins = so.bins;
        a.range_lo = kSimpleBins;
        a.range_hi = kKeyInline;
        (r->scene.host.textured() ? k_shade_path_textured : r->scene.host.record_shapes ? k_shade_path_records : k_shade_path)
            <<<shade_grid, 256, 0, r->stream>>>(a);
        r->launches += 1;
      }
      stage_end(r, ev);
      r->launches += 4;
      if (a.ray_mask && s < steps - 1) {  // the next step's ray list, in path order
        ev = stage_begin(r, DFC_KERNEL_RAY_LIST);
        k_ray_list_ordered<<<(r->paths + kRayListBlock - 1) / kRayListBlock, kRayListBlock, 0, r->stream>>>(
            a.ray_mask, r->paths, a.next_ray_list, a.next_ray_count, a.ordered_work ? a.next_work_list : nullptr, a.next_work_count);
        stage_end(r, ev);
        r->launches += 1;
      }
    }
  } else if (algo == DFC_RAY_TRACING) {
    ShadeArgs a = shade_args(r, 0);
    k_ray_trace<<<r->sm_count * r->rt_blocks, kTraceThreads, 0, r->stream>>>(a, r->d_overflow.as<unsigned>(),
                                                                             r->d_ray_total.as<unsigned long long>());
    r->launches += 1;
  } else {
    trace_kernel(r)<<<trace_grid, kTraceThreads, 0, r->stream>>>(trace_args(r, 0));
    ShadeArgs a = shade_args(r, 0);
    const int kind = algo == DFC_AMBIENT_OCCLUSION ? DFC_ALGO_AO : (algo == DFC_DEPTH_CAMERA ? DFC_ALGO_DEPTH : DFC_ALGO_RAY_CASTING);
    k_shade_primary<<<shade_grid, 256, 0, r->stream>>>(a, kind);
    r->launches += 2;
    if (kind == DFC_ALGO_AO) {
      AoArgs o{};
      o.scene = r->scene.view;
      o.paths = r->paths;
      o.samples = r->ao_samples;
      o.max_distance = r->max_distance;
      o.radiance = r->d_rad.as<float4>();
      o.ao_o = r->d_ao_o.as<float4>();
      o.ao_d = r->d_ao_d.as<float4>();
      o.ao_value = r->d_ao_v.as<float>();
      o.overflow = r->d_overflow.as<unsigned>();
      k_trace_ao<<<r->sm_count * r->ao_blocks, kTraceThreads, 0, r->stream>>>(o);
      k_ao_resolve<<<(r->paths + 255) / 256, 256, 0, r->stream>>>(a, r->d_ao_v.as<float>(), r->ao_samples);
      r->launches += 2;
    }
  }
  if (algo != DFC_RAY_TRACING)  // the ray tracer counts its own rays
    k_sum_counts<<<1, 1, 0, r->stream>>>(counts, algo == DFC_PATH_TRACING ? steps : 1, r->d_ray_total.as<unsigned long long>());
  DFC_CK(cudaGetLastError(), "kernel launch");
  r->pass++;
  r->total_paths += r->paths;
  return DFC_OK;
}

bool valid(const dfc_renderer* r) { return r != nullptr; }

}  // namespace

extern "C" {

int dfc_create(int device, dfc_renderer** out) {
  if (!out) return DFC_E_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) return DFC_E_CUDA;
  if (device < 0 || device >= count) return DFC_E_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return DFC_E_CUDA;
  dfc_renderer* r = new dfc_renderer();
  r->device = device;
  cudaDeviceGetAttribute(&r->sm_count, cudaDevAttrMultiProcessorCount, device);
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace, kTraceThreads, 0) == cudaSuccess && nb > 0) r->trace_blocks = nb;
  nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_records, kTraceThreads, 0) == cudaSuccess && nb > 0)
    r->trace_blocks = std::min(r->trace_blocks, nb);
  nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_ao, kTraceThreads, 0) == cudaSuccess && nb > 0) r->ao_blocks = nb;
  nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ray_trace, kTraceThreads, 0) == cudaSuccess && nb > 0) r->rt_blocks = nb;
  cudaGetLastError();
  if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&r->ev0) != cudaSuccess || cudaEventCreate(&r->ev1) != cudaSuccess) {
    delete r;
    return DFC_E_CUDA;
  }
  *out = r;
  return DFC_OK;
}

int dfc_destroy(dfc_renderer* r) {
  if (!r) return DFC_E_INVALID_ARG;
  {
    DFC_LOCK(r);
    cudaSetDevice(r->device);
    cudaStreamSynchronize(r->stream);
  }
  cudaEventDestroy(r->ev0);
  cudaEventDestroy(r->ev1);
  if (r->h_rgba) cudaFreeHost(r->h_rgba);
  for (cudaEvent_t e : r->ev_pool) cudaEventDestroy(e);
  cudaStream_t s = r->stream;
  delete r;  // DevBuf destructors free device memory
  cudaStreamDestroy(s);
  return DFC_OK;
}

const char* dfc_last_error(const dfc_renderer* r) { return r ? r->err.c_str() : "null handle"; }

int dfc_scene_put(dfc_renderer* r, const char* name, const void* data, int64_t count, int type) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (!name) return fail(r, DFC_E_INVALID_ARG, "name == null");
  if (count < 0 || (count > 0 && !data)) return fail(r, DFC_E_INVALID_ARG, "data == null or negative count");
  if (type != DFC_F32 && type != DFC_I32) return fail(r, DFC_E_INVALID_ARG, "type must be DFC_F32 or DFC_I32");
  try {  // the staging arrays are page-locked host memory (PinnedAllocator)
    if (type == DFC_F32) {
      stage_copy(r->staged.f32[name], static_cast<const float*>(data), (size_t)count);
    } else {
      stage_copy(r->staged.i32[name], static_cast<const int32_t*>(data), (size_t)count);
    }
  } catch (const std::bad_alloc&) {
    return fail(r, DFC_E_OOM, std::string("no page-locked host memory to stage ") + name);
  }
  return DFC_OK;
}

int dfc_scene_commit(dfc_renderer* r, int layout_version) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  RecycleOnExit recycle{r->staged};
  cudaSetDevice(r->device);
  HostScene hs;
  std::string err;
  const auto t0 = std::chrono::steady_clock::now();
  int rc = ingest_scene(r->staged, layout_version, &hs, &err, r->bvh_builder == DFC_BVH_DEVICE);
  if (rc != DFC_OK) return fail(r, rc, err);
  const auto t1 = std::chrono::steady_clock::now();
  r->commit_ms[0] = std::chrono::duration<float, std::milli>(t1 - t0).count();
  r->commit_ms[1] = hs.blas_ms;
  r->commit_ms[2] = hs.tlas_ms;
  DFC_CK(upload_scene(std::move(hs), r->stream, &r->scene), "scene upload");
  r->commit_ms[3] = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t1).count();
  r->have_scene = true;
  r->full_bsdf = r->scene.host.textured();
  for (const DMaterial& m : r->scene.host.materials) r->full_bsdf = r->full_bsdf || m.kind >= kSimpleKinds;
  if (r->image_from_camera) {
    r->width = (int)r->scene.host.camera[17];
    r->height = (int)r->scene.host.camera[18];
  }
  r->set_up = false;
  return DFC_OK;
}

int dfc_set_image(dfc_renderer* r, int width, int height) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (width == 0 && height == 0) {
    r->image_from_camera = 1;
    if (r->have_scene) { r->width = (int)r->scene.host.camera[17]; r->height = (int)r->scene.host.camera[18]; }
  } else {
    if (width < 1 || height < 1 || (int64_t)width * height > (1LL << 27)) return fail(r, DFC_E_INVALID_ARG, "resolution out of range");
    r->image_from_camera = 0;
    r->width = width;
    r->height = height;
  }
  r->set_up = false;
  return DFC_OK;
}

#define DFC_SETTER(fn, field, lo, hi, msg)                                            \
  int fn(dfc_renderer* r, int v) {                                                    \
    if (!valid(r)) return DFC_E_INVALID_ARG;                                          \
    DFC_LOCK(r);                                            \
    if (v < (lo) || v > (hi)) return fail(r, DFC_E_INVALID_ARG, msg);                 \
    r->field = v;                                                                     \
    return DFC_OK;                                                                    \
  }
DFC_SETTER(dfc_set_maximum_bounce, max_bounce, 0, 4096, "maximumBounce out of range")
DFC_SETTER(dfc_set_minimum_bounce_russian_roulette, min_rr, 0, 1 << 30, "minimumBounceRussianRoulette out of range")
DFC_SETTER(dfc_set_rendering_algorithm, algorithm, 0, 4, "unknown rendering algorithm")
DFC_SETTER(dfc_set_samples, ao_samples, 1, 4096, "samples out of range")
DFC_SETTER(dfc_set_tone_mapper, tone_mapper, 0, 5, "unknown tone mapper")
DFC_SETTER(dfc_set_preview_mode, preview, 0, 1, "preview mode is 0 or 1")

int dfc_set_maximum_distance(dfc_renderer* r, float v) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (!std::isfinite(v)) return fail(r, DFC_E_INVALID_ARG, "maximumDistance must be finite");
  r->max_distance = v;
  return DFC_OK;
}

int dfc_set_stage_timing(dfc_renderer* r, int on) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  r->stage_timing = on ? 1 : 0;
  return DFC_OK;
}

int dfc_set_seed(dfc_renderer* r, uint32_t seed) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  r->seed = seed;
  return DFC_OK;
}

int dfc_setup(dfc_renderer* r) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (!r->have_scene) return fail(r, DFC_E_STATE, "setup() before setScene()");
  cudaSetDevice(r->device);
  int rc = alloc_wavefront(r);
  if (rc) return rc;
  rc = clear_film(r);
  if (rc) return rc;
  r->set_up = true;
  return DFC_OK;
}

}  // extern "C"

namespace {

// Resolves the film into the RGBA8 image on the handle's stream
// (renderer/gpu/AbstractImageKernel.java:1104-1325; the tone mapper applies to
// PATH_TRACING only, GPURenderer.java:108-110, :312-335).
void enqueue_resolve(dfc_renderer* r) {
  const int tm = r->algorithm == DFC_PATH_TRACING ? r->tone_mapper : DFC_TONE_MAPPER_NONE;
  k_resolve_rgba8<<<(r->pixels + 255) / 256, 256, 0, r->stream>>>(r->d_film_sum.as<float4>(), (int)r->pixels, tm, 1.0f, r->d_rgba.as<uchar4>(),
                                                                  r->film_filter == 1 ? r->d_film_consts.as<float>() : nullptr);
}

// Calls the observer with the handle marked as observing on this thread.
void notify(dfc_renderer* r, dfc_observer_fn fn, void* user, int event, int pass, double progress, double millis, bool image) {
  dfc_pass_event ev{};
  ev.event = event;
  ev.render_pass = pass;
  ev.progress = progress;
  ev.millis = millis;
  ev.rgba = image ? r->h_rgba : nullptr;
  ev.width = r->width;
  ev.height = r->height;
  t_observing = r;
  fn(user, &ev);
  t_observing = nullptr;
}

// The image after the last pass into the pinned host copy handed to observers
// (AbstractGPURenderer.doUpdateImageF, :668-712).
int update_host_image(dfc_renderer* r) {
  const size_t bytes = (size_t)r->pixels * 4;
  if (r->h_rgba_bytes < bytes) {
    if (r->h_rgba) cudaFreeHost(r->h_rgba);
    r->h_rgba = nullptr;
    r->h_rgba_bytes = 0;
    DFC_CK(cudaMallocHost(reinterpret_cast<void**>(&r->h_rgba), bytes), "observer image");
    r->h_rgba_bytes = bytes;
  }
  enqueue_resolve(r);
  DFC_CK(cudaMemcpyAsync(r->h_rgba, r->d_rgba.p, bytes, cudaMemcpyDeviceToHost, r->stream), "observer image");
  DFC_CK(cudaStreamSynchronize(r->stream), "observer image");
  return DFC_OK;
}

// render(renderPasses) with the lock held.  Without an observer the passes are
// enqueued back to back and the host waits once; with one, every pass follows
// AbstractGPURenderer.render() (:231-297): onRenderDisplay of the cleared image
// on the first pass after a clear, onRenderPassProgress(0.0), the pass, the
// image update, onRenderPassProgress(1.0), onRenderDisplay and
// onRenderPassComplete(millis), the host waiting for each pass.
int render_locked(dfc_renderer* r, int passes, dfc_observer_fn fn, void* user, int* completed) {
  if (passes < 1) return fail(r, DFC_E_INVALID_ARG, "renderPasses < 1");  // AbstractGPURenderer.java:323
  if (!r->set_up) return fail(r, DFC_E_STATE, "render() before setup()");
  cudaSetDevice(r->device);
  if (r->algorithm == DFC_AMBIENT_OCCLUSION) {
    const size_t n = (size_t)r->paths * r->ao_samples;
    DFC_CK(r->d_ao_o.ensure(n * 16), "AO rays");
    DFC_CK(r->d_ao_d.ensure(n * 16), "AO rays");
    DFC_CK(r->d_ao_v.ensure(n * 4), "AO rays");
  }
  r->stop.store(false);
  DFC_CK(cudaEventRecord(r->ev0, r->stream), "event");
  int done = 0;
  for (int k = 0; k < passes; ++k) {
    if (r->stop.load()) break;
    if (fn) {
      if (r->pass == 0) {  // a cleared film: the observer sees the cleared image first
        if (int rc = update_host_image(r)) return rc;
        notify(r, fn, user, DFC_OBSERVE_DISPLAY, 0, 0.0, 0.0, true);
      }
      const int pass_no = (int)r->pass + 1;
      notify(r, fn, user, DFC_OBSERVE_PASS_PROGRESS, pass_no, 0.0, 0.0, false);
      const auto t0 = std::chrono::steady_clock::now();
      if (int rc = enqueue_pass(r)) return rc;
      if (int rc = update_host_image(r)) return rc;
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      ++done;
      notify(r, fn, user, DFC_OBSERVE_PASS_PROGRESS, pass_no, 1.0, 0.0, false);
      notify(r, fn, user, DFC_OBSERVE_DISPLAY, pass_no, 1.0, 0.0, true);
      notify(r, fn, user, DFC_OBSERVE_PASS_COMPLETE, pass_no, 1.0, ms, false);
    } else {
      if (int rc = enqueue_pass(r)) return rc;
      ++done;
    }
  }
  DFC_CK(cudaEventRecord(r->ev1, r->stream), "event");
  DFC_CK(cudaEventSynchronize(r->ev1), "render");
  DFC_CK(cudaGetLastError(), "render");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, r->ev0, r->ev1);
  r->last_ms[0] = ms;
  collect_stages(r);
  unsigned ov = 0;
  DFC_CK(cudaMemcpy(&ov, r->d_overflow.p, 4, cudaMemcpyDeviceToHost), "readback");
  if (completed) *completed = done;
  if (ov) return fail(r, DFC_E_TIMEOUT, "traversal stack bound exceeded on " + std::to_string(ov) + " node visits");
  if (done < passes) return fail(r, DFC_E_STOPPED, "render stopped");
  return DFC_OK;
}

}  // namespace

extern "C" {

int dfc_render(dfc_renderer* r, int passes, int* completed) {
  if (completed) *completed = 0;
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  return render_locked(r, passes, nullptr, nullptr, completed);
}

int dfc_render_observed(dfc_renderer* r, int passes, dfc_observer_fn fn, void* user, int* completed) {
  if (completed) *completed = 0;
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (!fn) return fail(r, DFC_E_INVALID_ARG, "observer == null");
  return render_locked(r, passes, fn, user, completed);
}

int dfc_render_shutdown(dfc_renderer* r) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  r->stop.store(true);
  return DFC_OK;
}

int dfc_clear(dfc_renderer* r) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (!r->set_up) return DFC_OK;
  cudaSetDevice(r->device);
  return clear_film(r);
}

int dfc_update_camera(dfc_renderer* r, const float* camera19) {
  if (!valid(r) || !camera19) return fail(r, DFC_E_INVALID_ARG, "camera == null");
  DFC_LOCK(r);
  if (!r->have_scene) return fail(r, DFC_E_STATE, "updateCamera() before setScene()");
  std::memcpy(r->scene.host.camera, camera19, 19 * sizeof(float));
  DFC_CK(cudaMemcpyAsync(r->scene.camera.p, camera19, 19 * sizeof(float), cudaMemcpyHostToDevice, r->stream), "camera");
  DFC_CK(cudaStreamSynchronize(r->stream), "camera");
  return DFC_OK;
}

int dfc_update_matrices(dfc_renderer* r, const float* m, int64_t n) {
  if (!valid(r) || !m) return fail(r, DFC_E_INVALID_ARG, "matrices == null");
  DFC_LOCK(r);
  if (!r->have_scene) return fail(r, DFC_E_STATE, "updateMatrix44Fs() before setScene()");
  if (n != (int64_t)r->scene.host.prims.size()) return fail(r, DFC_E_INVALID_ARG, "matrix count differs from the primitive count");
  // The top level is built over compiled bounding volumes; moving primitives
  // requires a new setScene so that the hierarchy sees their new boxes.
  for (int64_t p = 0; p < n; ++p) {
    DPrim& pr = r->scene.host.prims[p];
    const float* q = m + p * 32;
    std::memcpy(pr.o2w, q, 12 * sizeof(float));
    std::memcpy(pr.w2o, q + 16, 12 * sizeof(float));
    bool id = true;
    for (int k = 0; k < 16; ++k) id = id && q[k] == ((k % 5) == 0 ? 1.0f : 0.0f) && q[16 + k] == ((k % 5) == 0 ? 1.0f : 0.0f);
    pr.identity = id;
  }
  DFC_CK(cudaMemcpyAsync(r->scene.prims.p, r->scene.host.prims.data(), n * sizeof(DPrim), cudaMemcpyHostToDevice, r->stream), "matrices");
  DFC_CK(cudaStreamSynchronize(r->stream), "matrices");
  return DFC_OK;
}

int dfc_read_image_rgba8(dfc_renderer* r, uint8_t* dst, int64_t cap) {
  if (!valid(r) || !dst) return fail(r, DFC_E_INVALID_ARG, "dst == null");
  DFC_LOCK(r);
  if (!r->set_up) return fail(r, DFC_E_STATE, "no film");
  if (cap < (int64_t)r->pixels * 4) return fail(r, DFC_E_INVALID_ARG, "destination too small");
  enqueue_resolve(r);
  DFC_CK(cudaMemcpyAsync(dst, r->d_rgba.p, (size_t)r->pixels * 4, cudaMemcpyDeviceToHost, r->stream), "readback");
  DFC_CK(cudaStreamSynchronize(r->stream), "readback");
  return DFC_OK;
}

int dfc_read_film(dfc_renderer* r, float* dst, int64_t cap) {
  if (!valid(r) || !dst) return fail(r, DFC_E_INVALID_ARG, "dst == null");
  DFC_LOCK(r);
  if (!r->set_up) return fail(r, DFC_E_STATE, "no film");
  if (r->film_filter != 0) return fail(r, DFC_E_STATE, "the film is the Gaussian pixel film: read it with dfc_read_pixel_film");
  const size_t P = r->pixels;
  if (cap < (int64_t)P * 7) return fail(r, DFC_E_INVALID_ARG, "destination too small");
  std::vector<float> s(P * 4), q(P * 4);
  DFC_CK(cudaMemcpyAsync(s.data(), r->d_film_sum.p, P * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
  DFC_CK(cudaMemcpyAsync(q.data(), r->d_film_sq.p, P * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
  DFC_CK(cudaStreamSynchronize(r->stream), "readback");
  for (size_t i = 0; i < P; ++i) {
    dst[i * 7 + 0] = s[i * 4 + 0]; dst[i * 7 + 1] = s[i * 4 + 1]; dst[i * 7 + 2] = s[i * 4 + 2];
    dst[i * 7 + 3] = q[i * 4 + 0]; dst[i * 7 + 4] = q[i * 4 + 1]; dst[i * 7 + 5] = q[i * 4 + 2];
    dst[i * 7 + 6] = s[i * 4 + 3];
  }
  return DFC_OK;
}

int dfc_set_bvh_builder(dfc_renderer* r, int builder) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (builder != DFC_BVH_HOST && builder != DFC_BVH_DEVICE) return fail(r, DFC_E_INVALID_ARG, "builder is DFC_BVH_HOST or DFC_BVH_DEVICE");
  r->bvh_builder = builder;
  return DFC_OK;
}

int dfc_set_film_filter(dfc_renderer* r, int filter) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (filter != 0 && filter != 1) return fail(r, DFC_E_INVALID_ARG, "film filter is 0 (box) or 1 (Gaussian pixel film)");
  r->film_filter = filter;
  r->set_up = false;  // a new film: call setup() again
  return DFC_OK;
}

int dfc_read_pixel_film(dfc_renderer* r, float* dst, int64_t cap) {
  if (!valid(r) || !dst) return fail(r, DFC_E_INVALID_ARG, "dst == null");
  DFC_LOCK(r);
  if (!r->set_up) return fail(r, DFC_E_STATE, "no film");
  if (r->film_filter != 1) return fail(r, DFC_E_STATE, "the film is the box film: read it with dfc_read_film");
  if (cap < (int64_t)r->pixels * 4) return fail(r, DFC_E_INVALID_ARG, "destination too small");
  DFC_CK(cudaMemcpyAsync(dst, r->d_film_sum.p, (size_t)r->pixels * 16, cudaMemcpyDeviceToHost, r->stream), "readback");
  DFC_CK(cudaStreamSynchronize(r->stream), "readback");
  return DFC_OK;
}

int dfc_read_primary_hits(dfc_renderer* r, int32_t* prim, float* t, int64_t cap) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (!r->set_up) return fail(r, DFC_E_STATE, "no film");
  if (cap < (int64_t)r->pixels) return fail(r, DFC_E_INVALID_ARG, "destination too small");
  if (prim) DFC_CK(cudaMemcpyAsync(prim, r->d_primary_prim.p, (size_t)r->pixels * 4, cudaMemcpyDeviceToHost, r->stream), "readback");
  if (t) DFC_CK(cudaMemcpyAsync(t, r->d_primary_t.p, (size_t)r->pixels * 4, cudaMemcpyDeviceToHost, r->stream), "readback");
  DFC_CK(cudaStreamSynchronize(r->stream), "readback");
  return DFC_OK;
}

int dfc_read_counters(dfc_renderer* r, int64_t* out4) {
  if (!valid(r) || !out4) return fail(r, DFC_E_INVALID_ARG, "out == null");
  DFC_LOCK(r);
  unsigned long long rays = 0;
  if (r->set_up) {
    DFC_CK(cudaMemcpyAsync(&rays, r->d_ray_total.p, 8, cudaMemcpyDeviceToHost, r->stream), "readback");
    DFC_CK(cudaStreamSynchronize(r->stream), "readback");
  }
  out4[0] = r->pass;
  out4[1] = r->total_paths;
  out4[2] = (int64_t)rays;
  out4[3] = r->launches;
  return DFC_OK;
}

int dfc_read_commit_times(dfc_renderer* r, float* out4) {
  if (!valid(r) || !out4) return fail(r, DFC_E_INVALID_ARG, "out == null");
  DFC_LOCK(r);
  std::memcpy(out4, r->commit_ms, sizeof r->commit_ms);
  return DFC_OK;
}

int dfc_read_stage_times(dfc_renderer* r, float* out5) {
  if (!valid(r) || !out5) return fail(r, DFC_E_INVALID_ARG, "out == null");
  DFC_LOCK(r);
  const float* m = r->last_ms;
  out5[0] = m[0];
  out5[1] = m[DFC_KERNEL_RAYGEN];
  out5[2] = m[DFC_KERNEL_TRACE];
  out5[3] = m[DFC_KERNEL_SHADE] + m[DFC_KERNEL_SORT_COUNT] + m[DFC_KERNEL_SORT_SCATTER] + m[DFC_KERNEL_RAY_LIST];
  out5[4] = m[DFC_KERNEL_FILM];
  return DFC_OK;
}

int dfc_read_kernel_stats(dfc_renderer* r, float* ms, int64_t* launches, int64_t* items, int n) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (n < 1 || n > DFC_KERNEL_KINDS) return fail(r, DFC_E_INVALID_ARG, "n must be 1 .. DFC_KERNEL_KINDS");
  unsigned long long tot[4] = {0, 0, 0, 0};
  if (r->set_up) {
    DFC_CK(cudaMemcpyAsync(tot, r->d_ray_total.p, sizeof tot, cudaMemcpyDeviceToHost, r->stream), "readback");
    DFC_CK(cudaStreamSynchronize(r->stream), "readback");
  }
  int64_t it[DFC_KERNEL_KINDS] = {};
  it[0] = r->total_paths;
  it[DFC_KERNEL_RAYGEN] = r->total_paths;
  it[DFC_KERNEL_TRACE] = (int64_t)tot[0];
  it[DFC_KERNEL_SHADE] = it[DFC_KERNEL_SORT_COUNT] = it[DFC_KERNEL_SORT_SCATTER] = (int64_t)tot[1];
  it[DFC_KERNEL_RAY_LIST] = (int64_t)(tot[0] - tot[2]);
  for (int k = 0; k < n; ++k) {
    if (ms) ms[k] = r->last_ms[k];
    if (launches) launches[k] = k == 0 ? r->launches : r->last_launches[k];
    if (items) items[k] = it[k];
  }
  return DFC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// dfc_trace_rays_noalloc: closest-hit traversal of caller-supplied rays that
// makes no device allocation.  It is for callers that must not have the
// library allocate device memory on their behalf: a host that owns a fixed
// device arena and hands out every byte itself, or an interactive loop that
// cannot afford cudaMalloc/cudaFree, which may synchronise the whole device.
// Rays, hits and the committed scene live in memory the caller or
// dfc_scene_commit already owns; the traversal's own scratch (the ray list
// k_trace walks, its ray count, its fetch cursor and its overflow flag) lives
// in the static device array below instead of a cudaMalloc'd buffer.
//
// The scratch is one array per device per process.  Two calls on one device
// that overlapped in time would race on it, so every call holds
// g_noalloc_mu from its first launch until its stream has drained.

constexpr int64_t kNoAllocMaxRays = int64_t(1) << 20;   // 1,048,576 rays per call
constexpr int kNoAllocHeader = 64;                        // words: [0] ray count, [1] fetch cursor, [2] overflow flag
constexpr int kNoAllocMaxDevices = 64;

// 4 MiB + 256 B of device memory, set aside when the module loads.
static __device__ __align__(256) unsigned g_noalloc_scratch[kNoAllocHeader + kNoAllocMaxRays];

namespace {

std::mutex g_noalloc_mu;
unsigned* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// First kernel of every call: the fetch cursor and the overflow flag must be
// zero when k_trace starts, and are set here in stream order, so nothing
// depends on the load-time zero fill or on how an earlier call ended.
__global__ void k_noalloc_prepare(unsigned* scratch, unsigned n) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) scratch[kNoAllocHeader + i] = i << 3;  // slot i, closest-hit ray
  if (i == 0) { scratch[0] = n; scratch[1] = 0u; scratch[2] = 0u; }
}

// Once per device, with that device current: resolves the scratch address and
// loads both kernels, so later calls do no module loading.
int noalloc_setup(dfc_renderer* r, unsigned** out) {
  if (r->device < 0 || r->device >= kNoAllocMaxDevices)
    return fail(r, DFC_E_UNSUPPORTED, "dfc_trace_rays_noalloc supports device ordinals below 64");
  if (!g_noalloc_ptr[r->device]) {
    void* p = nullptr;
    DFC_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch), "dfc_trace_rays_noalloc scratch address");
    cudaFuncAttributes fa;
    DFC_CK(cudaFuncGetAttributes(&fa, k_noalloc_prepare), "dfc_trace_rays_noalloc set-up");
    DFC_CK(cudaFuncGetAttributes(&fa, k_trace), "dfc_trace_rays_noalloc set-up");
    DFC_CK(cudaFuncGetAttributes(&fa, k_trace_records), "dfc_trace_rays_noalloc set-up");
    g_noalloc_ptr[r->device] = static_cast<unsigned*>(p);
  }
  *out = g_noalloc_ptr[r->device];
  return DFC_OK;
}

bool device_pointer_on(const void* p, int device) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == device;
}

}  // namespace

extern "C" int dfc_trace_rays_noalloc(dfc_renderer* r, const float* d_origins, const float* d_directions, float* d_hits,
                                      int64_t count) {
  if (!valid(r)) return DFC_E_INVALID_ARG;
  DFC_LOCK(r);
  if (count < 0) return fail(r, DFC_E_INVALID_ARG, "count < 0");
  if (count > kNoAllocMaxRays)
    return fail(r, DFC_E_INVALID_ARG, "count " + std::to_string(count) + " exceeds the " + std::to_string(kNoAllocMaxRays) +
                                          "-ray limit of dfc_trace_rays_noalloc's static scratch; split the batch");
  if (!r->have_scene) return fail(r, DFC_E_STATE, "dfc_trace_rays_noalloc before setScene()");
  DFC_CK(cudaSetDevice(r->device), "cudaSetDevice");
  std::lock_guard<std::mutex> glk(g_noalloc_mu);
  unsigned* scratch = nullptr;
  if (int rc = noalloc_setup(r, &scratch)) return rc;
  if (count == 0) return DFC_OK;
  const void* ptrs[3] = {d_origins, d_directions, d_hits};
  for (const void* p : ptrs) {
    if (!p) return fail(r, DFC_E_INVALID_ARG, "ray or hit pointer == NULL");
    if (reinterpret_cast<uintptr_t>(p) % 16u) return fail(r, DFC_E_INVALID_ARG, "ray and hit arrays must be 16-byte aligned");
    if (!device_pointer_on(p, r->device))
      return fail(r, DFC_E_INVALID_ARG, "ray and hit arrays must be device memory of the handle's device");
  }
  const unsigned n = (unsigned)count;
  k_noalloc_prepare<<<(n + 255u) / 256u, 256, 0, r->stream>>>(scratch, n);
  TraceArgs t{};
  t.scene = r->scene.view;
  t.ray_list = scratch + kNoAllocHeader;
  t.ray_count = scratch;
  t.fetch = scratch + 1;
  t.overflow = scratch + 2;
  t.ray_o = reinterpret_cast<const float4*>(d_origins);
  t.ray_d = reinterpret_cast<const float4*>(d_directions);
  t.hits = reinterpret_cast<float4*>(d_hits);
  t.paths = n;
  trace_kernel(r)<<<r->sm_count * r->trace_blocks, kTraceThreads, 0, r->stream>>>(t);
  DFC_CK(cudaGetLastError(), "dfc_trace_rays_noalloc launch");
  unsigned ov = 0;
  DFC_CK(cudaMemcpyAsync(&ov, scratch + 2, 4, cudaMemcpyDeviceToHost, r->stream), "dfc_trace_rays_noalloc readback");
  DFC_CK(cudaStreamSynchronize(r->stream), "dfc_trace_rays_noalloc");
  if (ov) return fail(r, DFC_E_TIMEOUT, "traversal stack bound exceeded on " + std::to_string(ov) + " node visits");
  return DFC_OK;
}
