// Kernel argument blocks and entry points of the wavefront render path.
#pragma once

#include <cuda_runtime.h>

#include "dfc_scene.h"

namespace dfc {

enum { DFC_ALGO_AO = 0, DFC_ALGO_DEPTH = 1, DFC_ALGO_PATH = 2, DFC_ALGO_RAY_CASTING = 3, DFC_ALGO_RAY_TRACING = 4 };
// DJob::kind (the C ABI's DFC_JOB_* values)
enum : int { kJobPathTracing = 0, kJobRayCasting = 1, kJobDepthCamera = 2, kJobAmbientOcclusion = 3, kJobRayTracing = 4 };

// Path flags (PathMeta.w)
enum : unsigned { kFlagAlive = 1u, kFlagSpecular = 2u, kFlagPendShadow = 4u, kFlagPendMis = 8u, kFlagShadowAny = 16u, kFlagNoSample = 32u };

// One render job of the batch/serving engine as the kernels read it (a ring
// of power-of-two capacity indexed by sequence number & mask).  Path q of a
// job is pixel q % pixels of sample q / pixels (sample-major, so a partial
// film is a progressive image).
struct DJob {
  float camera[19];          // the scene's compiled camera with the job's resolution in [17], [18]
  int scene;                 // index into the engine's scene table
  unsigned width, pixels;
  int max_bounce, min_rr;
  uint32_t seed;
  int kind;                  // kJob*
  int ao_samples;            // AMBIENT_OCCLUSION: rays per camera sample
  float ao_distance;         //                    maximum distance (<= 0: occlusion only)
  unsigned cancelled;        // 1: start no more paths of this job (the plan skips them)
  float4* film_sum;          // per pixel: sum of accepted samples (xyz), count (w)
  float4* film_sq;           // per pixel: sum of squares (xyz)
};

// A run of consecutive paths of one job in the engine's global path sequence:
// global indices [start, start + count) are the job's paths [q0, q0 + count).
// The host appends segments (its scheduling policy decides whose) into a ring
// indexed by segment sequence number & mask; starts increase with the
// sequence number.
struct DSegment {
  unsigned long long start;
  unsigned long long q0;
  unsigned long long count;
  unsigned job;              // job ring index
  unsigned pad;
};

// Words the host writes between wavefront iterations (stream-ordered copies).
struct BatchControl {
  unsigned long long admitted;  // end of the last appended segment
  unsigned seg_lo, seg_hi;      // sequence numbers of the segments that may still hand out paths
};

// Words the wavefront iterations keep on the device.
struct BatchState {
  unsigned long long cursor;    // next global path index to hand out
  unsigned long long rays;      // rays traced (all iterations)
  unsigned long long retired;   // paths retired
  unsigned free_top;            // slots on the free stack
  unsigned regen_k;             // plan -> regen: paths to start this iteration
  unsigned regen_base;          //                first free-stack entry they take
  unsigned iterations;
  unsigned long long regen_cursor;  //            global index of the first of them
};

struct TraceArgs {
  SceneView scene;
  // batch engine only: per-slot job, job ring and scene table (the scene of
  // a ray is scenes[jobs[slot_job[slot]].scene])
  const SceneView* scenes;
  const DJob* jobs;
  const unsigned* slot_job;
  const unsigned* ray_list;
  const unsigned* ray_count;
  const float4* ray_o;  // 3 slots per path: [type * paths + p]
  const float4* ray_d;
  float4* hits;         // t_world, prim (int bits, -1 miss), aux (int bits), t_object
  unsigned paths;
  unsigned* overflow;
  unsigned* fetch;      // rays handed out so far in this launch (starts at 0)
};

struct RaygenArgs {
  SceneView scene;
  unsigned paths, pixels, width, sample_base;
  uint32_t seed;
  float4* beta;
  float4* radiance;
  uint4* meta;          // pixel, rng key, bounce | step << 16, flags
  float4* ray_o;
  float4* ray_d;
  unsigned* ray_list;
  unsigned* ray_count;
  unsigned* work_list;
  unsigned* work_count;
};

struct ShadeArgs {
  SceneView scene;
  // PixelImageF film (Gaussian XYZ splat): filter table [0, 256) and sRGB -> XYZ
  // matrix [256, 265); nullptr: the per-pixel box film (sum, sum of squares)
  const float* pixel_film;
  unsigned width, height;
  // batch engine only (see TraceArgs); retired slots go back on the free stack
  const SceneView* scenes;
  const DJob* jobs;
  const unsigned* slot_job;
  unsigned* free_stack;
  unsigned* free_top;
  unsigned long long* job_done;  // per job ring entry: paths retired
  BatchState* state;
  unsigned paths, pixels;
  int max_bounce, min_rr, preview, last_step, record_primary, ao_samples;
  const unsigned* work_list;
  const unsigned* work_count;
  // When set, the kernel shades only the work items of sort keys
  // [range_lo, range_hi): a range of the sorted work list found from these
  // bin counts (SortArgs::bins of this step).
  const unsigned* range_bins;
  int range_lo, range_hi;
  unsigned* overflow;  // batch engine: traversal stack bound exceeded (the inline AO and ray-tracing kernel)
  unsigned* next_work_list;
  unsigned* next_work_count;
  unsigned* next_ray_list;
  unsigned* next_ray_count;
  // When set (per-job renderer), shading records each path's new rays here
  // (bit 0 extension, 1 shadow, 2 MIS, 3 shadow is any-hit) instead of
  // appending them, and k_ray_list_ordered builds the next ray list in path
  // order.  With ordered_work set, bit 4 (kMaskKeep) marks a path that is
  // shaded again and the next work list is built in path order the same way.
  unsigned char* ray_mask;
  int ordered_work;
  float4* beta;
  float4* radiance;
  uint4* meta;
  float4* ray_o;
  float4* ray_d;
  const float4* hits;
  float4* pend_shadow;
  float4* pend_mis;
  float4* film_sum;
  float4* film_sq;
  int* primary_prim;
  float* primary_t;
  float4* ao_o;
  float4* ao_d;
};

struct AoArgs {
  SceneView scene;
  unsigned paths;
  int samples;
  float max_distance;
  const float4* radiance;
  const float4* ao_o;
  const float4* ao_d;
  float* ao_value;
  unsigned* overflow;
};

// Material sort of a shade work list by the material kind of the extension
// hit.  The keys put the kinds whose BSDF has at most two lobes (no BSDF,
// matte, mirror, glass, metal, plastic: kinds 0 .. kSimpleKinds - 1) first,
// then a miss, then a path with nothing left to shade (pending light rays
// only), then the other kinds; the first kSimpleBins keys are shaded by the
// two-lobe kernel, the rest by the general one.
constexpr int kSortBins = kMatKinds + 3;
constexpr int kKeyInline = kMatKinds + 2;  // batch engine: AMBIENT_OCCLUSION and RAY_TRACING paths (k_shade_inline_batch)
constexpr int kSimpleKinds = kMatPlastic + 1;
constexpr int kKeyMiss = kSimpleKinds;
constexpr int kKeyNothing = kSimpleKinds + 1;
constexpr int kSimpleBins = kSimpleKinds + 2;
__host__ __device__ inline int material_sort_key(int kind) { return kind < kSimpleKinds ? kind : kind + 2; }
struct SortArgs {
  SceneView scene;
  const SceneView* scenes;  // batch engine only (see TraceArgs)
  const DJob* jobs;
  const unsigned* slot_job;
  unsigned paths;
  const unsigned* work_list;
  const unsigned* work_count;
  const uint4* meta;
  const float4* hits;
  unsigned char* keys;     // one per work item
  unsigned* bins;          // kSortBins counts, then kSortBins cursors
  unsigned* sorted;        // the work list in key order
};
__global__ void k_sort_count(SortArgs a);
__global__ void k_sort_count_batch(SortArgs a);
__global__ void k_sort_scatter(SortArgs a);

// Batch engine: one wavefront iteration is
//   plan -> regen -> trace -> sort count -> sort scatter -> shade
// with the lists and counters of parity (iteration & 1).
struct BatchArgs {
  const DJob* jobs;
  const DSegment* segs;
  unsigned seg_mask;
  const BatchControl* ctl;
  BatchState* state;
  unsigned long long* job_done;  // per job ring entry: paths retired (or skipped by a cancel)
  unsigned* free_stack;
  unsigned* slot_job;
  unsigned capacity;
  unsigned* counts_cur;    // {ray count, work count, fetch, -} of this iteration
  unsigned* counts_next;   // of the next one (zeroed by plan)
  unsigned* sort_bins;     // 2 * kSortBins of this iteration (zeroed by plan)
  float4* beta;
  float4* radiance;
  uint4* meta;
  float4* ray_o;
  float4* ray_d;
  unsigned* ray_list;      // of this iteration
  unsigned* work_list;
};
__global__ void k_batch_init(BatchArgs a);
__global__ void k_batch_plan(BatchArgs a);
__global__ void k_batch_regen(BatchArgs a);

__global__ void k_raygen(RaygenArgs a);
// Closest/any hit of the listed rays.  k_trace_records also tests disk,
// cylinder, cone, paraboloid, hyperboloid, cuboid and torus primitives; launch
// it when the scene has any (SceneView has no flag for it: the host knows).
__global__ void k_trace(TraceArgs a);
__global__ void k_trace_records(TraceArgs a);
__global__ void k_trace_batch(TraceArgs a);          // batch engine: scene per ray from the job table
__global__ void k_trace_batch_records(TraceArgs a);
__global__ void k_shade_path(ShadeArgs a);
__global__ void k_shade_path_records(ShadeArgs a);  // with the disk ... torus surfaces
// two-lobe BSDFs only (the material kinds below kSimpleKinds), in registers, at four blocks per SM
__global__ void k_shade_path_simple(ShadeArgs a);
__global__ void k_shade_path_simple_records(ShadeArgs a);
__global__ void k_shade_path_batch_simple(ShadeArgs a);
__global__ void k_shade_path_batch_simple_records(ShadeArgs a);
__global__ void k_shade_path_batch(ShadeArgs a);     // batch engine: scene, film and limits per path from the job table
__global__ void k_shade_path_batch_records(ShadeArgs a);
// with record shapes and materials evaluated per hit (textures, modifiers, composite materials)
__global__ void k_shade_path_textured(ShadeArgs a);
__global__ void k_shade_path_batch_textured(ShadeArgs a);
__global__ void k_shade_primary(ShadeArgs a, int algorithm);
// The next step's ray list from ShadeArgs::ray_mask, paths in index order
// within each block of kRayListBlock paths.
constexpr int kRayListBlock = 256;
constexpr unsigned kMaskKeep = 16u;
__global__ void k_ray_list_ordered(const unsigned char* ray_mask, unsigned paths, unsigned* ray_list, unsigned* ray_count,
                                   unsigned* work_list, unsigned* work_count);
__global__ void k_trace_ao(AoArgs a);
// RAY_TRACING (scene/Scene.java:786 doRadianceRayTracer): one thread per camera
// sample walks the sample's specular reflection/transmission tree depth first.
__global__ void k_ray_trace(ShadeArgs a, unsigned* overflow, unsigned long long* rays);
__global__ void k_ao_resolve(ShadeArgs a, const float* ao_value, int samples);
// Batch engine: AMBIENT_OCCLUSION and RAY_TRACING paths, finished in one step (sort key kKeyInline).
__global__ void k_shade_inline_batch(ShadeArgs a);
// film_consts: nullptr for the box film (mean, tone mapper, sRGB); else the
// PixelImageF resolve (filmRender: XYZ -> RGB over the weight sum, negative
// parts dropped, sRGB) with the XYZ -> sRGB matrix at film_consts[265, 274).
__global__ void k_resolve_rgba8(const float4* film_sum, int pixels, int tone_mapper, float exposure, uchar4* out,
                                const float* film_consts = nullptr);
constexpr int kFilmTable = 16;  // Filter2F.TABLE_SIZE

constexpr int kTraceThreads = 128;

}  // namespace dfc
