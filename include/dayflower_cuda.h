/*
 * dayflower_cuda.h - C ABI of libdayflower_cuda, the B200 render path that
 * stands in for Dayflower's GPURenderer.
 *
 * Every entry point takes plain pointers and sizes.  Each one names the member
 * of the reference's GPURenderer API (org.dayflower.renderer.gpu, paths are
 * relative to src/main/java/org/dayflower/) that it replaces.
 *
 * Ownership: the caller owns every host array it passes; the library copies
 * what it keeps before returning.  The library owns all device memory.
 *
 * Errors: every call returns a dfc_status.  DFC_E_INVALID_ARG stands where the
 * reference throws NullPointerException or IllegalArgumentException,
 * DFC_E_UNSUPPORTED where the scene uses a shape, material, texture or light
 * this renderer does not implement.  dfc_last_error() gives the message of the
 * last failing call on a handle.
 *
 * Threading: a handle is not re-entrant (calls on one handle take its lock);
 * dfc_render_shutdown() may be called from any thread while dfc_render() runs.
 * Different handles are independent.
 */
#ifndef DAYFLOWER_CUDA_H
#define DAYFLOWER_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum dfc_status {
  DFC_OK = 0,
  DFC_E_INVALID_ARG = 1,   /* NullPointerException / IllegalArgumentException */
  DFC_E_UNSUPPORTED = 2,   /* unknown or unimplemented shape, material, texture or light id */
  DFC_E_OOM = 3,           /* device (or page-locked host staging) allocation failed */
  DFC_E_CUDA = 4,          /* any other CUDA runtime error */
  DFC_E_TIMEOUT = 5,       /* a device-side iteration bound ran out (traversal stack overflow etc.) */
  DFC_E_STOPPED = 6,       /* dfc_render_shutdown() ended the render early */
  DFC_E_STATE = 7          /* call out of order (e.g. render before setup) */
} dfc_status;

/* RenderingAlgorithm ordinals, renderer/RenderingAlgorithm.java:33-53 */
enum {
  DFC_AMBIENT_OCCLUSION = 0,
  DFC_DEPTH_CAMERA = 1,
  DFC_PATH_TRACING = 2,
  DFC_RAY_CASTING = 3,
  DFC_RAY_TRACING = 4
};

/* Tone mapper ids, renderer/gpu/AbstractGPURenderer.java:54-79 */
enum {
  DFC_TONE_MAPPER_FILMIC_CURVE_ACES_MODIFIED_VERSION_1 = 0,
  DFC_TONE_MAPPER_NONE = 1,
  DFC_TONE_MAPPER_REINHARD = 2,
  DFC_TONE_MAPPER_REINHARD_MODIFIED_VERSION_1 = 3,
  DFC_TONE_MAPPER_REINHARD_MODIFIED_VERSION_2 = 4,
  DFC_TONE_MAPPER_UNREAL_3 = 5
};

/* Element types for dfc_scene_put */
enum { DFC_F32 = 0, DFC_I32 = 1 };

typedef struct dfc_renderer dfc_renderer;

/* new GPURenderer(rendererObserver), renderer/gpu/GPURenderer.java:43-57.
 * Binds CUDA device `device`.  Defaults follow AbstractGPURenderer.java:148-158:
 * 800x800 image, PATH_TRACING, maximum distance 20, maximum bounce 20,
 * Russian roulette from bounce 5, 10 AO samples, tone mapper NONE. */
int dfc_create(int device, dfc_renderer** out);

/* dispose(), renderer/gpu/AbstractKernel.java:166.  Frees all device memory. */
int dfc_destroy(dfc_renderer* r);

/* Message of the last failing call on this handle ("" if none). */
const char* dfc_last_error(const dfc_renderer* r);

/* setScene(scene) part 1: one Aparapi put() of a CompiledScene array,
 * renderer/gpu/AbstractSceneKernel.java:1777-1852.  `name` is the kernel field
 * the reference uploads (e.g. "primitiveArray", "shape3FTriangle3FArray");
 * `type` is DFC_F32 or DFC_I32; `count` elements are copied into page-locked
 * host memory that the handle keeps for the next commits (the upload then runs
 * by DMA); DFC_E_OOM if that memory cannot be had. */
int dfc_scene_put(dfc_renderer* r, const char* name, const void* data, int64_t count, int type);

/* setScene(scene) part 2: decodes the staged arrays, builds the acceleration
 * structure and uploads the scene.  layout_version 1 is the reference packing
 * (scene/compiler/*, utility/Ints.java:237/:258); 2 widens material records to
 * four int32 lanes per packed slot (no 8-bit texture limit). */
int dfc_scene_commit(dfc_renderer* r, int layout_version);

/* setImage(), AbstractGPURenderer.java:417-440: film resolution.  0,0 takes the
 * resolution from the compiled camera. */
int dfc_set_image(dfc_renderer* r, int width, int height);

/* setMaximumBounce :448, setMinimumBounceRussianRoulette :468,
 * setRenderingAlgorithm :504, setSamples :515 (AO rays), setMaximumDistance :458,
 * setToneMapper :524, setPreviewMode :478 */
int dfc_set_maximum_bounce(dfc_renderer* r, int maximum_bounce);
int dfc_set_minimum_bounce_russian_roulette(dfc_renderer* r, int minimum_bounce);
int dfc_set_rendering_algorithm(dfc_renderer* r, int algorithm);
int dfc_set_samples(dfc_renderer* r, int samples);
int dfc_set_maximum_distance(dfc_renderer* r, float maximum_distance);
int dfc_set_tone_mapper(dfc_renderer* r, int tone_mapper);
int dfc_set_preview_mode(dfc_renderer* r, int preview_mode);

/* Seed of the counter-based random numbers (no reference counterpart: the
 * Aparapi kernel seeds its per-pixel generators from ThreadLocalRandom). */
int dfc_set_seed(dfc_renderer* r, uint32_t seed);

/* Per-stage device timing of later dfc_render calls (CUDA events around every
 * launch; no reference counterpart: the reference times whole passes only,
 * AbstractGPURenderer.java:281-291).  Read with dfc_read_stage_times. */
int dfc_set_stage_timing(dfc_renderer* r, int on);

/* setup(), AbstractGPURenderer.java:532: allocates the film and the wavefront
 * queues for the current image and clears the film. */
int dfc_setup(dfc_renderer* r);

/* render(renderPasses), AbstractGPURenderer.java:322: renderPasses passes of one
 * sample per pixel each.  *completed receives the passes done (may be NULL).
 * Returns DFC_E_STOPPED if dfc_render_shutdown() interrupted it. */
int dfc_render(dfc_renderer* r, int render_passes, int* completed);

/* render(renderPasses) with a RendererObserver, AbstractGPURenderer.java:231-297
 * and :322-332 (render(int) is a loop of render()).  Each pass calls fn, on the
 * caller's thread, as the reference notifies its observer:
 *   DFC_OBSERVE_PASS_PROGRESS (progress 0.0)   onRenderPassProgress(renderer, renderPass, 0.0)
 *   ... the pass, then the image update (doUpdateImageF, :668-712) ...
 *   DFC_OBSERVE_PASS_PROGRESS (progress 1.0)   onRenderPassProgress(renderer, renderPass, 1.0)
 *   DFC_OBSERVE_DISPLAY (rgba = the image)     onRenderDisplay(renderer, image)
 *   DFC_OBSERVE_PASS_COMPLETE (millis)         onRenderPassComplete(renderer, renderPass, elapsedTimeMillis)
 * and the first pass after dfc_setup/dfc_clear starts with DFC_OBSERVE_DISPLAY
 * of the cleared image (render_pass 0), as render() does after filmClear.
 * render_pass counts from 1 after a clear.  The host waits for every pass, so
 * an observed render is slower than dfc_render by one RGBA8 resolve and
 * read-back per pass.  fn runs with the handle locked: it may call
 * dfc_render_shutdown, and any other call on the same handle returns
 * DFC_E_STATE.  rgba (width * height * 4 bytes, rows top to bottom) is valid
 * only during the call. */
typedef enum dfc_observe_event {
  DFC_OBSERVE_PASS_PROGRESS = 0,
  DFC_OBSERVE_DISPLAY = 1,
  DFC_OBSERVE_PASS_COMPLETE = 2
} dfc_observe_event;

typedef struct dfc_pass_event {
  int event;             /* dfc_observe_event */
  int render_pass;
  double progress;       /* PASS_PROGRESS: 0.0 before the pass, 1.0 after it */
  double millis;         /* PASS_COMPLETE: host milliseconds of the pass and its image update */
  const uint8_t* rgba;   /* DISPLAY: the RGBA8 image (tone mapped, sRGB) */
  int width, height;
} dfc_pass_event;

typedef void (*dfc_observer_fn)(void* user, const dfc_pass_event* event);

int dfc_render_observed(dfc_renderer* r, int render_passes, dfc_observer_fn fn, void* user, int* completed);

/* renderShutdown(), AbstractGPURenderer.java:342: asynchronous stop request. */
int dfc_render_shutdown(dfc_renderer* r);

/* clear(), AbstractGPURenderer.java:409: resets the film (next render starts at pass 0). */
int dfc_clear(dfc_renderer* r);

/* updateCamera(), AbstractSceneKernel.java:278: new 19-float compiled camera. */
int dfc_update_camera(dfc_renderer* r, const float* camera19);

/* updateMatrix44Fs(), AbstractSceneKernel.java:292: new object-to-world/world-to-object
 * pairs, 32 floats per primitive, primitive_count * 32 floats. */
int dfc_update_matrices(dfc_renderer* r, const float* matrices, int64_t primitive_count);

/* getImage(): the film as RGBA8 after tone mapping and sRGB encoding
 * (renderer/gpu/AbstractImageKernel.java:1104-1160), width*height*4 bytes. */
int dfc_read_image_rgba8(dfc_renderer* r, uint8_t* dst, int64_t capacity_bytes);

/* The radiance film: per pixel sum of accepted samples (3 floats), sum of their
 * squares (3 floats) and sample count (1 float), width*height*7 floats. */
int dfc_read_film(dfc_renderer* r, float* dst, int64_t capacity_floats);

/* Film of later setup() calls: 0 (default) the per-pixel box film read by
 * dfc_read_film; 1 the CPU renderer's film (image/PixelImageF.java:569
 * filmAddColorXYZ, GaussianFilter2F(2, 2, 2)): each sample is converted to XYZ
 * and splatted, filter-weighted, to the pixels within radius 2 of its film
 * position; dfc_read_image_rgba8 then resolves it as PixelImageF.filmRender
 * (XYZ -> sRGB over the weight sum, sRGB gamma, no tone mapper). */
int dfc_set_film_filter(dfc_renderer* r, int filter);

/* Builder of the triangle-mesh hierarchies for later scene commits: 0 the
 * host binned-SAH builder, 1 (default) the device builder (Morton-ordered
 * radix tree collapsed to 4-wide nodes, built from the uploaded triangle
 * records; about 9x faster to commit a 2M-triangle mesh, about 3% slower to
 * trace; its temporaries come from a per-device memory pool that keeps up to
 * 1 GiB of device memory reserved between commits, for the life of the
 * process).  The
 * reference builds its mesh hierarchies on the host (BVHNode3Fs.create,
 * geometry/boundingvolume/hierarchy/BVHNode3Fs.java:63-237); both produce the
 * same node format and the same hits. */
#define DFC_BVH_HOST 0
#define DFC_BVH_DEVICE 1
int dfc_set_bvh_builder(dfc_renderer* r, int builder);

/* The Gaussian pixel film: per pixel X, Y, Z sums and the filter weight sum,
 * width*height*4 floats (film filter 1 only). */
int dfc_read_pixel_film(dfc_renderer* r, float* dst, int64_t capacity_floats);

/* Per-pixel primitive index hit by the first pass's primary ray (-1 on a miss)
 * and its world-space distance.  Either pointer may be NULL. */
int dfc_read_primary_hits(dfc_renderer* r, int32_t* prim, float* t, int64_t capacity);

/* Counters since the last dfc_setup/dfc_clear: passes, paths, rays traced,
 * kernel launches.  out[4]. */
int dfc_read_counters(dfc_renderer* r, int64_t* out4);

/* Device time of the last dfc_render call, split by stage in milliseconds:
 * out[0] total, [1] ray generation, [2] traversal, [3] shading, [4] film.
 * Stages [1]-[4] are filled only while dfc_set_stage_timing is on. */
int dfc_read_stage_times(dfc_renderer* r, float* out5);

/* Per-kernel device time of the last dfc_render call (while dfc_set_stage_timing
 * is on; CUDA events around every launch), launches, and the work items those
 * kernels processed since the last dfc_setup/dfc_clear; index 0 is the whole
 * call (its time, all launches, paths).  Kernel kinds and their items:
 *   DFC_KERNEL_RAYGEN        camera paths started
 *   DFC_KERNEL_TRACE         rays traced
 *   DFC_KERNEL_SHADE         shade work items (also the two sort kernels')
 *   DFC_KERNEL_FILM          (resolves; no items)
 *   DFC_KERNEL_SORT_COUNT, DFC_KERNEL_SORT_SCATTER  material sort of the work items
 *   DFC_KERNEL_RAY_LIST      rays listed in path order (all but the camera rays)
 * ms, launches, items: n entries each (any may be NULL), n <= DFC_KERNEL_KINDS.
 * No counterpart in the reference (it times whole passes only). */
enum {
  DFC_KERNEL_RAYGEN = 1,
  DFC_KERNEL_TRACE = 2,
  DFC_KERNEL_SHADE = 3,
  DFC_KERNEL_FILM = 4,
  DFC_KERNEL_SORT_COUNT = 5,
  DFC_KERNEL_SORT_SCATTER = 6,
  DFC_KERNEL_RAY_LIST = 7,
  DFC_KERNEL_KINDS = 8
};
int dfc_read_kernel_stats(dfc_renderer* r, float* ms, int64_t* launches, int64_t* items, int n);

/* Host wall time of the last dfc_scene_commit in milliseconds: out[0] decode
 * and acceleration builds, [1] of which bottom-level (mesh) builds, [2] of
 * which the top-level build, [3] upload to the device.  No counterpart in the
 * reference (setScene there is untimed). */
int dfc_read_commit_times(dfc_renderer* r, float* out4);

/* Closest-hit traversal of `count` caller-supplied rays against the committed
 * scene, with no device allocation.  No counterpart in the reference.
 *
 * For callers that must not have the library allocate device memory: a host
 * that owns a fixed device arena and hands out every byte itself, or an
 * interactive loop that cannot afford cudaMalloc/cudaFree, which may
 * synchronise the whole device.  The traversal scratch (ray list, ray count,
 * fetch cursor, overflow flag) is a static device array of 4 MiB + 256 B in
 * this library, one per device per process.
 *
 * All three arrays are device memory of the handle's device, 16-byte aligned,
 * `count` float4 each:
 *   d_origins[i]    = (x, y, z, unused)
 *   d_directions[i] = (dx, dy, dz, tmax)   hits need t in (0.0001, tmax)
 *   d_hits[i]       = (t, primitive index as int32 bits or -1 on a miss,
 *                      shape-specific int32 bits, t in object space)
 * t is the ray parameter, the distance for a unit direction.  Nothing the
 * caller passes must start at zero: the call zeroes the scratch's fetch cursor
 * and overflow flag itself before it traverses.
 *
 * Limit: count <= 1048576 (DFC_E_INVALID_ARG beyond, with the limit in the
 * message; split larger batches).  count == 0 does only the set-up.
 * Set-up: the first call on each device resolves the scratch address with
 * cudaGetSymbolAddress and loads the kernels; make that first call (count 0
 * suffices) before any stream capture begins on that device.
 * Concurrency: calls on one device that overlapped in time would race on the
 * one scratch array, so the library runs them one after another under a
 * process-wide lock.  The call uses the handle's stream and returns once the
 * hits are written; make the rays visible to that stream first (synchronise
 * the stream that produced them).  DFC_E_STATE before dfc_scene_commit,
 * DFC_E_TIMEOUT if the traversal stack bound ran out. */
int dfc_trace_rays_noalloc(dfc_renderer* r, const float* d_origins, const float* d_directions, float* d_hits,
                           int64_t count);

/* ------------------------------------------------------------------------
 * Batch and serving engine.  The reference renders one image per
 * GPURenderer, one pass per execute() (AbstractGPURenderer.java:231-297), so
 * these entry points have no single counterpart: each render job is what a
 * GPURenderer would do for setScene(scene) + setImage(w, h) +
 * setMaximumBounce(b) + setMinimumBounceRussianRoulette(r) + setup() +
 * render(spp) with PATH_TRACING, and the engine runs many such jobs at once in
 * one wavefront of path slots.  A job's samples are those the per-job renderer
 * draws for the same seed, so its image is the same alone, in a mix, or on a
 * GPURenderer handle, up to the order of the film's float additions.
 *
 * Scenes are committed once and stay resident, reference-counted by the
 * caller and by every unfinished job on them.  Jobs are admitted against a
 * device-memory budget (wavefront + resident scenes + per-job films) and
 * start their paths in the running wavefront at the next bounce iteration.
 * Films can be read while a job runs (a progressive image).
 *
 * Threading: every dfc_engine_* / dfc_job_* call is thread-safe.  Either call
 * dfc_engine_run() (the wavefront runs in the calling thread until every
 * submitted job is finished) or dfc_engine_start()/dfc_engine_stop() (it runs
 * on an engine thread; jobs may be submitted from any thread meanwhile).
 * ------------------------------------------------------------------------ */
typedef struct dfc_engine dfc_engine;

enum { DFC_JOB_QUEUED = 0, DFC_JOB_RUNNING = 1, DFC_JOB_DONE = 2, DFC_JOB_CANCELLED = 3, DFC_JOB_FAILED = 4 };

typedef struct dfc_job_desc {
  int32_t scene;                            /* id from dfc_engine_scene_commit */
  int32_t width, height;                    /* film resolution (the camera's field of view is kept) */
  int32_t samples;                          /* samples per pixel: render(samples) on a GPURenderer */
  int32_t maximum_bounce;                   /* setMaximumBounce */
  int32_t minimum_bounce_russian_roulette;  /* setMinimumBounceRussianRoulette */
  uint32_t seed;                            /* seed of the counter-based random numbers (dfc_set_seed) */
  int32_t kind;                             /* DFC_JOB_PATH_TRACING (0) or another DFC_JOB_* algorithm */
  int32_t ambient_occlusion_samples;        /* AMBIENT_OCCLUSION: setSamples (rays per camera sample, 1 .. 4096) */
  float maximum_distance;                   /* AMBIENT_OCCLUSION: setMaximumDistance (<= 0: occlusion only) */
} dfc_job_desc;

/* Rendering algorithm of an engine job (dfc_job_desc.kind), the
 * RenderingAlgorithm of setRenderingAlgorithm (renderer/gpu/
 * AbstractGPURenderer.java:504) that GPURenderer.run dispatches on
 * (renderer/gpu/GPURenderer.java:65-77), each shaded as the per-job renderer
 * shades it: PATH_TRACING in the bounce wavefront; RAY_CASTING and
 * DEPTH_CAMERA end at their camera ray; AMBIENT_OCCLUSION and RAY_TRACING
 * trace their camera ray in the wavefront and then their occlusion rays or
 * their ray tree in one step on the path's thread. */
#define DFC_JOB_PATH_TRACING 0
#define DFC_JOB_RAY_CASTING 1
#define DFC_JOB_DEPTH_CAMERA 2
#define DFC_JOB_AMBIENT_OCCLUSION 3
#define DFC_JOB_RAY_TRACING 4

typedef struct dfc_job_info {
  int32_t state;                 /* DFC_JOB_* */
  int32_t scene;
  int64_t paths_total;           /* width * height * samples */
  int64_t paths_done;            /* retired paths as of the engine's last progress read */
  double submit_s, admit_s, done_s;  /* engine clock in seconds (0 until reached) */
} dfc_job_info;

/* Scheduling policies: the host hands the device runs ("segments") of
 * consecutive paths of one job, at most `lookahead_paths` ahead of the paths
 * started so far.  ROUND_ROBIN gives every admitted job one segment in turn
 * (processor sharing: small jobs finish early while large ones run); FIFO
 * finishes jobs in admission order; SHORTEST_FIRST gives the next segment to
 * the admitted job with the fewest paths left to hand out (small jobs stay
 * fast under overload, large ones wait; a small lookahead_paths lets new
 * arrivals overtake sooner). */
enum { DFC_SCHEDULE_ROUND_ROBIN = 0, DFC_SCHEDULE_FIFO = 1, DFC_SCHEDULE_SHORTEST_FIRST = 2 };

typedef struct dfc_engine_config {
  int64_t capacity;              /* path slots of the wavefront (0: default 2^20) */
  int32_t trace_blocks_per_sm;   /* resident blocks per SM of the traversal kernel (0: occupancy maximum) */
  int32_t shade_blocks_per_sm;   /* blocks per SM of the shade kernels (0: 32); the sort's kernels use at most 8 */
  int32_t shade_threads;         /* threads per shade block: 128 or 256 (0: 256) */
  int32_t iterations_per_launch; /* bounce iterations per CUDA-graph launch, even (0: 4) */
  int32_t policy;                /* DFC_SCHEDULE_* */
  int32_t reserved;              /* 0 */
  int64_t segment_paths;         /* paths per segment (0: 65536) */
  int64_t lookahead_paths;       /* appended but unstarted paths the host keeps queued (0: 8 x capacity) */
} dfc_engine_config;

typedef struct dfc_engine_stats {
  int64_t iterations, graph_launches, kernel_launches;
  int64_t paths_retired, rays;
  int64_t jobs_submitted, jobs_done;
  int64_t device_bytes_used, device_bytes_budget;
  int64_t overflow;              /* traversal stack bound hits (0 in a correct run) */
  double busy_s;                 /* engine-clock seconds with work on the device */
} dfc_engine_stats;

/* Creates an engine on CUDA device `device` that admits work while its
 * device memory (wavefront, resident scenes, job films) stays within
 * `memory_budget_bytes` (0: 90% of the device's free memory). */
int dfc_engine_create(int device, int64_t memory_budget_bytes, dfc_engine** out);
/* Stops the engine thread if running, frees all device memory. */
int dfc_engine_destroy(dfc_engine* e);
const char* dfc_engine_last_error(const dfc_engine* e);

/* Scene staging and commit, as dfc_scene_put/dfc_scene_commit; the committed
 * scene gets an id and one caller reference.  DFC_E_OOM if it would exceed the
 * budget. */
int dfc_engine_scene_put(dfc_engine* e, const char* name, const void* data, int64_t count, int type);
int dfc_engine_scene_commit(dfc_engine* e, int layout_version, int32_t* scene_id);
/* Builder of the triangle-mesh hierarchies of later dfc_engine_scene_commit
 * calls (DFC_BVH_HOST or DFC_BVH_DEVICE, as dfc_set_bvh_builder). */
int dfc_engine_set_bvh_builder(dfc_engine* e, int builder);
/* Drops the caller's reference; the scene is freed once no unfinished job uses it. */
int dfc_engine_scene_release(dfc_engine* e, int32_t scene_id);

/* Wavefront shape (see dfc_engine_config); takes effect at the next run. */
int dfc_engine_configure(dfc_engine* e, const dfc_engine_config* cfg);
int dfc_engine_get_config(dfc_engine* e, dfc_engine_config* out);
/* Picks capacity, block shapes and iterations per launch by timing
 * candidates on `n` sample jobs (each candidate renders all of them), keeps
 * the fastest and writes it to *out (may be NULL).  With `cache_path` set, a
 * result stored there under `key` for this GPU is used instead of timing, and
 * a new result is stored.  Only while the engine has no other jobs. */
int dfc_engine_autotune(dfc_engine* e, const dfc_job_desc* jobs, int n, const char* cache_path, const char* key,
                        dfc_engine_config* out);

/* Queues a job; *job_id receives its id.  DFC_E_INVALID_ARG for a bad
 * descriptor or unknown scene. */
int dfc_job_submit(dfc_engine* e, const dfc_job_desc* desc, int64_t* job_id);
int dfc_job_get_info(dfc_engine* e, int64_t job_id, dfc_job_info* out);
/* Blocks until the job is done, cancelled or failed, or `timeout_s` passed
 * (DFC_E_TIMEOUT).  Needs a running engine (dfc_engine_start) or another
 * thread in dfc_engine_run. */
int dfc_job_wait(dfc_engine* e, int64_t job_id, double timeout_s);
/* Stops handing out the job's remaining paths; it ends as DFC_JOB_CANCELLED. */
int dfc_job_cancel(dfc_engine* e, int64_t job_id);
/* The job's film as dfc_read_film lays it out (width*height*7 floats), read
 * while it runs (a progressive image) or after it finished. */
int dfc_job_read_film(dfc_engine* e, int64_t job_id, float* dst, int64_t capacity_floats);
/* Tone-mapped sRGB RGBA8 of the job's film, width*height*4 bytes. */
int dfc_job_read_image_rgba8(dfc_engine* e, int64_t job_id, int tone_mapper, uint8_t* dst, int64_t capacity_bytes);
/* Frees the job's film and forgets it (a running job is cancelled first). */
int dfc_job_release(dfc_engine* e, int64_t job_id);

/* Runs the wavefront in the calling thread until every submitted job is
 * finished (DFC_E_TIMEOUT after `timeout_s` seconds, <= 0: no limit). */
int dfc_engine_run(dfc_engine* e, double timeout_s);
/* Runs the wavefront on an engine thread until dfc_engine_stop. */
int dfc_engine_start(dfc_engine* e);
int dfc_engine_stop(dfc_engine* e);
int dfc_engine_get_stats(dfc_engine* e, dfc_engine_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* DAYFLOWER_CUDA_H */
