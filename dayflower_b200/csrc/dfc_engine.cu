// Batch and serving engine of libdayflower_cuda: many render jobs in one
// wavefront of path slots.
//
// Device side (dfc_kernels.cu): a fixed pool of `capacity` path slots.  One
// bounce iteration is
//   k_batch_plan -> k_batch_regen -> k_trace_batch -> k_sort_count_batch
//   -> k_sort_scatter -> k_shade_path_batch_simple -> k_shade_path_batch
//   -> k_shade_inline_batch (AMBIENT_OCCLUSION and RAY_TRACING jobs)
// Regen starts new paths of admitted jobs in the slots the previous shade
// retired, so jobs that arrive while others run join the wavefront at the
// next iteration.  Every count the kernels need lives in device memory, so
// `iterations_per_launch` iterations are captured once into a CUDA graph and
// replayed; the host only writes job records and the admission window between
// launches (stream-ordered) and reads progress back.
//
// Host side (this file): resident scenes with reference counts, a job queue
// admitted against a device-memory budget, per-job films from the
// stream-ordered allocator, and a driver loop that keeps one graph launch in
// flight while it reads the previous one's progress.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dayflower_cuda.h"
#include "dfc_devscene.h"
#include "dfc_ingest.h"
#include "dfc_kernels.h"

using namespace dfc;

namespace {

constexpr int kMaxScenes = 64;
static_assert(kJobPathTracing == DFC_JOB_PATH_TRACING && kJobRayCasting == DFC_JOB_RAY_CASTING && kJobDepthCamera == DFC_JOB_DEPTH_CAMERA &&
                  kJobAmbientOcclusion == DFC_JOB_AMBIENT_OCCLUSION && kJobRayTracing == DFC_JOB_RAY_TRACING,
              "job kinds of the kernels and of the C ABI");
constexpr unsigned kJobRing = 4096;    // job records on the device (power of two)
constexpr unsigned kSegRing = 65536;   // segment records on the device (power of two)
constexpr int64_t kDefaultCapacity = int64_t(1) << 20;
constexpr int64_t kDefaultSegment = 65536;
constexpr int64_t kMaxCapacity = int64_t(1) << 26;
// Device bytes per path slot: state 3 x 16, three ray slots (origin, direction,
// hit) 3 x 48, pending light terms 2 x 16, ray lists 2 x 3 x 4, work lists 2 x 4,
// sort key 1 + sorted list 4, free stack 4, slot job 4.
constexpr size_t kSlotBytes = 48 + 144 + 32 + 24 + 8 + 5 + 8;

struct SceneEntry {
  std::unique_ptr<DeviceScene> ds;
  int caller_refs = 0;
  int job_refs = 0;  // queued or running jobs on this scene
  bool live = false;
  int variant = 0;  // kernel variant it needs: 0 plain, 1 record shapes, 2 materials evaluated per hit
  size_t bytes = 0;
};

struct JobRec {
  dfc_job_desc d{};
  int state = DFC_JOB_QUEUED;
  bool cancel_req = false, cancel_sent = false;
  unsigned seq = 0;
  unsigned long long paths = 0, appended = 0, done = 0;  // total, handed to the device in segments, retired
  float4* film = nullptr;  // sum (pixels float4), then sum of squares (pixels float4)
  size_t film_bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
};

}  // namespace

struct dfc_engine {
  int device = 0;
  int bvh_builder = DFC_BVH_DEVICE;  // mesh hierarchies of later scene commits
  int sm_count = 148;
  int max_trace_blocks = 6;
  int inline_blocks = 2;  // resident blocks per SM of k_shade_inline_batch
  cudaStream_t stream = nullptr, upload_stream = nullptr, read_stream = nullptr;
  cudaEvent_t ev_order = nullptr;
  // `mu` guards all host state and every enqueue on `stream`; nothing waits
  // on the device while holding it.  `drive_mu`: one driver loop at a time.
  // `commit_mu`: one scene ingest at a time (it runs without `mu`).
  std::mutex mu, drive_mu, commit_mu;
  std::condition_variable cv;
  std::string err;
  std::chrono::steady_clock::time_point t0;
  size_t budget = 0;
  // scenes
  Staged staged;
  SceneEntry scenes[kMaxScenes];
  bool table_dirty = true;
  size_t scene_bytes = 0;
  // jobs
  int64_t next_id = 1;
  std::map<int64_t, JobRec> jobs;
  std::deque<int64_t> queue;
  std::vector<int64_t> ring_id = std::vector<int64_t>(kJobRing, 0);
  unsigned seq_next = 0, seq_oldest = 0;
  std::vector<int64_t> sched;    // admitted jobs with paths left to append, in admission order
  size_t rr = 0;                 // round-robin position in `sched`
  unsigned seg_next = 0, seg_lo = 0;
  unsigned long long admitted_paths = 0;  // end of the last appended segment
  unsigned long long cursor_seen = 0;     // the device's path cursor at the last progress read
  bool ctl_dirty = true;
  size_t film_bytes = 0;
  int64_t jobs_submitted = 0, jobs_done = 0;
  // wavefront
  dfc_engine_config cfg{};
  dfc_engine_config active{};
  bool built = false;
  size_t wave_bytes = 0;
  DevBuf d_scene_table, d_jobs, d_segs, d_job_done, d_ctl, d_state;
  DevBuf d_beta, d_rad, d_meta, d_ray_o, d_ray_d, d_hits, d_pend_s, d_pend_m;
  DevBuf d_ray_list[2], d_work_list[2], d_counts, d_sort_keys, d_sort_bins, d_sorted, d_free_stack, d_slot_job, d_overflow;
  cudaGraphExec_t graph = nullptr;
  int graph_variant = 0;
  // progress read-back (pinned), double-buffered
  BatchState* h_state[2] = {nullptr, nullptr};
  unsigned long long* h_done[2] = {nullptr, nullptr};
  unsigned* h_overflow[2] = {nullptr, nullptr};
  unsigned read_seq[2] = {0, 0};  // seq_next when the read-back was enqueued
  unsigned read_seg[2] = {0, 0};  // seg_next when the read-back was enqueued
  std::vector<unsigned long long> seg_end = std::vector<unsigned long long>(kSegRing, 0);  // end of each ring segment
  cudaEvent_t ev_read[2] = {nullptr, nullptr};
  // stats
  int64_t iterations = 0, graph_launches = 0, kernel_launches = 0, paths_retired = 0, rays = 0, overflow = 0;
  int64_t base_iterations = 0, base_retired = 0, base_rays = 0, base_overflow = 0;  // before the last rebuild
  double busy_s = 0.0;
  // engine thread
  std::thread worker;
  std::atomic<bool> stop_req{false};
  bool serving = false;
  bool failed = false;
};

namespace {

double now_s(const dfc_engine* e) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - e->t0).count();
}

int efail(dfc_engine* e, int code, const std::string& msg) {
  if (e) e->err = msg;
  return code;
}

int ecuda(dfc_engine* e, cudaError_t c, const char* what) {
  const int code = (c == cudaErrorMemoryAllocation) ? DFC_E_OOM : DFC_E_CUDA;
  return efail(e, code, std::string(what) + ": " + cudaGetErrorString(c));
}

#define DFC_ECK(expr, what)                               \
  do {                                                    \
    cudaError_t c_ = (expr);                              \
    if (c_ != cudaSuccess) return ecuda(e, c_, what);     \
  } while (0)

size_t used_bytes(const dfc_engine* e) { return e->wave_bytes + e->scene_bytes + e->film_bytes; }

// The most general kernel variant a live scene needs (the captured graph serves every resident scene).
int kernel_variant(const dfc_engine* e) {
  int v = 0;
  for (const SceneEntry& s : e->scenes)
    if (s.live) v = std::max(v, s.variant);
  return v;
}

dfc_engine_config resolved(const dfc_engine* e, dfc_engine_config c) {
  if (c.capacity <= 0) c.capacity = kDefaultCapacity;
  if (c.trace_blocks_per_sm <= 0 || c.trace_blocks_per_sm > e->max_trace_blocks) c.trace_blocks_per_sm = e->max_trace_blocks;
  // shading: more blocks than fit at once (4096 path slots per SM at the default capacity), so that
  // the block scheduler balances SMs over the material-sorted work list
  if (c.shade_blocks_per_sm <= 0) c.shade_blocks_per_sm = 32;
  if (c.shade_threads != 128) c.shade_threads = 256;
  if (c.iterations_per_launch <= 0) c.iterations_per_launch = 4;
  c.iterations_per_launch += c.iterations_per_launch & 1;  // even: the graph ends on the parity it started with
  if (c.policy != DFC_SCHEDULE_FIFO && c.policy != DFC_SCHEDULE_SHORTEST_FIRST) c.policy = DFC_SCHEDULE_ROUND_ROBIN;
  c.reserved = 0;
  if (c.segment_paths <= 0) c.segment_paths = kDefaultSegment;
  if (c.lookahead_paths <= 0) c.lookahead_paths = 8 * c.capacity;
  return c;
}

bool same_config(const dfc_engine_config& a, const dfc_engine_config& b) {
  return a.capacity == b.capacity && a.trace_blocks_per_sm == b.trace_blocks_per_sm && a.shade_blocks_per_sm == b.shade_blocks_per_sm &&
         a.shade_threads == b.shade_threads && a.iterations_per_launch == b.iterations_per_launch && a.policy == b.policy &&
         a.segment_paths == b.segment_paths && a.lookahead_paths == b.lookahead_paths;
}

// Kernel arguments of one iteration of parity b.
void iteration_args(dfc_engine* e, int b, BatchArgs* ba, TraceArgs* ta, SortArgs* so, ShadeArgs* sa) {
  const unsigned P = (unsigned)e->active.capacity;
  unsigned* counts = e->d_counts.as<unsigned>();
  BatchState* st = e->d_state.as<BatchState>();
  const SceneView* table = e->d_scene_table.as<SceneView>();
  const DJob* jobs = e->d_jobs.as<DJob>();
  *ba = BatchArgs{};
  ba->jobs = jobs;
  ba->segs = e->d_segs.as<DSegment>();
  ba->seg_mask = kSegRing - 1;
  ba->ctl = e->d_ctl.as<BatchControl>();
  ba->state = st;
  ba->job_done = e->d_job_done.as<unsigned long long>();
  ba->free_stack = e->d_free_stack.as<unsigned>();
  ba->slot_job = e->d_slot_job.as<unsigned>();
  ba->capacity = P;
  ba->counts_cur = counts + 4 * b;
  ba->counts_next = counts + 4 * (b ^ 1);
  ba->sort_bins = e->d_sort_bins.as<unsigned>() + 2 * kSortBins * b;
  ba->beta = e->d_beta.as<float4>();
  ba->radiance = e->d_rad.as<float4>();
  ba->meta = e->d_meta.as<uint4>();
  ba->ray_o = e->d_ray_o.as<float4>();
  ba->ray_d = e->d_ray_d.as<float4>();
  ba->ray_list = e->d_ray_list[b].as<unsigned>();
  ba->work_list = e->d_work_list[b].as<unsigned>();

  *ta = TraceArgs{};
  ta->scenes = table;
  ta->jobs = jobs;
  ta->slot_job = ba->slot_job;
  ta->ray_list = ba->ray_list;
  ta->ray_count = counts + 4 * b;
  ta->fetch = counts + 4 * b + 2;
  ta->ray_o = ba->ray_o;
  ta->ray_d = ba->ray_d;
  ta->hits = e->d_hits.as<float4>();
  ta->paths = P;
  ta->overflow = e->d_overflow.as<unsigned>();

  *so = SortArgs{};
  so->scenes = table;
  so->jobs = jobs;
  so->slot_job = ba->slot_job;
  so->paths = P;
  so->work_list = ba->work_list;
  so->work_count = counts + 4 * b + 1;
  so->meta = ba->meta;
  so->hits = ta->hits;
  so->keys = e->d_sort_keys.as<unsigned char>();
  so->bins = ba->sort_bins;
  so->sorted = e->d_sorted.as<unsigned>();

  *sa = ShadeArgs{};
  sa->scenes = table;
  sa->jobs = jobs;
  sa->slot_job = ba->slot_job;
  sa->free_stack = ba->free_stack;
  sa->free_top = &st->free_top;
  sa->job_done = e->d_job_done.as<unsigned long long>();
  sa->state = st;
  sa->paths = P;
  sa->pixels = 0;
  sa->overflow = e->d_overflow.as<unsigned>();
  sa->work_list = so->sorted;
  sa->work_count = so->work_count;
  sa->next_work_list = e->d_work_list[b ^ 1].as<unsigned>();
  sa->next_work_count = counts + 4 * (b ^ 1) + 1;
  sa->next_ray_list = e->d_ray_list[b ^ 1].as<unsigned>();
  sa->next_ray_count = counts + 4 * (b ^ 1);
  sa->beta = ba->beta;
  sa->radiance = ba->radiance;
  sa->meta = ba->meta;
  sa->ray_o = ba->ray_o;
  sa->ray_d = ba->ray_d;
  sa->hits = ta->hits;
  sa->pend_shadow = e->d_pend_s.as<float4>();
  sa->pend_mis = e->d_pend_m.as<float4>();
}

constexpr int kKernelsPerIteration = 8;

void enqueue_iteration(dfc_engine* e, int b, int variant) {
  BatchArgs ba;
  TraceArgs ta;
  SortArgs so;
  ShadeArgs sa;
  iteration_args(e, b, &ba, &ta, &so, &sa);
  const dfc_engine_config& c = e->active;
  const int shade_grid = e->sm_count * c.shade_blocks_per_sm;
  // the sort's kernels end each block with global atomics per key: they keep at most 8 blocks per SM
  const int sort_grid = e->sm_count * std::min(c.shade_blocks_per_sm, 8);
  k_batch_plan<<<1, 32, 0, e->stream>>>(ba);
  k_batch_regen<<<e->sm_count * 4, 256, 0, e->stream>>>(ba);
  (variant >= 1 ? k_trace_batch_records : k_trace_batch)<<<e->sm_count * c.trace_blocks_per_sm, kTraceThreads, 0, e->stream>>>(ta);
  k_sort_count_batch<<<sort_grid, 256, 0, e->stream>>>(so);
  k_sort_scatter<<<sort_grid, 256, 0, e->stream>>>(so);
  // the two-lobe kernel over the matte ... plastic hits, misses and light-ray-only paths, the general one over the rest
  ShadeArgs simple = sa;
  simple.range_bins = so.bins;
  simple.range_lo = 0;
  simple.range_hi = kSimpleBins;
  (variant >= 1 ? k_shade_path_batch_simple_records : k_shade_path_batch_simple)<<<shade_grid, 256, 0, e->stream>>>(simple);
  ShadeArgs full = sa;
  full.range_bins = so.bins;
  full.range_lo = kSimpleBins;
  full.range_hi = kKeyInline;
  (variant == 2 ? k_shade_path_batch_textured : variant == 1 ? k_shade_path_batch_records : k_shade_path_batch)
      <<<shade_grid, c.shade_threads, 0, e->stream>>>(full);
  // AMBIENT_OCCLUSION and RAY_TRACING paths finish in one step, tracing their rays on their own threads
  sa.range_bins = so.bins;
  sa.range_lo = kKeyInline;
  sa.range_hi = kSortBins;
  k_shade_inline_batch<<<e->sm_count * e->inline_blocks, kTraceThreads, 0, e->stream>>>(sa);
}

// Captures iterations_per_launch iterations (alternating parity) into the graph.
int capture_graph(dfc_engine* e, int variant) {
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  DFC_ECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
  for (int it = 0; it < e->active.iterations_per_launch; ++it) enqueue_iteration(e, it & 1, variant);
  cudaGraph_t g = nullptr;
  cudaError_t c = cudaStreamEndCapture(e->stream, &g);
  if (c == cudaSuccess) c = cudaGetLastError();
  if (c != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return ecuda(e, c, "graph capture");
  }
  c = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (c != cudaSuccess) return ecuda(e, c, "graph instantiate");
  e->graph_variant = variant;
  return DFC_OK;
}

// (Re)allocates the wavefront for the requested configuration and resets the
// device state; only while no job is admitted and nothing is in flight.
int build_wavefront(dfc_engine* e) {
  const dfc_engine_config c = resolved(e, e->cfg);
  const size_t P = (size_t)c.capacity;
  const size_t need = P * kSlotBytes;
  const size_t other = e->scene_bytes + e->film_bytes;
  if (need + other > e->budget)
    return efail(e, DFC_E_OOM, "wavefront of " + std::to_string(P) + " path slots does not fit the device-memory budget");
  e->wave_bytes = 0;
  DFC_ECK(e->d_beta.ensure(P * 16), "wavefront");
  DFC_ECK(e->d_rad.ensure(P * 16), "wavefront");
  DFC_ECK(e->d_meta.ensure(P * 16), "wavefront");
  DFC_ECK(e->d_ray_o.ensure(3 * P * 16), "wavefront");
  DFC_ECK(e->d_ray_d.ensure(3 * P * 16), "wavefront");
  DFC_ECK(e->d_hits.ensure(3 * P * 16), "wavefront");
  DFC_ECK(e->d_pend_s.ensure(P * 16), "wavefront");
  DFC_ECK(e->d_pend_m.ensure(P * 16), "wavefront");
  for (int k = 0; k < 2; ++k) {
    DFC_ECK(e->d_ray_list[k].ensure(3 * P * 4), "wavefront");
    DFC_ECK(e->d_work_list[k].ensure(P * 4), "wavefront");
  }
  DFC_ECK(e->d_sort_keys.ensure(P), "wavefront");
  DFC_ECK(e->d_sorted.ensure(P * 4), "wavefront");
  DFC_ECK(e->d_free_stack.ensure(P * 4), "wavefront");
  DFC_ECK(e->d_slot_job.ensure(P * 4), "wavefront");
  DFC_ECK(e->d_counts.ensure(8 * sizeof(unsigned)), "wavefront");
  DFC_ECK(e->d_sort_bins.ensure(4 * kSortBins * sizeof(unsigned)), "wavefront");
  DFC_ECK(e->d_overflow.ensure(16), "wavefront");
  e->wave_bytes = need;
  e->active = c;
  e->base_iterations = e->iterations;
  e->base_rays = e->rays;
  e->base_retired = e->paths_retired;
  e->base_overflow = e->overflow;
  DFC_ECK(cudaMemsetAsync(e->d_counts.p, 0, 8 * sizeof(unsigned), e->stream), "wavefront");
  DFC_ECK(cudaMemsetAsync(e->d_state.p, 0, sizeof(BatchState), e->stream), "wavefront");
  DFC_ECK(cudaMemsetAsync(e->d_overflow.p, 0, 16, e->stream), "wavefront");
  // no job is running: the global path sequence restarts at 0, and the
  // search window starts at the next segment appended (older ring records
  // hold starts of the previous sequence)
  e->admitted_paths = 0;
  e->cursor_seen = 0;
  e->seg_lo = e->seg_next;
  e->ctl_dirty = true;
  BatchArgs ba;
  TraceArgs ta;
  SortArgs so;
  ShadeArgs sa;
  iteration_args(e, 0, &ba, &ta, &so, &sa);
  k_batch_init<<<e->sm_count * 4, 256, 0, e->stream>>>(ba);
  DFC_ECK(cudaGetLastError(), "wavefront init");
  int rc = capture_graph(e, kernel_variant(e));
  if (rc) return rc;
  e->built = true;
  return DFC_OK;
}

bool has_running(const dfc_engine* e) { return e->seq_oldest != e->seq_next; }

// Host-side work before a launch (holding mu): scene table, cancellations,
// wavefront (re)build when idle, admission of queued jobs, control words.
int service(dfc_engine* e, bool idle_device) {
  if (!has_running(e) && idle_device && (!e->built || !same_config(resolved(e, e->cfg), e->active))) {
    if (!e->queue.empty() || !e->built) {
      int rc = build_wavefront(e);
      if (rc) return rc;
    }
  }
  if (!e->built) return DFC_OK;
  // free scenes nobody holds
  for (SceneEntry& s : e->scenes) {
    if (s.live && s.caller_refs == 0 && s.job_refs == 0) {
      s.ds.reset();
      s.live = false;
      e->scene_bytes -= s.bytes;
      s.bytes = 0;
      e->table_dirty = true;
    }
  }
  if (e->table_dirty) {
    std::vector<SceneView> table(kMaxScenes, SceneView{});
    for (int i = 0; i < kMaxScenes; ++i)
      if (e->scenes[i].live) table[i] = e->scenes[i].ds->view;
    DFC_ECK(cudaMemcpyAsync(e->d_scene_table.p, table.data(), table.size() * sizeof(SceneView), cudaMemcpyHostToDevice, e->stream),
            "scene table");
    e->table_dirty = false;
    const int var = kernel_variant(e);
    if (var != e->graph_variant) {
      int rc = capture_graph(e, var);
      if (rc) return rc;
    }
  }
  // cancellations of running jobs
  for (unsigned s = e->seq_oldest; s != e->seq_next; ++s) {
    auto it = e->jobs.find(e->ring_id[s & (kJobRing - 1)]);
    if (it == e->jobs.end()) continue;
    JobRec& J = it->second;
    if (J.cancel_req && !J.cancel_sent && J.state == DFC_JOB_RUNNING) {
      static const unsigned one = 1u;
      DJob* dj = e->d_jobs.as<DJob>() + (s & (kJobRing - 1));
      DFC_ECK(cudaMemcpyAsync(&dj->cancelled, &one, sizeof one, cudaMemcpyHostToDevice, e->stream), "cancel");
      J.cancel_sent = true;
    }
  }
  // admission: film, job record
  while (!e->queue.empty()) {
    const int64_t id = e->queue.front();
    auto it = e->jobs.find(id);
    if (it == e->jobs.end() || it->second.state != DFC_JOB_QUEUED) {
      e->queue.pop_front();
      continue;
    }
    JobRec& J = it->second;
    if (e->seq_next - e->seq_oldest >= kJobRing) break;
    const size_t pixels = (size_t)J.d.width * (size_t)J.d.height;
    const size_t fb = pixels * 32;
    if (used_bytes(e) + fb > e->budget) {
      if (e->wave_bytes + e->scene_bytes + fb > e->budget) {  // cannot fit even with every film released
        J.state = DFC_JOB_FAILED;
        J.t_done = now_s(e);
        e->scenes[J.d.scene].job_refs--;
        e->jobs_done++;
        e->queue.pop_front();
        e->cv.notify_all();
        continue;
      }
      break;
    }
    void* film = nullptr;
    DFC_ECK(cudaMallocAsync(&film, fb, e->stream), "job film");
    DFC_ECK(cudaMemsetAsync(film, 0, fb, e->stream), "job film");
    const unsigned seq = e->seq_next;
    const unsigned r = seq & (kJobRing - 1);
    DJob dj{};
    const DeviceScene& ds = *e->scenes[J.d.scene].ds;
    std::memcpy(dj.camera, ds.host.camera, sizeof dj.camera);
    dj.camera[17] = (float)J.d.width;
    dj.camera[18] = (float)J.d.height;
    dj.scene = J.d.scene;
    dj.width = (unsigned)J.d.width;
    dj.pixels = (unsigned)pixels;
    dj.max_bounce = J.d.maximum_bounce;
    dj.min_rr = J.d.minimum_bounce_russian_roulette;
    dj.seed = J.d.seed;
    dj.kind = J.d.kind;
    dj.ao_samples = J.d.ambient_occlusion_samples;
    dj.ao_distance = J.d.maximum_distance;
    dj.cancelled = 0;
    dj.film_sum = static_cast<float4*>(film);
    dj.film_sq = static_cast<float4*>(film) + pixels;
    // pageable source: the copy has taken the bytes when the call returns
    DFC_ECK(cudaMemcpyAsync(e->d_jobs.as<DJob>() + r, &dj, sizeof dj, cudaMemcpyHostToDevice, e->stream), "job record");
    DFC_ECK(cudaMemsetAsync(e->d_job_done.as<unsigned long long>() + r, 0, sizeof(unsigned long long), e->stream), "job record");
    J.film = static_cast<float4*>(film);
    J.film_bytes = fb;
    J.seq = seq;
    J.paths = (unsigned long long)pixels * (unsigned long long)J.d.samples;
    J.appended = 0;
    J.done = 0;
    J.state = DFC_JOB_RUNNING;
    J.t_admit = now_s(e);
    e->film_bytes += fb;
    e->ring_id[r] = id;
    e->seq_next = seq + 1;
    e->sched.push_back(id);
    e->queue.pop_front();
  }
  // scheduling: append segments of admitted jobs while fewer than
  // lookahead_paths appended paths are unstarted
  {
    const dfc_engine_config& c = e->active;
    std::vector<DSegment> add;
    unsigned long long backlog = e->admitted_paths - std::min(e->cursor_seen, e->admitted_paths);
    while (backlog < (unsigned long long)c.lookahead_paths && !e->sched.empty() &&
           e->seg_next + (unsigned)add.size() - e->seg_lo < kSegRing) {
      if (e->rr >= e->sched.size()) e->rr = 0;
      size_t pick = c.policy == DFC_SCHEDULE_FIFO ? 0 : e->rr;
      if (c.policy == DFC_SCHEDULE_SHORTEST_FIRST) {  // the admitted job with the fewest paths left to hand out
        unsigned long long best = ~0ull;
        for (size_t q = 0; q < e->sched.size(); ++q) {
          auto jt = e->jobs.find(e->sched[q]);
          const unsigned long long left = jt == e->jobs.end() ? 0ull : jt->second.paths - std::min(jt->second.appended, jt->second.paths);
          if (left < best) { best = left; pick = q; }
        }
      }
      const int64_t id = e->sched[pick];
      auto it = e->jobs.find(id);
      if (it == e->jobs.end() || it->second.state != DFC_JOB_RUNNING || it->second.cancel_req ||
          it->second.appended >= it->second.paths) {
        e->sched.erase(e->sched.begin() + (long)pick);
        continue;
      }
      JobRec& J = it->second;
      const unsigned long long n = std::min((unsigned long long)c.segment_paths, J.paths - J.appended);
      DSegment sg{};
      sg.start = e->admitted_paths;
      sg.q0 = J.appended;
      sg.count = n;
      sg.job = J.seq & (kJobRing - 1);
      add.push_back(sg);
      J.appended += n;
      e->admitted_paths += n;
      backlog += n;
      if (J.appended >= J.paths) e->sched.erase(e->sched.begin() + (long)pick);
      else if (c.policy == DFC_SCHEDULE_ROUND_ROBIN) e->rr = pick + 1;
    }
    // one copy per contiguous run of ring slots
    size_t k = 0;
    while (k < add.size()) {
      const unsigned first = (e->seg_next + (unsigned)k) & (kSegRing - 1);
      const size_t run = std::min(add.size() - k, (size_t)(kSegRing - first));
      DFC_ECK(cudaMemcpyAsync(e->d_segs.as<DSegment>() + first, add.data() + k, run * sizeof(DSegment), cudaMemcpyHostToDevice,
                              e->stream), "segments");
      k += run;
    }
    for (size_t q = 0; q < add.size(); ++q) e->seg_end[(e->seg_next + (unsigned)q) & (kSegRing - 1)] = add[q].start + add[q].count;
    if (!add.empty()) {
      e->seg_next += (unsigned)add.size();
      e->ctl_dirty = true;
    }
  }
  if (e->ctl_dirty) {
    BatchControl c{};
    c.admitted = e->admitted_paths;
    c.seg_lo = e->seg_lo;
    c.seg_hi = e->seg_next;
    DFC_ECK(cudaMemcpyAsync(e->d_ctl.p, &c, sizeof c, cudaMemcpyHostToDevice, e->stream), "control");
    e->ctl_dirty = false;
  }
  return DFC_OK;
}

// Reads one progress record (holding mu): job completions, the lower end of
// the segment window, counters.
void process(dfc_engine* e, int b) {
  const BatchState& st = *e->h_state[b];
  const unsigned long long* done = e->h_done[b];
  e->iterations = e->base_iterations + st.iterations;
  e->rays = e->base_rays + (int64_t)st.rays;
  e->paths_retired = e->base_retired + (int64_t)st.retired;
  e->overflow = e->base_overflow + *e->h_overflow[b];
  const double t = now_s(e);
  bool changed = false;
  // jobs admitted after this read-back was enqueued have fresh counters on the device: skip them
  for (unsigned s = e->seq_oldest; s != e->read_seq[b]; ++s) {
    auto it = e->jobs.find(e->ring_id[s & (kJobRing - 1)]);
    if (it == e->jobs.end()) continue;
    JobRec& J = it->second;
    if (J.state != DFC_JOB_RUNNING) continue;
    // a cancelled job ends once the paths it was given are done; no more are appended after the request
    const unsigned long long target = J.cancel_req ? J.appended : J.paths;
    J.done = std::min(done[s & (kJobRing - 1)], J.paths);
    if (J.done >= target) {
      J.state = J.cancel_req ? DFC_JOB_CANCELLED : DFC_JOB_DONE;
      J.t_done = t;
      e->scenes[J.d.scene].job_refs--;
      e->jobs_done++;
      changed = true;
    }
  }
  while (e->seq_oldest != e->seq_next) {
    const unsigned r = e->seq_oldest & (kJobRing - 1);
    auto it = e->jobs.find(e->ring_id[r]);
    if (it != e->jobs.end() && it->second.state == DFC_JOB_RUNNING) break;
    e->ring_id[r] = 0;
    e->seq_oldest++;
  }
  // segments wholly behind the cursor hand out nothing more: the window
  // starts at the one holding the cursor, and their ring slots can be reused
  e->cursor_seen = st.cursor;
  // (the device copy of the segments is only read inside [seg_lo, seg_hi))
  unsigned lo = e->seg_lo;
  const unsigned hi = e->read_seg[b];
  while (lo != hi && e->seg_end[lo & (kSegRing - 1)] <= st.cursor) ++lo;
  if (lo != e->seg_lo) {
    e->seg_lo = lo;
    e->ctl_dirty = true;
  }
  if (changed) e->cv.notify_all();
}

void fail_all(dfc_engine* e) {
  e->failed = true;
  for (auto& kv : e->jobs) {
    JobRec& J = kv.second;
    if (J.state == DFC_JOB_QUEUED || J.state == DFC_JOB_RUNNING) {
      J.state = DFC_JOB_FAILED;
      J.t_done = now_s(e);
    }
  }
  e->cv.notify_all();
}

// The driver loop: admits, launches the iteration graph, keeps one launch in
// flight while it reads the previous launch's progress.  until_idle: return
// once nothing is queued or running; otherwise run until stop is requested.
int drive(dfc_engine* e, bool until_idle, double timeout_s) {
  std::lock_guard<std::mutex> drive_lock(e->drive_mu);
  cudaSetDevice(e->device);
  const double t_start = now_s(e);
  double t_mark = t_start;
  bool pending[2] = {false, false};
  int b = 0;
  int rc = DFC_OK;
  bool stopping = false;
  while (true) {
    bool launched = false;
    {
      std::unique_lock<std::mutex> lk(e->mu);
      if (e->failed) {
        rc = DFC_E_CUDA;
        break;
      }
      if (!stopping) {
        rc = service(e, !pending[0] && !pending[1]);
        if (rc) {
          fail_all(e);
          break;
        }
        if (has_running(e) && e->built) {
          cudaError_t c = cudaGraphLaunch(e->graph, e->stream);
          if (c == cudaSuccess) c = cudaMemcpyAsync(e->h_state[b], e->d_state.p, sizeof(BatchState), cudaMemcpyDeviceToHost, e->stream);
          if (c == cudaSuccess)
            c = cudaMemcpyAsync(e->h_done[b], e->d_job_done.p, kJobRing * sizeof(unsigned long long), cudaMemcpyDeviceToHost, e->stream);
          if (c == cudaSuccess) c = cudaMemcpyAsync(e->h_overflow[b], e->d_overflow.p, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream);
          if (c == cudaSuccess) c = cudaEventRecord(e->ev_read[b], e->stream);
          if (c != cudaSuccess) {
            rc = ecuda(e, c, "graph launch");
            fail_all(e);
            break;
          }
          e->read_seq[b] = e->seq_next;
          e->read_seg[b] = e->seg_next;
          pending[b] = true;
          launched = true;
          e->graph_launches++;
          e->kernel_launches += (int64_t)kKernelsPerIteration * e->active.iterations_per_launch;
        }
      }
    }
    const int o = b ^ 1;
    if (pending[o]) {
      const cudaError_t c = cudaEventSynchronize(e->ev_read[o]);
      std::unique_lock<std::mutex> lk(e->mu);
      if (c != cudaSuccess) {
        rc = ecuda(e, c, "wavefront");
        fail_all(e);
        break;
      }
      process(e, o);
      pending[o] = false;
    } else if (!launched && !pending[b]) {
      // nothing in flight
      if (stopping) break;
      std::unique_lock<std::mutex> lk(e->mu);
      if (until_idle) {
        if (e->queue.empty() && !has_running(e)) break;
        if (!has_running(e)) {
          // queued jobs wait for device memory that finished jobs' films hold
          rc = efail(e, DFC_E_OOM, "queued jobs need device memory held by finished jobs' films; release those jobs");
          break;
        }
      } else {
        if (e->stop_req.load()) break;
        e->cv.wait_for(lk, std::chrono::milliseconds(20));
      }
    }
    const double t = now_s(e);
    {
      std::lock_guard<std::mutex> lk(e->mu);
      if (launched || pending[0] || pending[1]) e->busy_s += t - t_mark;
    }
    t_mark = t;
    if (!stopping) {
      if (!until_idle && e->stop_req.load()) stopping = true;
      if (timeout_s > 0 && t - t_start > timeout_s) {
        stopping = true;
        rc = efail(e, DFC_E_TIMEOUT, "engine run timed out");
      }
    }
    b ^= 1;
  }
  // drain anything still in flight
  const cudaError_t c = cudaStreamSynchronize(e->stream);
  std::unique_lock<std::mutex> lk(e->mu);
  if (c != cudaSuccess && !e->failed) {
    rc = ecuda(e, c, "wavefront");
    fail_all(e);
  }
  if (!e->failed)
    for (int k = 0; k < 2; ++k)
      if (pending[k]) process(e, k);
  if (rc == DFC_OK && e->overflow) rc = efail(e, DFC_E_TIMEOUT, "traversal stack bound exceeded in the engine's wavefront");
  return rc;
}

JobRec* find_job(dfc_engine* e, int64_t id) {
  auto it = e->jobs.find(id);
  return it == e->jobs.end() ? nullptr : &it->second;
}

// Orders `read_stream` after everything enqueued on the engine stream so far
// (the job's film allocation and the launches that wrote it); holding mu.
int order_read(dfc_engine* e) {
  DFC_ECK(cudaEventRecord(e->ev_order, e->stream), "read order");
  DFC_ECK(cudaStreamWaitEvent(e->read_stream, e->ev_order, 0), "read order");
  return DFC_OK;
}

}  // namespace

extern "C" {

int dfc_engine_create(int device, int64_t budget, dfc_engine** out) {
  if (!out) return DFC_E_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) return DFC_E_CUDA;
  if (device < 0 || device >= count || budget < 0) return DFC_E_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return DFC_E_CUDA;
  std::unique_ptr<dfc_engine> e(new dfc_engine());
  e->device = device;
  e->t0 = std::chrono::steady_clock::now();
  cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, device);
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_batch, kTraceThreads, 0) == cudaSuccess && nb > 0) e->max_trace_blocks = nb;
  nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_batch_records, kTraceThreads, 0) == cudaSuccess && nb > 0)
    e->max_trace_blocks = std::min(e->max_trace_blocks, nb);
  nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shade_inline_batch, kTraceThreads, 0) == cudaSuccess && nb > 0) e->inline_blocks = nb;
  cudaGetLastError();
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return DFC_E_CUDA;
  e->budget = budget > 0 ? (size_t)budget : (size_t)(0.9 * (double)free_b);
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&e->upload_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&e->read_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&e->ev_order, cudaEventDisableTiming) != cudaSuccess)
    return DFC_E_CUDA;
  for (int k = 0; k < 2; ++k) {
    if (cudaEventCreateWithFlags(&e->ev_read[k], cudaEventDisableTiming) != cudaSuccess) return DFC_E_CUDA;
    if (cudaMallocHost((void**)&e->h_state[k], sizeof(BatchState)) != cudaSuccess) return DFC_E_OOM;
    if (cudaMallocHost((void**)&e->h_done[k], kJobRing * sizeof(unsigned long long)) != cudaSuccess) return DFC_E_OOM;
    if (cudaMallocHost((void**)&e->h_overflow[k], 16) != cudaSuccess) return DFC_E_OOM;
    std::memset(e->h_state[k], 0, sizeof(BatchState));
    std::memset(e->h_done[k], 0, kJobRing * sizeof(unsigned long long));
    std::memset(e->h_overflow[k], 0, 16);
  }
  // keep freed film memory in the pool instead of returning it to the driver
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  if (e->d_scene_table.ensure(kMaxScenes * sizeof(SceneView)) != cudaSuccess || e->d_jobs.ensure(kJobRing * sizeof(DJob)) != cudaSuccess ||
      e->d_segs.ensure(kSegRing * sizeof(DSegment)) != cudaSuccess ||
      e->d_job_done.ensure(kJobRing * sizeof(unsigned long long)) != cudaSuccess || e->d_ctl.ensure(sizeof(BatchControl)) != cudaSuccess ||
      e->d_state.ensure(sizeof(BatchState)) != cudaSuccess)
    return DFC_E_OOM;
  cudaMemsetAsync(e->d_scene_table.p, 0, kMaxScenes * sizeof(SceneView), e->stream);
  cudaMemsetAsync(e->d_jobs.p, 0, kJobRing * sizeof(DJob), e->stream);
  cudaMemsetAsync(e->d_segs.p, 0, kSegRing * sizeof(DSegment), e->stream);
  cudaMemsetAsync(e->d_job_done.p, 0, kJobRing * sizeof(unsigned long long), e->stream);
  cudaMemsetAsync(e->d_ctl.p, 0, sizeof(BatchControl), e->stream);
  cudaMemsetAsync(e->d_state.p, 0, sizeof(BatchState), e->stream);
  if (cudaStreamSynchronize(e->stream) != cudaSuccess) return DFC_E_CUDA;
  *out = e.release();
  return DFC_OK;
}

int dfc_engine_destroy(dfc_engine* e) {
  if (!e) return DFC_E_INVALID_ARG;
  dfc_engine_stop(e);
  {
    std::lock_guard<std::mutex> d(e->drive_mu);
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    std::lock_guard<std::mutex> lk(e->mu);
    for (auto& kv : e->jobs)
      if (kv.second.film) cudaFreeAsync(kv.second.film, e->stream);
    cudaStreamSynchronize(e->stream);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    for (int k = 0; k < 2; ++k) {
      cudaFreeHost(e->h_state[k]);
      cudaFreeHost(e->h_done[k]);
      cudaFreeHost(e->h_overflow[k]);
      cudaEventDestroy(e->ev_read[k]);
    }
    cudaEventDestroy(e->ev_order);
  }
  cudaStream_t s[3] = {e->stream, e->upload_stream, e->read_stream};
  delete e;  // DevBuf and DeviceScene destructors free the rest
  for (cudaStream_t x : s) cudaStreamDestroy(x);
  return DFC_OK;
}

const char* dfc_engine_last_error(const dfc_engine* e) { return e ? e->err.c_str() : "null engine"; }

int dfc_engine_scene_put(dfc_engine* e, const char* name, const void* data, int64_t count, int type) {
  if (!e) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> c(e->commit_mu);
  if (!name) return efail(e, DFC_E_INVALID_ARG, "name == null");
  if (count < 0 || (count > 0 && !data)) return efail(e, DFC_E_INVALID_ARG, "data == null or negative count");
  if (type != DFC_F32 && type != DFC_I32) return efail(e, DFC_E_INVALID_ARG, "type must be DFC_F32 or DFC_I32");
  try {  // the staging arrays are page-locked host memory (PinnedAllocator)
    if (type == DFC_F32) {
      stage_copy(e->staged.f32[name], static_cast<const float*>(data), (size_t)count);
    } else {
      stage_copy(e->staged.i32[name], static_cast<const int32_t*>(data), (size_t)count);
    }
  } catch (const std::bad_alloc&) {
    return efail(e, DFC_E_OOM, std::string("no page-locked host memory to stage ") + name);
  }
  return DFC_OK;
}

int dfc_engine_set_bvh_builder(dfc_engine* e, int builder) {
  if (!e || (builder != DFC_BVH_HOST && builder != DFC_BVH_DEVICE)) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> c(e->commit_mu);
  e->bvh_builder = builder;
  return DFC_OK;
}

int dfc_engine_scene_commit(dfc_engine* e, int layout_version, int32_t* scene_id) {
  if (!e || !scene_id) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> c(e->commit_mu);
  RecycleOnExit recycle{e->staged};
  cudaSetDevice(e->device);
  HostScene hs;
  std::string err;
  int rc = ingest_scene(e->staged, layout_version, &hs, &err, e->bvh_builder == DFC_BVH_DEVICE);
  if (rc != DFC_OK) return efail(e, rc, err);
  const size_t bytes = scene_device_bytes(hs);
  const int variant = hs.textured() ? 2 : hs.record_shapes ? 1 : 0;
  int slot = -1;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    for (int i = 0; i < kMaxScenes && slot < 0; ++i)
      if (!e->scenes[i].live && !e->scenes[i].ds) slot = i;
    if (slot < 0) return efail(e, DFC_E_OOM, "at most 64 scenes can be resident in one engine");
    if (used_bytes(e) + bytes > e->budget) return efail(e, DFC_E_OOM, "scene does not fit the device-memory budget");
    e->scenes[slot].ds.reset(new DeviceScene());  // reserves the slot
    e->scene_bytes += bytes;
  }
  std::unique_ptr<DeviceScene> ds(new DeviceScene());
  cudaError_t ce = upload_scene(std::move(hs), e->upload_stream, ds.get());
  std::lock_guard<std::mutex> lk(e->mu);
  if (ce != cudaSuccess) {
    e->scenes[slot].ds.reset();
    e->scene_bytes -= bytes;
    return ecuda(e, ce, "scene upload");
  }
  SceneEntry& s = e->scenes[slot];
  s.ds = std::move(ds);
  s.caller_refs = 1;
  s.job_refs = 0;
  s.live = true;
  s.variant = variant;
  s.bytes = bytes;
  e->table_dirty = true;
  *scene_id = slot;
  return DFC_OK;
}

int dfc_engine_scene_release(dfc_engine* e, int32_t id) {
  if (!e) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  if (id < 0 || id >= kMaxScenes || !e->scenes[id].live || e->scenes[id].caller_refs <= 0)
    return efail(e, DFC_E_INVALID_ARG, "unknown scene id " + std::to_string(id));
  e->scenes[id].caller_refs--;
  e->cv.notify_all();  // the driver frees it once no job holds it
  return DFC_OK;
}

int dfc_engine_configure(dfc_engine* e, const dfc_engine_config* cfg) {
  if (!e || !cfg) return DFC_E_INVALID_ARG;
  if (cfg->capacity < 0 || cfg->capacity > kMaxCapacity) return efail(e, DFC_E_INVALID_ARG, "capacity out of range");
  if (cfg->shade_threads != 0 && cfg->shade_threads != 128 && cfg->shade_threads != 256)
    return efail(e, DFC_E_INVALID_ARG, "shade_threads must be 128 or 256");
  if (cfg->iterations_per_launch < 0 || cfg->iterations_per_launch > 256) return efail(e, DFC_E_INVALID_ARG, "iterations_per_launch out of range");
  if (cfg->trace_blocks_per_sm < 0 || cfg->shade_blocks_per_sm < 0 || cfg->shade_blocks_per_sm > 64)
    return efail(e, DFC_E_INVALID_ARG, "blocks per SM out of range");
  std::lock_guard<std::mutex> lk(e->mu);
  e->cfg = *cfg;
  return DFC_OK;
}

int dfc_engine_get_config(dfc_engine* e, dfc_engine_config* out) {
  if (!e || !out) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  *out = resolved(e, e->cfg);
  return DFC_OK;
}

int dfc_job_submit(dfc_engine* e, const dfc_job_desc* d, int64_t* job_id) {
  if (!e || !d || !job_id) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  if (e->failed) return efail(e, DFC_E_CUDA, "engine failed: " + e->err);
  if (d->scene < 0 || d->scene >= kMaxScenes || !e->scenes[d->scene].live || e->scenes[d->scene].caller_refs <= 0)
    return efail(e, DFC_E_INVALID_ARG, "unknown scene id " + std::to_string(d->scene));
  if (d->width < 1 || d->height < 1 || (int64_t)d->width * d->height > (int64_t(1) << 27))
    return efail(e, DFC_E_INVALID_ARG, "resolution out of range");
  if (d->samples < 1) return efail(e, DFC_E_INVALID_ARG, "renderPasses < 1");  // AbstractGPURenderer.java:323
  if (d->maximum_bounce < 0 || d->maximum_bounce > 4096) return efail(e, DFC_E_INVALID_ARG, "maximumBounce out of range");
  if (d->minimum_bounce_russian_roulette < 0) return efail(e, DFC_E_INVALID_ARG, "minimumBounceRussianRoulette out of range");
  if (d->kind < DFC_JOB_PATH_TRACING || d->kind > DFC_JOB_RAY_TRACING) return efail(e, DFC_E_INVALID_ARG, "unknown job kind");
  if (d->kind == DFC_JOB_AMBIENT_OCCLUSION) {
    if (d->ambient_occlusion_samples < 1 || d->ambient_occlusion_samples > 4096)
      return efail(e, DFC_E_INVALID_ARG, "samples out of range");  // setSamples, AbstractGPURenderer.java:515
    if (!std::isfinite(d->maximum_distance)) return efail(e, DFC_E_INVALID_ARG, "maximumDistance must be finite");
  }
  const int64_t id = e->next_id++;
  JobRec J;
  J.d = *d;
  J.t_submit = now_s(e);
  e->jobs.emplace(id, J);
  e->queue.push_back(id);
  e->scenes[d->scene].job_refs++;
  e->jobs_submitted++;
  *job_id = id;
  e->cv.notify_all();
  return DFC_OK;
}

int dfc_job_get_info(dfc_engine* e, int64_t id, dfc_job_info* out) {
  if (!e || !out) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  JobRec* J = find_job(e, id);
  if (!J) return efail(e, DFC_E_INVALID_ARG, "unknown job id " + std::to_string(id));
  out->state = J->state;
  out->scene = J->d.scene;
  out->paths_total = (int64_t)J->d.width * J->d.height * J->d.samples;
  out->paths_done = (int64_t)J->done;
  out->submit_s = J->t_submit;
  out->admit_s = J->t_admit;
  out->done_s = J->t_done;
  return DFC_OK;
}

int dfc_job_wait(dfc_engine* e, int64_t id, double timeout_s) {
  if (!e) return DFC_E_INVALID_ARG;
  std::unique_lock<std::mutex> lk(e->mu);
  const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9);
  while (true) {
    JobRec* J = find_job(e, id);
    if (!J) return efail(e, DFC_E_INVALID_ARG, "unknown job id " + std::to_string(id));
    if (J->state == DFC_JOB_DONE || J->state == DFC_JOB_CANCELLED) return DFC_OK;
    if (J->state == DFC_JOB_FAILED) return efail(e, DFC_E_CUDA, "job failed: " + e->err);
    if (e->cv.wait_until(lk, until) == std::cv_status::timeout) {
      J = find_job(e, id);
      if (J && (J->state == DFC_JOB_DONE || J->state == DFC_JOB_CANCELLED)) return DFC_OK;
      return efail(e, DFC_E_TIMEOUT, "job wait timed out");
    }
  }
}

int dfc_job_cancel(dfc_engine* e, int64_t id) {
  if (!e) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  JobRec* J = find_job(e, id);
  if (!J) return efail(e, DFC_E_INVALID_ARG, "unknown job id " + std::to_string(id));
  if (J->state == DFC_JOB_QUEUED) {
    J->state = DFC_JOB_CANCELLED;
    J->t_done = now_s(e);
    e->scenes[J->d.scene].job_refs--;
    e->jobs_done++;
    e->cv.notify_all();
  } else if (J->state == DFC_JOB_RUNNING) {
    J->cancel_req = true;
  }
  return DFC_OK;
}

int dfc_job_read_film(dfc_engine* e, int64_t id, float* dst, int64_t cap) {
  if (!e || !dst) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  JobRec* J = find_job(e, id);
  if (!J) return efail(e, DFC_E_INVALID_ARG, "unknown job id " + std::to_string(id));
  const size_t P = (size_t)J->d.width * J->d.height;
  if (cap < (int64_t)P * 7) return efail(e, DFC_E_INVALID_ARG, "destination too small");
  if (!J->film) {  // not admitted yet: an empty film
    std::memset(dst, 0, P * 7 * sizeof(float));
    return DFC_OK;
  }
  cudaSetDevice(e->device);
  if (int rc = order_read(e)) return rc;
  std::vector<float> s(P * 8);
  DFC_ECK(cudaMemcpyAsync(s.data(), J->film, P * 32, cudaMemcpyDeviceToHost, e->read_stream), "film read");
  DFC_ECK(cudaStreamSynchronize(e->read_stream), "film read");
  const float* q = s.data() + P * 4;
  for (size_t i = 0; i < P; ++i) {
    dst[i * 7 + 0] = s[i * 4 + 0]; dst[i * 7 + 1] = s[i * 4 + 1]; dst[i * 7 + 2] = s[i * 4 + 2];
    dst[i * 7 + 3] = q[i * 4 + 0]; dst[i * 7 + 4] = q[i * 4 + 1]; dst[i * 7 + 5] = q[i * 4 + 2];
    dst[i * 7 + 6] = s[i * 4 + 3];
  }
  return DFC_OK;
}

int dfc_job_read_image_rgba8(dfc_engine* e, int64_t id, int tone_mapper, uint8_t* dst, int64_t cap) {
  if (!e || !dst) return DFC_E_INVALID_ARG;
  if (tone_mapper < 0 || tone_mapper > 5) return efail(e, DFC_E_INVALID_ARG, "unknown tone mapper");
  std::lock_guard<std::mutex> lk(e->mu);
  JobRec* J = find_job(e, id);
  if (!J) return efail(e, DFC_E_INVALID_ARG, "unknown job id " + std::to_string(id));
  const size_t P = (size_t)J->d.width * J->d.height;
  if (cap < (int64_t)P * 4) return efail(e, DFC_E_INVALID_ARG, "destination too small");
  if (!J->film) {
    std::memset(dst, 0, P * 4);
    return DFC_OK;
  }
  cudaSetDevice(e->device);
  if (int rc = order_read(e)) return rc;
  void* img = nullptr;
  DFC_ECK(cudaMallocAsync(&img, P * 4, e->read_stream), "image");
  k_resolve_rgba8<<<(unsigned)((P + 255) / 256), 256, 0, e->read_stream>>>(J->film, (int)P, tone_mapper, 1.0f, static_cast<uchar4*>(img));
  cudaError_t c = cudaMemcpyAsync(dst, img, P * 4, cudaMemcpyDeviceToHost, e->read_stream);
  cudaFreeAsync(img, e->read_stream);
  if (c == cudaSuccess) c = cudaStreamSynchronize(e->read_stream);
  if (c != cudaSuccess) return ecuda(e, c, "image read");
  return DFC_OK;
}

int dfc_job_release(dfc_engine* e, int64_t id) {
  if (!e) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  JobRec* J = find_job(e, id);
  if (!J) return efail(e, DFC_E_INVALID_ARG, "unknown job id " + std::to_string(id));
  if (J->state == DFC_JOB_QUEUED) {
    e->scenes[J->d.scene].job_refs--;
    e->jobs_done++;
  } else if (J->state == DFC_JOB_RUNNING) {
    // still in the wavefront: cancel it and let the driver finish it first
    J->cancel_req = true;
    return efail(e, DFC_E_STATE, "job is running; it was cancelled, release it once it has finished");
  }
  if (J->film) {
    cudaSetDevice(e->device);
    DFC_ECK(cudaFreeAsync(J->film, e->stream), "film free");
    e->film_bytes -= J->film_bytes;
  }
  e->jobs.erase(id);
  e->cv.notify_all();
  return DFC_OK;
}

int dfc_engine_run(dfc_engine* e, double timeout_s) {
  if (!e) return DFC_E_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    if (e->serving) return efail(e, DFC_E_STATE, "the engine thread is running (dfc_engine_start)");
  }
  return drive(e, true, timeout_s);
}

int dfc_engine_start(dfc_engine* e) {
  if (!e) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  if (e->serving) return DFC_OK;
  e->stop_req = false;
  e->serving = true;
  e->worker = std::thread([e] { drive(e, false, 0.0); });
  return DFC_OK;
}

int dfc_engine_stop(dfc_engine* e) {
  if (!e) return DFC_E_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    if (!e->serving) return DFC_OK;
    e->stop_req = true;
    e->cv.notify_all();
  }
  if (e->worker.joinable()) e->worker.join();
  std::lock_guard<std::mutex> lk(e->mu);
  e->serving = false;
  return e->failed ? DFC_E_CUDA : DFC_OK;
}

int dfc_engine_get_stats(dfc_engine* e, dfc_engine_stats* out) {
  if (!e || !out) return DFC_E_INVALID_ARG;
  std::lock_guard<std::mutex> lk(e->mu);
  out->iterations = e->iterations;
  out->graph_launches = e->graph_launches;
  out->kernel_launches = e->kernel_launches;
  out->paths_retired = e->paths_retired;
  out->rays = e->rays;
  out->jobs_submitted = e->jobs_submitted;
  out->jobs_done = e->jobs_done;
  out->device_bytes_used = (int64_t)used_bytes(e);
  out->device_bytes_budget = (int64_t)e->budget;
  out->overflow = e->overflow;
  out->busy_s = e->busy_s;
  return DFC_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner: times candidate wavefront shapes on the caller's sample jobs.
namespace {

std::string cache_key(dfc_engine* e, const char* key) {
  cudaDeviceProp p{};
  cudaGetDeviceProperties(&p, e->device);
  std::ostringstream os;
  os << p.name << "|sm" << p.multiProcessorCount << "|" << (key ? key : "");
  return os.str();
}

bool cache_lookup(const char* path, const std::string& key, dfc_engine_config* c) {
  std::ifstream in(path);
  std::string line;
  while (std::getline(in, line)) {
    const size_t tab = line.find('\t');
    if (tab == std::string::npos || line.compare(0, tab, key) != 0 || tab != key.size()) continue;
    std::istringstream vs(line.substr(tab + 1));
    long long cap;
    int tb, sb, st, it;
    if (vs >> cap >> tb >> sb >> st >> it) {
      c->capacity = cap;
      c->trace_blocks_per_sm = tb;
      c->shade_blocks_per_sm = sb;
      c->shade_threads = st;
      c->iterations_per_launch = it;
      return true;
    }
  }
  return false;
}

void cache_store(const char* path, const std::string& key, const dfc_engine_config& c) {
  std::ofstream out(path, std::ios::app);
  out << key << '\t' << c.capacity << ' ' << c.trace_blocks_per_sm << ' ' << c.shade_blocks_per_sm << ' ' << c.shade_threads << ' '
      << c.iterations_per_launch << '\n';
}

// Renders all sample jobs once with configuration c; returns paths/s (0 on failure).
double time_config(dfc_engine* e, const dfc_job_desc* jobs, int n, const dfc_engine_config& c) {
  if (dfc_engine_configure(e, &c) != DFC_OK) return 0.0;
  std::vector<int64_t> ids;
  double paths = 0.0;
  for (int i = 0; i < n; ++i) {
    int64_t id = 0;
    if (dfc_job_submit(e, &jobs[i], &id) != DFC_OK) return 0.0;
    ids.push_back(id);
    paths += (double)jobs[i].width * jobs[i].height * jobs[i].samples;
  }
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = drive(e, true, 600.0);
  const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int64_t id : ids) dfc_job_release(e, id);
  return rc == DFC_OK && dt > 0.0 ? paths / dt : 0.0;
}

}  // namespace

extern "C" int dfc_engine_autotune(dfc_engine* e, const dfc_job_desc* jobs, int n, const char* cache_path, const char* key,
                                   dfc_engine_config* out) {
  if (!e || !jobs || n < 1) return DFC_E_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    if (e->serving || !e->queue.empty() || has_running(e)) return efail(e, DFC_E_STATE, "autotune needs an idle engine");
  }
  const std::string k = cache_key(e, key);
  dfc_engine_config best{};
  if (cache_path && cache_lookup(cache_path, k, &best)) {
    int rc = dfc_engine_configure(e, &best);
    if (rc) return rc;
    if (out) dfc_engine_get_config(e, out);
    return DFC_OK;
  }
  // coordinate search: capacity, then iterations per launch, then block shapes
  dfc_engine_config c{};
  c.capacity = kDefaultCapacity;
  double best_v = -1.0;
  auto consider = [&](const dfc_engine_config& cand) {
    const double v = time_config(e, jobs, n, cand);
    if (v > best_v) { best_v = v; best = cand; }
  };
  time_config(e, jobs, n, c);  // warm-up (module load, pool growth)
  for (int64_t cap : {int64_t(1) << 20, int64_t(1) << 21, int64_t(1) << 22}) {
    c.capacity = cap;
    consider(c);
  }
  c = best;
  for (int it : {2, 8}) {
    c.iterations_per_launch = it;
    consider(c);
  }
  c = best;
  {
    c.trace_blocks_per_sm = std::max(1, e->max_trace_blocks - 1);
    consider(c);
    c = best;
    c.shade_threads = 128;
    consider(c);
    for (int sb : {16, 64}) {  // more shading blocks than fit at once let the block scheduler balance the SMs
      c = best;
      c.shade_blocks_per_sm = sb;
      consider(c);
    }
  }
  if (best_v <= 0.0) return efail(e, DFC_E_CUDA, "autotune: no candidate ran: " + e->err);
  int rc = dfc_engine_configure(e, &best);
  if (rc) return rc;
  dfc_engine_config res{};
  dfc_engine_get_config(e, &res);
  if (cache_path) cache_store(cache_path, k, res);
  if (out) *out = res;
  return DFC_OK;
}
