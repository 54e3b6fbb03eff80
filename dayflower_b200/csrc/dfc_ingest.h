// Host-side scene ingest: reference compiled arrays -> device records.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <new>
#include <utility>
#include <string>
#include <vector>

#include "../../include/dayflower_cuda.h"
#include "dfc_scene.h"

namespace dfc {

// Page-locked host memory for the staging arrays: the scene upload then
// copies straight from them by DMA instead of through the driver's pageable
// bounce buffers, whose speed depends on the host's memory traffic.
template <typename T>
struct PinnedAllocator {
  using value_type = T;
  PinnedAllocator() = default;
  template <typename U>
  PinnedAllocator(const PinnedAllocator<U>&) {}
  T* allocate(size_t n) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, n * sizeof(T), cudaHostAllocPortable) != cudaSuccess) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_t) { cudaFreeHost(p); }
  // resize() default-initialises (no zero fill): every staged element is
  // written by stage_copy right after
  template <typename U>
  void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
  template <typename U>
  bool operator==(const PinnedAllocator<U>&) const { return true; }
  template <typename U>
  bool operator!=(const PinnedAllocator<U>&) const { return false; }
};
using StagedF = std::vector<float, PinnedAllocator<float>>;
using StagedI = std::vector<int32_t, PinnedAllocator<int32_t>>;

// Copies `count` elements into a staging array (capacity kept between
// commits), on the host's threads when the array is large.  Throws
// std::bad_alloc when no page-locked memory can be had.
void stage_copy(StagedF& dst, const float* src, size_t count);
void stage_copy(StagedI& dst, const int32_t* src, size_t count);

// Arrays staged by dfc_scene_put, by reference field name.
struct Staged {
  std::map<std::string, StagedF> f32;
  std::map<std::string, StagedI> i32;
  // Empties every array but keeps its allocation, so that staging the next
  // scene of a similar size copies into memory that is already mapped.
  void recycle() {
    for (auto& kv : f32) kv.second.clear();
    for (auto& kv : i32) kv.second.clear();
  }
};

// Recycles the staging arrays when a commit ends, on every path (they are read until the upload is done).
struct RecycleOnExit {
  Staged& st;
  ~RecycleOnExit() { st.recycle(); }
};

struct HostScene {
  std::vector<DPrim> prims;
  std::vector<DMaterial> materials;
  std::vector<DLight> lights;
  std::vector<BVH4Node> nodes;
  std::vector<int> tlas_items;
  std::vector<F4> tlas_bound;
  std::vector<int> unbounded;
  std::vector<int> unbounded_storage;  // non-empty stand-in when there are no unbounded primitives
  std::vector<F4> tri_pos;
  std::vector<float> rects, perez;
  // shape3FTriangle3FArray as staged (not copied): valid until the staging arrays are recycled,
  // which happens after the upload
  const float* tri_attr = nullptr;
  size_t tri_attr_count = 0;
  std::vector<float> shapes;  // pool of the record-sized shapes (disk ... torus), DPrim.data = float offset
  std::vector<DTexture> textures;      // texture nodes of the kMatTextured materials
  std::vector<unsigned> texels;        // their images (and normal-map modifier images), packed ARGB
  std::vector<DModifier> modifiers;
  std::vector<DComposite> composites;
  std::vector<DTexMaterial> texmats;
  float camera[19] = {0};
  int tlas_root = -1;
  int lights_storage_pad = 0;  // 1 when `lights` holds only a placeholder
  int64_t triangles = 0;
  bool record_shapes = false;  // any disk, cylinder, cone, paraboloid, hyperboloid, cuboid or torus primitive
  float blas_ms = 0.0f, tlas_ms = 0.0f;  // host time of the bottom- and top-level builds
  // Bottom levels built on the device (dfc_blas.cu) instead of here: the node
  // array then starts with a region of `blas_nodes` nodes the device builds
  // fill (the host nodes follow it), and the triangle array of `blas_tris`
  // triangles is written on the device as well.
  struct BlasJob { size_t index_off; int count, node_base, node_cap, tri_first; };
  std::vector<BlasJob> blas_jobs;
  std::vector<int> blas_tri_index;  // per job: its triangles' indices in shape3FTriangle3FArray
  int blas_nodes = 0;
  int64_t blas_tris = 0;
  // Materials evaluated per hit (textures, modifiers, composite materials): the textured shading variants.
  bool textured() const { return !texmats.empty() || !composites.empty(); }
};

// Decodes the staged arrays (layout 1 or 2).  Returns a dfc_status.  On
// success out->tri_attr points into `st`, which must outlive the upload.
// With `device_blas`, mesh hierarchies are left to build_blas_device (upload_scene runs it).
int ingest_scene(Staged& st, int layout, HostScene* out, std::string* err, bool device_blas = false);

}  // namespace dfc
