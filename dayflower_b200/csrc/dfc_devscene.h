// Device-resident scene: the buffers one committed scene occupies in HBM and
// the SceneView the kernels read.  Shared by the per-job renderer handle
// (dfc_api.cu) and the batch/serving engine (dfc_engine.cu), which keeps many
// of these resident at once.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "dfc_ingest.h"

namespace dfc {

// One cudaMalloc'd device buffer, grown on demand and freed on destruction.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, n ? n : 16);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

struct DeviceScene {
  DevBuf prims, mats, lights, nodes, tlas_items, tlas_bound, unbounded, tri_pos, tri_attr, rects, shapes, perez, camera;
  DevBuf textures, texels, modifiers, composites, texmats;
  SceneView view{};
  HostScene host;  // decoded records kept for updates (camera, matrices) and sizes
  size_t device_bytes() const;
};

// Bytes the scene's records take in device memory once uploaded.
size_t scene_device_bytes(const HostScene& hs);

// Uploads `hs` into `ds` on `stream` (synchronising it) and fills ds->view;
// `hs` is moved into ds->host.  Returns the CUDA error of the first failing step.
cudaError_t upload_scene(HostScene&& hs, cudaStream_t stream, DeviceScene* ds);

}  // namespace dfc
