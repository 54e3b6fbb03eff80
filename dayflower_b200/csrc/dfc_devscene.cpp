// Upload of a decoded scene (HostScene) into device buffers.
#include "dfc_devscene.h"

#include "dfc_blas.h"

namespace dfc {

namespace {

template <typename T>
size_t vbytes(const std::vector<T>& v) { return v.size() * sizeof(T); }

template <typename T>
cudaError_t put(DevBuf& b, const std::vector<T>& v, cudaStream_t s) {
  cudaError_t e = b.ensure(vbytes(v));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpyAsync(b.p, v.data(), vbytes(v), cudaMemcpyHostToDevice, s);
}

}  // namespace

size_t node_count(const HostScene& hs) { return (size_t)hs.blas_nodes + hs.nodes.size(); }
size_t tri_pos_count(const HostScene& hs) { return hs.blas_tris > 0 ? 3 * (size_t)hs.blas_tris : hs.tri_pos.size(); }

size_t scene_device_bytes(const HostScene& hs) {
  return vbytes(hs.prims) + vbytes(hs.materials) + vbytes(hs.lights) + node_count(hs) * sizeof(BVH4Node) + vbytes(hs.tlas_items) +
         vbytes(hs.tlas_bound) + vbytes(hs.unbounded.empty() ? hs.unbounded_storage : hs.unbounded) + tri_pos_count(hs) * sizeof(F4) +
         hs.tri_attr_count * sizeof(float) + vbytes(hs.rects) + vbytes(hs.shapes) + vbytes(hs.perez) + 19 * sizeof(float) +
         vbytes(hs.textures) + vbytes(hs.texels) + vbytes(hs.modifiers) + vbytes(hs.composites) + vbytes(hs.texmats);
}

size_t DeviceScene::device_bytes() const { return scene_device_bytes(host); }

cudaError_t upload_scene(HostScene&& hs, cudaStream_t s, DeviceScene* ds) {
  cudaError_t e = cudaStreamSynchronize(s);
#define DFC_PUT(buf, vec) \
  if (e == cudaSuccess) e = put(ds->buf, vec, s)
  DFC_PUT(prims, hs.prims);
  DFC_PUT(mats, hs.materials);
  DFC_PUT(lights, hs.lights);
  // nodes: the device-built bottom levels first (if any), then the host-built nodes
  if (e == cudaSuccess) e = ds->nodes.ensure(node_count(hs) * sizeof(BVH4Node));
  if (e == cudaSuccess && !hs.nodes.empty())
    e = cudaMemcpyAsync(ds->nodes.as<BVH4Node>() + hs.blas_nodes, hs.nodes.data(), vbytes(hs.nodes), cudaMemcpyHostToDevice, s);
  DFC_PUT(tlas_items, hs.tlas_items);
  DFC_PUT(tlas_bound, hs.tlas_bound);
  DFC_PUT(unbounded, hs.unbounded.empty() ? hs.unbounded_storage : hs.unbounded);
  if (hs.blas_tris > 0) {
    if (e == cudaSuccess) e = ds->tri_pos.ensure(tri_pos_count(hs) * sizeof(F4));
  } else {
    DFC_PUT(tri_pos, hs.tri_pos);
  }
  if (e == cudaSuccess) e = ds->tri_attr.ensure(hs.tri_attr_count * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpyAsync(ds->tri_attr.p, hs.tri_attr, hs.tri_attr_count * sizeof(float), cudaMemcpyHostToDevice, s);
  DFC_PUT(rects, hs.rects);
  DFC_PUT(shapes, hs.shapes);
  DFC_PUT(perez, hs.perez);
  const std::vector<float> cam(hs.camera, hs.camera + 19);
  DFC_PUT(camera, cam);
  DFC_PUT(textures, hs.textures);
  DFC_PUT(texels, hs.texels);
  DFC_PUT(modifiers, hs.modifiers);
  DFC_PUT(composites, hs.composites);
  DFC_PUT(texmats, hs.texmats);
#undef DFC_PUT
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  if (!hs.blas_jobs.empty()) {  // bottom levels on the device, from the uploaded triangle records
    int* idx = nullptr;
    e = cudaMallocAsync(reinterpret_cast<void**>(&idx), vbytes(hs.blas_tri_index), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(idx, hs.blas_tri_index.data(), vbytes(hs.blas_tri_index), cudaMemcpyHostToDevice, s);
    for (const HostScene::BlasJob& j : hs.blas_jobs) {
      if (e != cudaSuccess) break;
      cudaError_t be = cudaSuccess;
      const int w = build_blas_device(ds->tri_attr.as<float>(), idx + j.index_off, j.count, ds->nodes.as<BVH4Node>() + j.node_base,
                                      j.node_base, j.node_cap, ds->tri_pos.as<F4>() + 3 * (size_t)j.tri_first, j.tri_first, s, &be);
      if (w < 0) e = be != cudaSuccess ? be : cudaErrorUnknown;
    }
    if (idx) cudaFreeAsync(idx, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    std::vector<int>().swap(hs.blas_tri_index);
  }
  // leaf ranges (triangles, top-level items) must fit the 28 bits of a stack entry
  if ((long long)tri_pos_count(hs) / 3 >= kMaxLeafFirst || (long long)hs.tlas_items.size() >= kMaxLeafFirst) return cudaErrorInvalidValue;
  e = encode_node_entries(ds->nodes.as<BVH4Node>(), node_count(hs), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  SceneView& v = ds->view;
  v.prims = ds->prims.as<DPrim>();
  v.prim_count = (int)hs.prims.size();
  v.materials = ds->mats.as<DMaterial>();
  v.lights = ds->lights.as<DLight>();
  v.light_count = hs.lights_storage_pad ? 0 : (int)hs.lights.size();
  v.nodes = ds->nodes.as<BVH4Node>();
  v.tlas_root = hs.tlas_root;
  v.tlas_items = ds->tlas_items.as<int>();
  v.tlas_bound = ds->tlas_bound.as<F4>();
  v.unbounded = ds->unbounded.as<int>();
  v.unbounded_count = (int)hs.unbounded.size();
  v.tri_pos = ds->tri_pos.as<F4>();
  v.tri_attr = ds->tri_attr.as<float>();
  v.rects = ds->rects.as<float>();
  v.shapes = ds->shapes.as<float>();
  v.perez = ds->perez.as<float>();
  v.camera = ds->camera.as<float>();
  v.textures = ds->textures.as<DTexture>();
  v.texels = ds->texels.as<unsigned>();
  v.modifiers = ds->modifiers.as<DModifier>();
  v.composites = ds->composites.as<DComposite>();
  v.texmats = ds->texmats.as<DTexMaterial>();
  hs.tri_attr = nullptr;  // points into the staging arrays, which the caller recycles next
  ds->host = std::move(hs);
  return cudaSuccess;
}

}  // namespace dfc
