// Upload of a decoded scene (HostScene) into device buffers.
#include "dfc_devscene.h"

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

size_t scene_device_bytes(const HostScene& hs) {
  return vbytes(hs.prims) + vbytes(hs.materials) + vbytes(hs.lights) + vbytes(hs.nodes) + vbytes(hs.tlas_items) +
         vbytes(hs.tlas_bound) + vbytes(hs.unbounded.empty() ? hs.unbounded_storage : hs.unbounded) + vbytes(hs.tri_pos) +
         vbytes(hs.tri_attr) + vbytes(hs.rects) + vbytes(hs.shapes) + vbytes(hs.perez) + 19 * sizeof(float) +
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
  DFC_PUT(nodes, hs.nodes);
  DFC_PUT(tlas_items, hs.tlas_items);
  DFC_PUT(tlas_bound, hs.tlas_bound);
  DFC_PUT(unbounded, hs.unbounded.empty() ? hs.unbounded_storage : hs.unbounded);
  DFC_PUT(tri_pos, hs.tri_pos);
  DFC_PUT(tri_attr, hs.tri_attr);
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
  ds->host = std::move(hs);
  return cudaSuccess;
}

}  // namespace dfc
