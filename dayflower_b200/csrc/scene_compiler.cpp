// Host helper for the scene compiler: builds one triangle mesh's bounding
// volume hierarchy and emits it in the reference's threaded int-stream form.
//
// Reference: geometry/boundingvolume/hierarchy/BVHNode3Fs.java:63 (a node with
// fewer than four triangles is a leaf) and scene/compiler/CompiledShape3FCache.java
// :2652 doToBVHNode3F (depth-first order; tree node [ID 2, bvOffset, nextOffset,
// leftOffset, 0, 0, 0, 0]; leaf [ID 1, bvOffset, nextOffset, count, triangle
// offsets..., padding to 8]).  The split choice here is a 16-bin SAH over
// centroids, not the reference's sweep; any tree is a valid encoding of the mesh.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Box {
  float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  void grow(const float* p) { for (int k = 0; k < 3; ++k) { mn[k] = std::min(mn[k], p[k]); mx[k] = std::max(mx[k], p[k]); } }
  void grow(const Box& b) { for (int k = 0; k < 3; ++k) { mn[k] = std::min(mn[k], b.mn[k]); mx[k] = std::max(mx[k], b.mx[k]); } }
  float area() const {
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = std::max(0.0f, mx[k] - mn[k]);
    return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
  }
};

struct Builder {
  const float* tris;
  std::vector<Box> tbox;
  std::vector<float> cen;  // 3 per triangle
  std::vector<int64_t> idx;
  std::vector<Box> node_box;
  std::vector<int64_t> node_begin, node_count, node_end_index;  // count < 0 -> interior
  std::vector<int> node_depth;

  int64_t build(int64_t b, int64_t e, int depth) {
    const int64_t me = (int64_t)node_box.size();
    Box bb, cb;
    for (int64_t i = b; i < e; ++i) { bb.grow(tbox[idx[i]]); cb.grow(&cen[idx[i] * 3]); }
    node_box.push_back(bb); node_begin.push_back(b); node_count.push_back(e - b); node_end_index.push_back(0); node_depth.push_back(depth);
    const int64_t n = e - b;
    if (n < 4) { node_end_index[me] = me + 1; return me; }
    int best_axis = -1; int best_bin = -1; float best_cost = FLT_MAX;
    const int B = 16;
    for (int ax = 0; ax < 3; ++ax) {
      float lo = cb.mn[ax], hi = cb.mx[ax];
      if (!(hi > lo)) continue;
      Box bins[B]; int64_t cnt[B] = {0};
      const float sc = B / (hi - lo);
      for (int64_t i = b; i < e; ++i) {
        int k = std::min(B - 1, (int)((cen[idx[i] * 3 + ax] - lo) * sc));
        bins[k].grow(tbox[idx[i]]); cnt[k]++;
      }
      Box left[B]; int64_t lc[B];
      Box acc; int64_t c = 0;
      for (int k = 0; k < B; ++k) { acc.grow(bins[k]); c += cnt[k]; left[k] = acc; lc[k] = c; }
      Box racc; int64_t rc = 0;
      for (int k = B - 1; k >= 1; --k) {
        racc.grow(bins[k]); rc += cnt[k];
        if (lc[k - 1] == 0 || rc == 0) continue;
        float cost = left[k - 1].area() * lc[k - 1] + racc.area() * rc;
        if (cost < best_cost) { best_cost = cost; best_axis = ax; best_bin = k; }
      }
    }
    int64_t mid;
    if (best_axis < 0) {
      mid = b + n / 2;
    } else {
      float lo = cb.mn[best_axis], hi = cb.mx[best_axis];
      const float sc = B / (hi - lo);
      auto it = std::partition(idx.begin() + b, idx.begin() + e, [&](int64_t t) {
        return std::min(B - 1, (int)((cen[t * 3 + best_axis] - lo) * sc)) < best_bin;
      });
      mid = it - idx.begin();
      if (mid == b || mid == e) mid = b + n / 2;
    }
    node_count[me] = -1;
    build(b, mid, depth + 1);
    build(mid, e, depth + 1);
    node_end_index[me] = (int64_t)node_box.size();
    return me;
  }
};

}  // namespace

extern "C" {

// Builds the threaded BVH for `n` triangles given as compiled 24-float rows.
//   tri_offset_base  absolute offset of triangle 0 in shape3FTriangle3FArray
//                    (triangle i is at tri_offset_base + 24 * i)
//   aabb_base        relative index of this mesh's first box in
//                    boundingVolume3FAxisAlignedBoundingBox3FArray
//   stream           out: 8 ints per node (capacity 2n nodes)
//   aabbs            out: 8 floats per node [max xyz, min xyz, 0, 0] (capacity 2n)
// Returns the node count, or -1 on bad arguments.
long long dfc_sc_build_mesh_bvh(const float* tris, long long n, long long tri_offset_base, long long aabb_base,
                                int* stream, float* aabbs, long long capacity_nodes) {
  if (!tris || n <= 0 || !stream || !aabbs) return -1;
  Builder bld;
  bld.tris = tris;
  bld.tbox.resize(n); bld.cen.resize(n * 3); bld.idx.resize(n);
  for (long long i = 0; i < n; ++i) {
    const float* t = tris + i * 24;
    Box b; b.grow(t); b.grow(t + 3); b.grow(t + 6);
    bld.tbox[i] = b;
    for (int k = 0; k < 3; ++k) bld.cen[i * 3 + k] = (t[k] + t[3 + k] + t[6 + k]) * (1.0f / 3.0f);
    bld.idx[i] = i;
  }
  bld.node_box.reserve(2 * n);
  bld.build(0, n, 0);
  const long long nodes = (long long)bld.node_box.size();
  if (nodes > capacity_nodes) return -1;
  for (long long k = 0; k < nodes; ++k) {
    int* s = stream + k * 8;
    std::memset(s, 0, 8 * sizeof(int));
    const long long end = bld.node_end_index[k];
    s[1] = (int)(aabb_base + k);
    s[2] = end < nodes ? (int)(end * 8) : -1;
    if (bld.node_count[k] >= 0) {
      s[0] = 1;
      s[3] = (int)bld.node_count[k];
      for (long long j = 0; j < bld.node_count[k]; ++j) s[4 + j] = (int)(tri_offset_base + 24 * bld.idx[bld.node_begin[k] + j]);
    } else {
      s[0] = 2;
      s[3] = (int)((k + 1) * 8);
    }
    float* a = aabbs + k * 8;
    const Box& b = bld.node_box[k];
    a[0] = b.mx[0]; a[1] = b.mx[1]; a[2] = b.mx[2]; a[3] = b.mn[0]; a[4] = b.mn[1]; a[5] = b.mn[2]; a[6] = 0; a[7] = 0;
  }
  return nodes;
}

}  // extern "C"
