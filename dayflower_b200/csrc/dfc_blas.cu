// Device builder of the bottom-level 4-wide hierarchies (triangle meshes).
//
// The reference builds its mesh hierarchies on the host with an axis sweep
// (geometry/boundingvolume/hierarchy/BVHNode3Fs.java:63-237); the host
// builder of this library (dfc_bvh.cpp) uses binned SAH.  Both take hundreds
// of milliseconds for a 2M-triangle mesh.  This one runs on the device:
//
//   1. triangle boxes and centroid bounds           (k_blas_prep)
//   2. 63-bit Morton codes of the centroids         (k_blas_morton)
//   3. radix sort of (code, triangle) pairs         (cub::DeviceRadixSort)
//   4. the binary radix tree over the sorted codes  (k_blas_radix_tree: Karras,
//      "Maximizing parallelism in the construction of BVHs, octrees, and k-d
//      trees", HPG 2012; equal codes are ordered by index)
//   5. node boxes bottom-up                         (k_blas_boxes: the second
//      child to finish a node computes its box; no thread waits)
//   6. collapse into 4-wide nodes, level by level   (k_blas_collapse: the
//      largest-area interior child is opened until a node has four children;
//      subtrees of at most four triangles become leaves)
//   7. the reordered triangle array                 (k_blas_tri_pos)
//
// The nodes and the triangle array have exactly the layout the host builder
// writes, so traversal does not know which builder made them.
#include "dfc_blas.h"

#include <cub/device/device_radix_sort.cuh>

#include <cfloat>
#include <cstdint>
#include <mutex>

namespace dfc {
namespace {

constexpr int kLeafMax = 4;
constexpr int kBlock = 256;

struct RNode {
  int left, right;  // >= 0 interior node, < 0: ~(sorted leaf index)
  int first, last;  // sorted leaf range
};

__device__ __forceinline__ unsigned f2ord(float f) {  // monotone float -> uint map for atomicMin/Max
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

// 21 bits spread to every third bit of a 63-bit code
__device__ __forceinline__ unsigned long long spread3(unsigned a) {
  unsigned long long x = a & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

__global__ void k_blas_prep(const float* tri_attr, const int* tri_index, int n, float4* lo, float4* hi, float4* cen, unsigned* cbounds) {
  __shared__ unsigned smin[3], smax[3];
  if (threadIdx.x < 3) { smin[threadIdx.x] = 0xffffffffu; smax[threadIdx.x] = 0u; }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const float* t = tri_attr + (size_t)tri_index[i] * 24;
    const float ax = t[0], ay = t[1], az = t[2], bx = t[3], by = t[4], bz = t[5], cx = t[6], cy = t[7], cz = t[8];
    const float4 l = make_float4(fminf(ax, fminf(bx, cx)), fminf(ay, fminf(by, cy)), fminf(az, fminf(bz, cz)), 0.0f);
    const float4 h = make_float4(fmaxf(ax, fmaxf(bx, cx)), fmaxf(ay, fmaxf(by, cy)), fmaxf(az, fmaxf(bz, cz)), 0.0f);
    const float4 c = make_float4(0.5f * (l.x + h.x), 0.5f * (l.y + h.y), 0.5f * (l.z + h.z), 0.0f);
    lo[i] = l; hi[i] = h; cen[i] = c;
    atomicMin(&smin[0], f2ord(c.x)); atomicMin(&smin[1], f2ord(c.y)); atomicMin(&smin[2], f2ord(c.z));
    atomicMax(&smax[0], f2ord(c.x)); atomicMax(&smax[1], f2ord(c.y)); atomicMax(&smax[2], f2ord(c.z));
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    atomicMin(&cbounds[threadIdx.x], smin[threadIdx.x]);
    atomicMax(&cbounds[3 + threadIdx.x], smax[threadIdx.x]);
  }
}

__global__ void k_blas_morton(const float4* cen, int n, const unsigned* cbounds, unsigned long long* keys, int* vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // one cube over the centroid bounds (the largest extent on every axis), so that a code bit
  // halves space along an axis only where that axis is at least as long as the others
  const float lx = ord2f(cbounds[0]), ly = ord2f(cbounds[1]), lz = ord2f(cbounds[2]);
  const float e = fmaxf(ord2f(cbounds[3]) - lx, fmaxf(ord2f(cbounds[4]) - ly, ord2f(cbounds[5]) - lz));
  const float4 c = cen[i];
  const float s = 2097151.0f;  // 2^21 - 1
  auto q = [s, e](float v, float l) { return e > 0.0f ? (unsigned)fminf(fmaxf((v - l) / e * s, 0.0f), s) : 0u; };
  keys[i] = spread3(q(c.x, lx)) << 2 | spread3(q(c.y, ly)) << 1 | spread3(q(c.z, lz));
  vals[i] = i;
}

// Length of the common prefix of sorted codes i and j (index bits break ties); -1 outside [0, n).
__device__ __forceinline__ int prefix(const unsigned long long* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const unsigned long long a = k[i], b = k[j];
  return a == b ? 64 + __clz((unsigned)(i ^ j)) : __clzll(a ^ b);
}

__global__ void k_blas_radix_tree(const unsigned long long* k, int n, RNode* nodes, int* int_parent, int* leaf_parent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = prefix(k, n, i, i + 1) - prefix(k, n, i, i - 1) >= 0 ? 1 : -1;
  const int dmin = prefix(k, n, i, i - d);
  int lmax = 2;
  while (prefix(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (prefix(k, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = prefix(k, n, i, j);
  int s = 0;
  for (int div = 2;; div <<= 1) {
    const int t = (l + div - 1) / div;
    if (prefix(k, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
  }
  const int gamma = i + s * d + min(d, 0);
  const int first = min(i, j), last = max(i, j);
  RNode nd;
  nd.first = first; nd.last = last;
  nd.left = first == gamma ? ~gamma : gamma;
  nd.right = last == gamma + 1 ? ~(gamma + 1) : gamma + 1;
  nodes[i] = nd;
  if (nd.left < 0) leaf_parent[gamma] = i; else int_parent[gamma] = i;
  if (nd.right < 0) leaf_parent[gamma + 1] = i; else int_parent[gamma + 1] = i;
  if (i == 0) int_parent[0] = -1;
}

// Sorted leaf boxes (coalesced reads later).
__global__ void k_blas_sorted_boxes(const int* perm, int n, const float4* lo, const float4* hi, float4* slo, float4* shi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  slo[i] = lo[p]; shi[i] = hi[p];
}

__global__ void k_blas_boxes(int n, const RNode* nodes, const int* int_parent, const int* leaf_parent, const float4* slo,
                             const float4* shi, float4* ilo, float4* ihi, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = leaf_parent[i];
  while (p >= 0) {
    __threadfence();  // this thread's box (or the leaf box of an earlier kernel) before the arrival count
    if (atomicAdd(&flags[p], 1) == 0) return;  // the sibling is not done: it will build p
    __threadfence();
    const RNode nd = nodes[p];
    const float4 al = nd.left < 0 ? slo[~nd.left] : __ldcg(ilo + nd.left), ah = nd.left < 0 ? shi[~nd.left] : __ldcg(ihi + nd.left);
    const float4 bl = nd.right < 0 ? slo[~nd.right] : __ldcg(ilo + nd.right), bh = nd.right < 0 ? shi[~nd.right] : __ldcg(ihi + nd.right);
    __stcg(ilo + p, make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f));
    __stcg(ihi + p, make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f));
    p = int_parent[p];
  }
}

struct Front { int bn, slot; };

__device__ __forceinline__ float half_area(float4 l, float4 h) {
  const float dx = h.x - l.x, dy = h.y - l.y, dz = h.z - l.z;
  return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ void put_slot(BVH4Node& o, int s, float4 l, float4 h, int child, int count) {
  o.lox[s] = l.x; o.loy[s] = l.y; o.loz[s] = l.z;
  o.hix[s] = h.x; o.hiy[s] = h.y; o.hiz[s] = h.z;
  o.child[s] = child; o.count[s] = count;
}

// One 4-wide node per frontier entry; interior children that keep more than
// kLeafMax triangles get new nodes and go to the next frontier.
__global__ void k_blas_collapse(const Front* in, int n_in, Front* out, int* n_out, int* node_count, int node_cap, int* overflow,
                                const RNode* nodes, const float4* ilo, const float4* ihi, const float4* slo, const float4* shi,
                                BVH4Node* dst, int node_base, int tri_first) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_in) return;
  const Front f = in[e];
  auto size = [&](int c) { return c < 0 ? 1 : nodes[c].last - nodes[c].first + 1; };
  auto area = [&](int c) { return c < 0 ? half_area(slo[~c], shi[~c]) : half_area(ilo[c], ihi[c]); };
  int kids[4];
  int nk = 2;
  kids[0] = nodes[f.bn].left;
  kids[1] = nodes[f.bn].right;
  while (nk < 4) {
    int best = -1;
    float best_area = -1.0f;
    for (int k = 0; k < nk; ++k)
      if (kids[k] >= 0 && size(kids[k]) > kLeafMax && area(kids[k]) > best_area) { best = k; best_area = area(kids[k]); }
    if (best < 0) break;
    const int o = kids[best];
    kids[best] = nodes[o].left;
    kids[nk++] = nodes[o].right;
  }
  BVH4Node nd;
  const float4 elo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.0f), ehi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.0f);
  for (int s = 0; s < 4; ++s) put_slot(nd, s, elo, ehi, 0, 0);
  for (int s = 0; s < nk; ++s) {
    const int c = kids[s];
    if (c < 0) {
      put_slot(nd, s, slo[~c], shi[~c], ~(tri_first + ~c), 1);
    } else if (size(c) <= kLeafMax) {
      put_slot(nd, s, ilo[c], ihi[c], ~(tri_first + nodes[c].first), size(c));
    } else {
      const int slot = atomicAdd(node_count, 1);
      if (slot >= node_cap) { atomicExch(overflow, 1); put_slot(nd, s, elo, ehi, 0, 0); continue; }
      put_slot(nd, s, ilo[c], ihi[c], node_base + slot, 0);
      out[atomicAdd(n_out, 1)] = Front{c, slot};
    }
  }
  dst[f.slot] = nd;
}

// A root that is a single leaf (at most kLeafMax triangles): one slot over all of them.
__global__ void k_blas_leaf_root(int n, const float4* slo, const float4* shi, BVH4Node* dst, int tri_first) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float4 l = slo[0], h = shi[0];
  for (int i = 1; i < n; ++i) {
    const float4 a = slo[i], b = shi[i];
    l = make_float4(fminf(l.x, a.x), fminf(l.y, a.y), fminf(l.z, a.z), 0.0f);
    h = make_float4(fmaxf(h.x, b.x), fmaxf(h.y, b.y), fmaxf(h.z, b.z), 0.0f);
  }
  BVH4Node nd;
  const float4 elo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.0f), ehi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.0f);
  for (int s = 0; s < 4; ++s) put_slot(nd, s, elo, ehi, 0, 0);
  put_slot(nd, 0, l, h, ~tri_first, n);
  dst[0] = nd;
}

// Triangles in leaf order: v0 (w: triangle index in shape3FTriangle3FArray), v1, v2.
__global__ void k_blas_tri_pos(const float* tri_attr, const int* tri_index, const int* perm, int n, F4* tri_pos) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int ti = tri_index[perm[j]];
  const float* t = tri_attr + (size_t)ti * 24;
  tri_pos[3 * (size_t)j] = F4{t[0], t[1], t[2], __int_as_float(ti)};
  tri_pos[3 * (size_t)j + 1] = F4{t[3], t[4], t[5], 0.0f};
  tri_pos[3 * (size_t)j + 2] = F4{t[6], t[7], t[8], 0.0f};
}

// The builder's temporaries come from a memory pool of its own per device
// that keeps up to kKeepBytes reserved between builds: the device's default
// pool returns freed memory at every synchronisation, so each commit could map
// fresh device memory (with it the upload and build stage of a 2.1M-triangle
// scene took between 12 and 228 ms from run to run).
constexpr uint64_t kKeepBytes = 1ull << 30;
cudaMemPool_t builder_pool(cudaStream_t s) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = kKeepBytes;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  (void)s;
  return pools[dev];
}
template <typename T>
cudaError_t alloc(T** p, size_t n, cudaStream_t s) {
  const size_t bytes = (n ? n : 1) * sizeof(T);
  if (cudaMemPool_t pool = builder_pool(s)) return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, s);
  return cudaMallocAsync(reinterpret_cast<void**>(p), bytes, s);
}

// Rewrites each node's child words as the traversal's stack entries, so that
// a node visit loads one 16-byte word of children and pushes it as it is:
// an interior child keeps its index (tag bits 00), a leaf becomes
// 0x80000000 | first << 2 | (count - 1).  count[] is left as built.
__global__ void k_encode_entries(BVH4Node* nodes, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int4* cp = reinterpret_cast<int4*>(nodes + i) + 6;
  int4 c = cp[0];
  const int4 k = cp[1];
  auto enc = [](int child, int count) -> int {
    if (child >= 0 || count <= 0) return child >= 0 ? child : 0;  // interior, or an empty slot (never hit)
    return (int)(0x80000000u | ((unsigned)(~child) << 2) | (unsigned)(count - 1));
  };
  cp[0] = make_int4(enc(c.x, k.x), enc(c.y, k.y), enc(c.z, k.z), enc(c.w, k.w));
}

}  // namespace

cudaError_t encode_node_entries(BVH4Node* nodes, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_encode_entries<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(nodes, n);
  return cudaGetLastError();
}

int build_blas_device(const float* tri_attr, const int* tri_index, int n, BVH4Node* nodes_out, int node_base, int node_cap, F4* tri_pos,
                      int tri_first, cudaStream_t s, cudaError_t* err) {
  *err = cudaSuccess;
  if (n <= 0) return 0;
  float4 *lo = nullptr, *hi = nullptr, *cen = nullptr, *slo = nullptr, *shi = nullptr, *ilo = nullptr, *ihi = nullptr;
  unsigned long long *keys = nullptr, *keys2 = nullptr;
  int *vals = nullptr, *perm = nullptr, *int_parent = nullptr, *leaf_parent = nullptr, *flags = nullptr, *counters = nullptr;
  unsigned* cbounds = nullptr;
  RNode* rn = nullptr;
  Front *fa = nullptr, *fb = nullptr;
  void* temp = nullptr;
  size_t temp_bytes = 0;
  int written = -1;
  cudaError_t e = cudaSuccess;
  const int grid = (n + kBlock - 1) / kBlock;
#define DFC_B(x) \
  if (e == cudaSuccess) e = (x)
  DFC_B(alloc(&lo, n, s)); DFC_B(alloc(&hi, n, s)); DFC_B(alloc(&cen, n, s));
  DFC_B(alloc(&slo, n, s)); DFC_B(alloc(&shi, n, s)); DFC_B(alloc(&ilo, n, s)); DFC_B(alloc(&ihi, n, s));
  DFC_B(alloc(&keys, n, s)); DFC_B(alloc(&keys2, n, s)); DFC_B(alloc(&vals, n, s)); DFC_B(alloc(&perm, n, s));
  DFC_B(alloc(&int_parent, n, s)); DFC_B(alloc(&leaf_parent, n, s)); DFC_B(alloc(&flags, n, s));
  DFC_B(alloc(&counters, 4, s)); DFC_B(alloc(&cbounds, 6, s)); DFC_B(alloc(&rn, n, s));
  DFC_B(alloc(&fa, n, s)); DFC_B(alloc(&fb, n, s));
  DFC_B(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys2, vals, perm, n, 0, 63, s));
  DFC_B(alloc(reinterpret_cast<unsigned char**>(&temp), temp_bytes ? temp_bytes : 16, s));
  if (e == cudaSuccess) {
    unsigned init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    e = cudaMemcpyAsync(cbounds, init, sizeof init, cudaMemcpyHostToDevice, s);
    DFC_B(cudaStreamSynchronize(s));  // `init` lives on this stack frame
  }
  if (e == cudaSuccess) {
    k_blas_prep<<<grid, kBlock, 0, s>>>(tri_attr, tri_index, n, lo, hi, cen, cbounds);
    k_blas_morton<<<grid, kBlock, 0, s>>>(cen, n, cbounds, keys, vals);
    e = cudaGetLastError();
  }
  DFC_B(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys2, vals, perm, n, 0, 63, s));
  if (e == cudaSuccess) {
    k_blas_sorted_boxes<<<grid, kBlock, 0, s>>>(perm, n, lo, hi, slo, shi);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && n <= kLeafMax) {
    k_blas_leaf_root<<<1, 32, 0, s>>>(n, slo, shi, nodes_out, tri_first);
    e = cudaGetLastError();
    written = 1;
  } else if (e == cudaSuccess) {
    DFC_B(cudaMemsetAsync(flags, 0, (size_t)n * sizeof(int), s));
    DFC_B(cudaMemsetAsync(counters, 0, 4 * sizeof(int), s));
    if (e == cudaSuccess) {
      k_blas_radix_tree<<<grid, kBlock, 0, s>>>(keys2, n, rn, int_parent, leaf_parent);
      k_blas_boxes<<<grid, kBlock, 0, s>>>(n, rn, int_parent, leaf_parent, slo, shi, ilo, ihi, flags);
      e = cudaGetLastError();
    }
    // collapse, one launch per level of the 4-wide tree: counters[0] nodes, [1] next frontier, [2] overflow
    int h_counters[3] = {1, 0, 0};
    const Front root{0, 0};
    DFC_B(cudaMemcpyAsync(counters, h_counters, 3 * sizeof(int), cudaMemcpyHostToDevice, s));
    DFC_B(cudaMemcpyAsync(fa, &root, sizeof root, cudaMemcpyHostToDevice, s));
    int n_front = 1;
    for (int level = 0; e == cudaSuccess && n_front > 0; ++level) {
      if (level > 4 * 64) { e = cudaErrorInvalidValue; break; }  // a 4-wide tree over 63-bit codes is far shallower
      DFC_B(cudaMemsetAsync(counters + 1, 0, sizeof(int), s));
      if (e != cudaSuccess) break;
      k_blas_collapse<<<(n_front + kBlock - 1) / kBlock, kBlock, 0, s>>>(fa, n_front, fb, counters + 1, counters, node_cap,
                                                                         counters + 2, rn, ilo, ihi, slo, shi, nodes_out, node_base,
                                                                         tri_first);
      DFC_B(cudaGetLastError());
      DFC_B(cudaMemcpyAsync(h_counters, counters, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
      DFC_B(cudaStreamSynchronize(s));
      n_front = h_counters[1];
      Front* t = fa; fa = fb; fb = t;
    }
    if (e == cudaSuccess) {
      if (h_counters[2]) e = cudaErrorInvalidValue;  // more nodes than the capacity: cannot happen for a binary radix tree
      written = h_counters[0];
    }
  }
  if (e == cudaSuccess) {
    k_blas_tri_pos<<<grid, kBlock, 0, s>>>(tri_attr, tri_index, perm, n, tri_pos);
    e = cudaGetLastError();
  }
#undef DFC_B
  for (void* p : {(void*)lo, (void*)hi, (void*)cen, (void*)slo, (void*)shi, (void*)ilo, (void*)ihi, (void*)keys, (void*)keys2, (void*)vals,
                  (void*)perm, (void*)int_parent, (void*)leaf_parent, (void*)flags, (void*)counters, (void*)cbounds, (void*)rn,
                  (void*)fa, (void*)fb, temp})
    if (p) cudaFreeAsync(p, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  *err = e;
  return e == cudaSuccess ? written : -1;
}

}  // namespace dfc
