// Host builder for the 4-wide bounding volume hierarchies the traversal kernel
// walks.  A binned-SAH binary tree (16 bins per axis, leaves of at most
// `max_leaf` items) is collapsed into 4-wide nodes by repeatedly opening the
// child with the largest surface area.  Items of a leaf are contiguous in the
// returned order, so a leaf is (first, count).
//
// This replaces the reference's mesh hierarchy (geometry/boundingvolume/
// hierarchy/BVHNode3Fs.java:63-237, threaded binary tree walked left-first)
// and adds a top level over primitives, which the reference GPU path does not
// have (renderer/gpu/AbstractSceneKernel.java:318 loops over every primitive).
#include "dfc_bvh.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <thread>

namespace dfc {
namespace {

struct BNode {
  Box box;
  int left = -1, right = -1;
  int first = 0, count = 0;  // leaf range when left < 0
};

struct Binary {
  const std::vector<Box>& items;
  std::vector<float> cen;
  std::vector<int> order;
  std::vector<BNode> nodes;
  int max_leaf;

  Binary(const std::vector<Box>& it, int ml) : items(it), max_leaf(ml) {
    const size_t n = it.size();
    cen.resize(n * 3);
    order.resize(n);
    for (size_t i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) cen[i * 3 + k] = 0.5f * (it[i].lo[k] + it[i].hi[k]);
      order[i] = (int)i;
    }
    nodes.reserve(n * 2 / std::max(1, ml - 1) + 16);
  }

  int make(int first, int count) {
    BNode nd;
    for (int i = first; i < first + count; ++i) nd.box.grow(items[order[i]]);
    nd.first = first;
    nd.count = count;
    nodes.push_back(nd);
    return (int)nodes.size() - 1;
  }

  void split(int ni) {
    // iterative to bound the host stack depth
    std::vector<int> todo{ni};
    while (!todo.empty()) {
      int id = todo.back();
      todo.pop_back();
      const int first = nodes[id].first, count = nodes[id].count;
      if (count <= 1) continue;
      Box cb;
      for (int i = first; i < first + count; ++i) cb.grow_point(&cen[order[i] * 3]);
      const int B = 16;
      int best_axis = -1, best_bin = 0;
      float best_cost = FLT_MAX;
      for (int ax = 0; ax < 3; ++ax) {
        const float lo = cb.lo[ax], hi = cb.hi[ax];
        if (!(hi > lo)) continue;
        Box bins[B];
        int cnt[B] = {0};
        const float sc = B / (hi - lo);
        for (int i = first; i < first + count; ++i) {
          int k = std::min(B - 1, (int)((cen[order[i] * 3 + ax] - lo) * sc));
          bins[k].grow(items[order[i]]);
          cnt[k]++;
        }
        Box la[B];
        int lc[B];
        Box acc;
        int c = 0;
        for (int k = 0; k < B; ++k) { acc.grow(bins[k]); c += cnt[k]; la[k] = acc; lc[k] = c; }
        Box racc;
        int rc = 0;
        for (int k = B - 1; k >= 1; --k) {
          racc.grow(bins[k]);
          rc += cnt[k];
          if (lc[k - 1] == 0 || rc == 0) continue;
          float cost = la[k - 1].area() * lc[k - 1] + racc.area() * rc;
          if (cost < best_cost) { best_cost = cost; best_axis = ax; best_bin = k; }
        }
      }
      const float leaf_cost = nodes[id].box.area() * count;
      if (count <= max_leaf && (best_axis < 0 || best_cost * 1.0f + nodes[id].box.area() * 0.125f >= leaf_cost)) continue;
      int mid;
      if (best_axis < 0) {
        mid = first + count / 2;
      } else {
        const float lo = cb.lo[best_axis], hi = cb.hi[best_axis];
        const float sc = B / (hi - lo);
        auto it = std::partition(order.begin() + first, order.begin() + first + count, [&](int t) {
          return std::min(B - 1, (int)((cen[t * 3 + best_axis] - lo) * sc)) < best_bin;
        });
        mid = (int)(it - order.begin());
        if (mid == first || mid == first + count) mid = first + count / 2;
      }
      int l = make(first, mid - first);
      int r = make(mid, first + count - mid);
      nodes[id].left = l;
      nodes[id].right = r;
      todo.push_back(r);
      todo.push_back(l);
    }
  }
};

void set_child(BVH4Node& n, int slot, const Box& b, int child, int count) {
  float* lo[3] = {n.lox, n.loy, n.loz};
  float* hi[3] = {n.hix, n.hiy, n.hiz};
  for (int k = 0; k < 3; ++k) { lo[k][slot] = b.lo[k]; hi[k][slot] = b.hi[k]; }
  n.child[slot] = child;
  n.count[slot] = count;
}

}  // namespace

int build_bvh4(const std::vector<Box>& items, int max_leaf, std::vector<BVH4Node>& out, std::vector<int>& order) {
  order.clear();
  if (items.empty()) return -1;
  Binary bin(items, max_leaf);
  int root = bin.make(0, (int)items.size());
  bin.split(root);
  order = bin.order;
  const int base = (int)out.size();
  // Collapse: breadth-first so parents precede children.
  std::vector<std::pair<int, int>> queue;  // (binary node, 4-wide slot index)
  out.push_back(BVH4Node{});
  queue.push_back({root, base});
  size_t head = 0;
  while (head < queue.size()) {
    const int bn = queue[head].first;
    const int slot_index = queue[head].second;
    ++head;
    int kids[4];
    int nk = 0;
    if (bin.nodes[bn].left < 0) {
      kids[nk++] = bn;  // a leaf root
    } else {
      kids[nk++] = bin.nodes[bn].left;
      kids[nk++] = bin.nodes[bn].right;
      while (nk < 4) {
        int best = -1;
        float best_area = -1.0f;
        for (int k = 0; k < nk; ++k) {
          if (bin.nodes[kids[k]].left >= 0 && bin.nodes[kids[k]].box.area() > best_area) { best = k; best_area = bin.nodes[kids[k]].box.area(); }
        }
        if (best < 0) break;
        int opened = kids[best];
        kids[best] = bin.nodes[opened].left;
        kids[nk++] = bin.nodes[opened].right;
      }
    }
    BVH4Node node;
    Box empty;  // inverted: lo = +max, hi = -max, never hit
    for (int s = 0; s < 4; ++s) set_child(node, s, empty, 0, 0);
    for (int s = 0; s < nk; ++s) {
      const BNode& c = bin.nodes[kids[s]];
      if (c.left < 0) {
        set_child(node, s, c.box, ~c.first, c.count);
      } else {
        int idx = (int)out.size();
        out.push_back(BVH4Node{});
        queue.push_back({kids[s], idx});
        set_child(node, s, c.box, idx, 0);
      }
    }
    out[slot_index] = node;
  }
  return base;
}

}  // namespace dfc
