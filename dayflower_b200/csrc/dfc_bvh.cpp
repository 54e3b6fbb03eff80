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
#include <atomic>
#include <thread>

namespace dfc {
namespace {

struct BNode {
  Box box;
  int left = -1, right = -1;
  int first = 0, count = 0;  // leaf range when left < 0
};

constexpr int kBins = 16;

struct Binning {
  Box bins[3][kBins];
  int cnt[3][kBins] = {};
};

// One item as the builder moves it: box, centroid and original index, kept
// together so that every pass over a node's range reads memory in order.
struct Rec {
  Box box;
  float cen[3];
  int id;
};

// Shared state of one build.  Nodes own disjoint ranges of `recs`, so
// subtrees can be split concurrently.
struct Builder {
  std::vector<Rec> recs;
  int max_leaf;
  int threads;

  Builder(const std::vector<Box>& it, int ml, int th) : max_leaf(ml), threads(th) {
    const size_t n = it.size();
    recs.resize(n);
    const int parts = n >= (1u << 16) ? threads : 1;
    run_parts(parts, [&](int p) {
      for (size_t i = n * p / parts; i < n * (p + 1) / parts; ++i) {
        Rec& r = recs[i];
        r.box = it[i];
        for (int k = 0; k < 3; ++k) r.cen[k] = 0.5f * (it[i].lo[k] + it[i].hi[k]);
        r.id = (int)i;
      }
    });
  }

  std::vector<int> order() const {
    std::vector<int> o(recs.size());
    for (size_t i = 0; i < recs.size(); ++i) o[i] = recs[i].id;
    return o;
  }

  static int bin_of(const Rec& r, int ax, float lo, float sc) { return std::min(kBins - 1, (int)((r.cen[ax] - lo) * sc)); }

  // Centroid bounds and the 3 x kBins binning of order[first, first + count);
  // ranges above kParallelItems are split over `threads` workers.
  void bin_range(int first, int count, Box* cb, Binning* bn) const {
    constexpr int kParallelItems = 1 << 15;
    const int parts = (count >= kParallelItems && threads > 1) ? threads : 1;
    std::vector<Box> cbs(parts);
    auto centroids = [&](int p) {
      const int a = first + (int)((int64_t)count * p / parts), b = first + (int)((int64_t)count * (p + 1) / parts);
      for (int i = a; i < b; ++i) cbs[p].grow_point(recs[i].cen);
    };
    run_parts(parts, centroids);
    for (int p = 0; p < parts; ++p) cb->grow(cbs[p]);
    float lo[3], sc[3];
    bool ok[3];
    for (int ax = 0; ax < 3; ++ax) {
      lo[ax] = cb->lo[ax];
      ok[ax] = cb->hi[ax] > cb->lo[ax];
      sc[ax] = ok[ax] ? kBins / (cb->hi[ax] - cb->lo[ax]) : 0.0f;
    }
    std::vector<Binning> part_bins(parts);
    auto binning = [&](int p) {
      const int a = first + (int)((int64_t)count * p / parts), b = first + (int)((int64_t)count * (p + 1) / parts);
      Binning& pb = part_bins[p];
      for (int i = a; i < b; ++i) {
        const Rec& t = recs[i];
        for (int ax = 0; ax < 3; ++ax) {
          if (!ok[ax]) continue;
          const int k = bin_of(t, ax, lo[ax], sc[ax]);
          pb.bins[ax][k].grow(t.box);
          pb.cnt[ax][k]++;
        }
      }
    };
    run_parts(parts, binning);
    for (int p = 0; p < parts; ++p)
      for (int ax = 0; ax < 3; ++ax)
        for (int k = 0; k < kBins; ++k) { bn->bins[ax][k].grow(part_bins[p].bins[ax][k]); bn->cnt[ax][k] += part_bins[p].cnt[ax][k]; }
  }

  template <typename F>
  static void run_parts(int parts, F&& f) {
    if (parts == 1) { f(0); return; }
    std::vector<std::thread> ws;
    for (int p = 1; p < parts; ++p) ws.emplace_back(f, p);
    f(0);
    for (auto& w : ws) w.join();
  }

  Box range_box(int first, int count) const {
    Box b;
    for (int i = first; i < first + count; ++i) b.grow(recs[i].box);
    return b;
  }

  // Binned-SAH decision for one node; partitions its range in place.  Returns
  // false when the node stays a leaf, else the split point and child boxes.
  bool split_node(const BNode& nd, int* mid, Box* lbox, Box* rbox) {
    const int first = nd.first, count = nd.count;
    if (count <= 1) return false;
    Box cb;
    Binning bn;
    bin_range(first, count, &cb, &bn);
    int best_axis = -1, best_bin = 0;
    float best_cost = FLT_MAX;
    Box best_l, best_r;
    for (int ax = 0; ax < 3; ++ax) {
      if (!(cb.hi[ax] > cb.lo[ax])) continue;
      Box la[kBins];
      int lc[kBins];
      Box acc;
      int c = 0;
      for (int k = 0; k < kBins; ++k) { acc.grow(bn.bins[ax][k]); c += bn.cnt[ax][k]; la[k] = acc; lc[k] = c; }
      Box racc;
      int rc = 0;
      for (int k = kBins - 1; k >= 1; --k) {
        racc.grow(bn.bins[ax][k]);
        rc += bn.cnt[ax][k];
        if (lc[k - 1] == 0 || rc == 0) continue;
        float cost = la[k - 1].area() * lc[k - 1] + racc.area() * rc;
        if (cost < best_cost) { best_cost = cost; best_axis = ax; best_bin = k; best_l = la[k - 1]; best_r = racc; }
      }
    }
    const float leaf_cost = nd.box.area() * count;
    if (count <= max_leaf && (best_axis < 0 || best_cost * 1.0f + nd.box.area() * 0.125f >= leaf_cost)) return false;
    int m = -1;
    if (best_axis >= 0) {
      const float lo = cb.lo[best_axis], sc = kBins / (cb.hi[best_axis] - cb.lo[best_axis]);
      auto it = std::partition(recs.begin() + first, recs.begin() + first + count,
                               [&](const Rec& t) { return bin_of(t, best_axis, lo, sc) < best_bin; });
      m = (int)(it - recs.begin());
      if (m == first || m == first + count) m = -1;
    }
    if (m < 0) {
      m = first + count / 2;
      best_l = range_box(first, m - first);
      best_r = range_box(m, first + count - m);
    }
    *mid = m;
    *lbox = best_l;
    *rbox = best_r;
    return true;
  }

  // Splits node `root` of `nodes` and all its descendants (iterative).
  void split_subtree(std::vector<BNode>& nodes, int root) {
    std::vector<int> todo{root};
    while (!todo.empty()) {
      const int id = todo.back();
      todo.pop_back();
      int mid;
      Box lb, rb;
      if (!split_node(nodes[id], &mid, &lb, &rb)) continue;
      const int first = nodes[id].first, count = nodes[id].count;
      BNode l, r;
      l.box = lb; l.first = first; l.count = mid - first;
      r.box = rb; r.first = mid; r.count = first + count - mid;
      nodes.push_back(l);
      nodes.push_back(r);
      const int li = (int)nodes.size() - 2;
      nodes[id].left = li;
      nodes[id].right = li + 1;
      todo.push_back(li + 1);
      todo.push_back(li);
    }
  }

  // The whole binary tree, root at index 0.  The top is split on this thread
  // (with parallel binning of large ranges) until every open node holds at
  // most `cut` items; those subtrees are then built concurrently into private
  // arrays and appended in task order, so the result does not depend on the
  // thread count or on scheduling.
  std::vector<BNode> build() {
    std::vector<BNode> nodes;
    BNode root;
    root.box = range_box(0, (int)recs.size());
    root.first = 0;
    root.count = (int)recs.size();
    nodes.push_back(root);
    if (threads <= 1) { split_subtree(nodes, 0); return nodes; }
    const int cut = std::max(4096, (int)(recs.size() / (size_t)(8 * threads)));
    std::vector<int> tasks;
    std::vector<int> queue{0};
    for (size_t h = 0; h < queue.size(); ++h) {
      const int id = queue[h];
      if (nodes[id].count <= cut) { tasks.push_back(id); continue; }
      int mid;
      Box lb, rb;
      if (!split_node(nodes[id], &mid, &lb, &rb)) continue;
      const int first = nodes[id].first, count = nodes[id].count;
      BNode l, r;
      l.box = lb; l.first = first; l.count = mid - first;
      r.box = rb; r.first = mid; r.count = first + count - mid;
      nodes.push_back(l);
      nodes.push_back(r);
      const int li = (int)nodes.size() - 2;
      nodes[id].left = li;
      nodes[id].right = li + 1;
      queue.push_back(li);
      queue.push_back(li + 1);
    }
    std::vector<std::vector<BNode>> sub(tasks.size());
    std::vector<int> by_size(tasks.size());
    for (size_t i = 0; i < tasks.size(); ++i) by_size[i] = (int)i;
    std::sort(by_size.begin(), by_size.end(), [&](int a, int b) { return nodes[tasks[a]].count > nodes[tasks[b]].count; });
    std::atomic<int> next{0};
    auto worker = [&](int) {
      for (int k = next.fetch_add(1); k < (int)by_size.size(); k = next.fetch_add(1)) {
        const int t = by_size[k];
        sub[t].push_back(nodes[tasks[t]]);
        split_subtree(sub[t], 0);
      }
    };
    run_parts(threads, worker);
    std::vector<size_t> at(tasks.size());
    size_t total = nodes.size();
    for (size_t t = 0; t < tasks.size(); ++t) { at[t] = total; total += sub[t].size() - 1; }
    nodes.resize(total);
    std::atomic<int> next_copy{0};
    auto copier = [&](int) {
      for (int t = next_copy.fetch_add(1); t < (int)tasks.size(); t = next_copy.fetch_add(1)) {
        const std::vector<BNode>& L = sub[t];
        // local index j >= 1 lands at at[t] + j - 1; local 0 is the task's node
        auto map = [&](int j) { return j < 0 ? j : (j == 0 ? tasks[t] : (int)(at[t] + (size_t)j - 1)); };
        nodes[tasks[t]].left = map(L[0].left);
        nodes[tasks[t]].right = map(L[0].right);
        for (size_t j = 1; j < L.size(); ++j) {
          BNode c = L[j];
          c.left = map(c.left);
          c.right = map(c.right);
          nodes[at[t] + j - 1] = c;
        }
      }
    };
    run_parts(threads, copier);
    return nodes;
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

namespace {

// The 4-wide node for binary node `bn`: its children after opening the
// largest-area interior child until there are four.  Interior children are
// queued (binary node, index in `dst` + index_base) and get fresh slots of `dst`.
void collapse_one(const std::vector<BNode>& tree, int bn, std::vector<BVH4Node>& dst, int index_base,
                  std::vector<std::pair<int, int>>& queue, BVH4Node* node) {
  int kids[4];
  int nk = 0;
  if (tree[bn].left < 0) {
    kids[nk++] = bn;  // a leaf root
  } else {
    kids[nk++] = tree[bn].left;
    kids[nk++] = tree[bn].right;
    while (nk < 4) {
      int best = -1;
      float best_area = -1.0f;
      for (int k = 0; k < nk; ++k) {
        if (tree[kids[k]].left >= 0 && tree[kids[k]].box.area() > best_area) { best = k; best_area = tree[kids[k]].box.area(); }
      }
      if (best < 0) break;
      int opened = kids[best];
      kids[best] = tree[opened].left;
      kids[nk++] = tree[opened].right;
    }
  }
  Box empty;  // inverted: lo = +max, hi = -max, never hit
  for (int s = 0; s < 4; ++s) set_child(*node, s, empty, 0, 0);
  for (int s = 0; s < nk; ++s) {
    const BNode& c = tree[kids[s]];
    if (c.left < 0) {
      set_child(*node, s, c.box, ~c.first, c.count);
    } else {
      const int idx = (int)dst.size() + index_base;
      dst.push_back(BVH4Node{});
      queue.push_back({kids[s], idx});
      set_child(*node, s, c.box, idx, 0);
    }
  }
}

// Breadth-first collapse of the subtree under `bn` into a private array;
// local node 0 is `bn`'s node and interior children carry local indices.
void collapse_subtree(const std::vector<BNode>& tree, int bn, std::vector<BVH4Node>& dst) {
  std::vector<std::pair<int, int>> queue{{bn, 0}};
  dst.push_back(BVH4Node{});
  for (size_t h = 0; h < queue.size(); ++h) {
    BVH4Node node;
    collapse_one(tree, queue[h].first, dst, 0, queue, &node);
    dst[queue[h].second] = node;
  }
}

}  // namespace

int build_bvh4(const std::vector<Box>& items, int max_leaf, std::vector<BVH4Node>& out, std::vector<int>& order) {
  order.clear();
  if (items.empty()) return -1;
  const unsigned hw = std::thread::hardware_concurrency();
  const int threads = (int)std::max(1u, std::min(hw, 64u));
  Builder b(items, max_leaf, threads);
  const std::vector<BNode> tree = b.build();
  order = b.order();
  const int base = (int)out.size();
  // Collapse breadth-first from the root until enough subtrees are pending,
  // then collapse those concurrently into private arrays and append them in
  // queue order (parents precede children; the layout does not depend on the
  // thread count's scheduling).
  std::vector<std::pair<int, int>> queue;  // (binary node, 4-wide node index)
  out.push_back(BVH4Node{});
  queue.push_back({0, base});
  const size_t want = threads > 1 ? (size_t)threads * 8 : (size_t)-1;
  size_t head = 0;
  while (head < queue.size() && queue.size() - head < want) {
    BVH4Node node;
    std::vector<BVH4Node> fresh;
    collapse_one(tree, queue[head].first, fresh, (int)out.size(), queue, &node);
    out.insert(out.end(), fresh.begin(), fresh.end());
    out[queue[head].second] = node;
    ++head;
  }
  const size_t ntask = queue.size() - head;
  if (ntask == 0) return base;
  std::vector<std::vector<BVH4Node>> sub(ntask);
  std::atomic<size_t> next{0};
  auto worker = [&](int) {
    for (size_t k = next.fetch_add(1); k < ntask; k = next.fetch_add(1)) collapse_subtree(tree, queue[head + k].first, sub[k]);
  };
  Builder::run_parts(std::min<int>(threads, (int)ntask), worker);
  std::vector<size_t> at(ntask);
  size_t total = out.size();
  for (size_t k = 0; k < ntask; ++k) { at[k] = total; total += sub[k].size() - 1; }
  out.resize(total);
  std::atomic<size_t> next_copy{0};
  auto copier = [&](int) {
    for (size_t k = next_copy.fetch_add(1); k < ntask; k = next_copy.fetch_add(1)) {
      const std::vector<BVH4Node>& L = sub[k];
      auto remap = [&](BVH4Node n) {  // local interior index j >= 1 lands at at[k] + j - 1
        for (int s = 0; s < 4; ++s)
          if (n.count[s] == 0 && n.child[s] > 0) n.child[s] = (int)(at[k] + (size_t)n.child[s] - 1);
        return n;
      };
      out[queue[head + k].second] = remap(L[0]);
      for (size_t j = 1; j < L.size(); ++j) out[at[k] + j - 1] = remap(L[j]);
    }
  };
  Builder::run_parts(std::min<int>(threads, (int)ntask), copier);
  return base;
}

}  // namespace dfc
