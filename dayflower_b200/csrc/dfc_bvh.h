// 4-wide BVH builder interface (host side).
#pragma once

#include <cfloat>
#include <vector>

#include "dfc_scene.h"

namespace dfc {

struct Box {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
  float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  void grow(const Box& b) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = lo[k] < b.lo[k] ? lo[k] : b.lo[k];
      hi[k] = hi[k] > b.hi[k] ? hi[k] : b.hi[k];
    }
  }
  void grow_point(const float* p) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = lo[k] < p[k] ? lo[k] : p[k];
      hi[k] = hi[k] > p[k] ? hi[k] : p[k];
    }
  }
  float area() const {
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = hi[k] > lo[k] ? hi[k] - lo[k] : 0.0f;
    return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
  }
};

// Appends the nodes of a new hierarchy over `items` to `out` and returns the
// root node index.  `order` receives the item permutation: leaf (first, count)
// covers order[first .. first + count).
int build_bvh4(const std::vector<Box>& items, int max_leaf, std::vector<BVH4Node>& out, std::vector<int>& order);

}  // namespace dfc
