// Device builder of the bottom-level hierarchies (triangle meshes).
#pragma once

#include <cuda_runtime.h>

#include "dfc_scene.h"

namespace dfc {

// Builds the 4-wide hierarchy of `count` triangles on `stream`:
//   tri_attr   shape3FTriangle3FArray on the device (24 floats per triangle)
//   tri_index  the mesh's triangle indices (device, `count` ints)
//   nodes      the mesh's node range; node 0 of it is the root; capacity `node_cap` (>= blas_node_capacity(count))
//   node_base  index of nodes[0] in the scene's node array (interior children are absolute)
//   tri_pos    the mesh's range of the reordered triangle array (3 * count F4)
//   tri_first  index of tri_pos[0] in the scene's triangle array (leaf ranges are absolute)
// Returns the number of nodes written, or -1 on a CUDA error (*err set).
int build_blas_device(const float* tri_attr, const int* tri_index, int count, BVH4Node* nodes, int node_base, int node_cap,
                      F4* tri_pos, int tri_first, cudaStream_t stream, cudaError_t* err);

// Rewrites the child words of `n` device nodes as traversal stack entries (an
// interior child's index; 0x80000000 | first << 2 | (count - 1) for a leaf of
// `count` items from `first`), once every level of the scene is in place.
// Leaf ranges must start below 2^28.
cudaError_t encode_node_entries(BVH4Node* nodes, size_t n, cudaStream_t stream);
constexpr long long kMaxLeafFirst = 1ll << 28;

// Nodes a mesh of `count` triangles may need (an upper bound).
inline int blas_node_capacity(int count) { return count > 1 ? count : 1; }

}  // namespace dfc
