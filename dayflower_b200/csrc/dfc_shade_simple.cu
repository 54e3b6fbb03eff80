// Shading kernels for the material kinds whose BSDF has at most two lobes
// (no BSDF, matte, mirror, glass, metal, plastic): the lobes stay in
// registers and the other materials' lobe code is not compiled in.
#include "dfc_shade.cuh"

namespace dfc {

#ifndef DFC_SHADE_SIMPLE_BLOCKS
#define DFC_SHADE_SIMPLE_BLOCKS 4
#endif
constexpr int kShadeSimpleBlocks = DFC_SHADE_SIMPLE_BLOCKS;
__global__ void __launch_bounds__(256, kShadeSimpleBlocks) k_shade_path_simple(ShadeArgs a) {
  shade_path<false, false, false, kSimpleLobes>(a);
}
__global__ void __launch_bounds__(256, kShadeSimpleBlocks) k_shade_path_simple_records(ShadeArgs a) {
  shade_path<true, false, false, kSimpleLobes>(a);
}
__global__ void __launch_bounds__(256, kShadeSimpleBlocks) k_shade_path_batch_simple(ShadeArgs a) {
  shade_path<false, true, false, kSimpleLobes>(a);
}
__global__ void __launch_bounds__(256, kShadeSimpleBlocks) k_shade_path_batch_simple_records(ShadeArgs a) {
  shade_path<true, true, false, kSimpleLobes>(a);
}

}  // namespace dfc
