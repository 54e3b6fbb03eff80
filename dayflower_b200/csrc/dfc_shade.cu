// Shading kernels with the general BSDF (up to eight lobes, held in local
// memory): every material kind, textures and composite materials.
#include "dfc_shade.cuh"

namespace dfc {

// At most 256 threads a block, two blocks per SM: the shading kernels fit in
// 128 registers (the general BSDF asks for ~156, which left one 256-thread
// block per SM); the batch and textured variants spill at most 44 bytes.
constexpr int kShadeMinBlocks = 2;
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path(ShadeArgs a) { shade_path<false, false>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_records(ShadeArgs a) { shade_path<true, false>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_batch(ShadeArgs a) { shade_path<false, true>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_batch_records(ShadeArgs a) { shade_path<true, true>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_textured(ShadeArgs a) { shade_path<true, false, true>(a); }
__global__ void __launch_bounds__(256, kShadeMinBlocks) k_shade_path_batch_textured(ShadeArgs a) { shade_path<true, true, true>(a); }

}  // namespace dfc
