// The traversal kernels (persistent, per-lane refill): per-job renderer and
// batch engine, with and without the disk ... torus record shapes.
#include "dfc_trav.cuh"

namespace dfc {

__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace(TraceArgs a) { trace_rays<false, false>(a); }
__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace_records(TraceArgs a) { trace_rays<true, false>(a); }
__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace_batch(TraceArgs a) { trace_rays<false, true>(a); }
__global__ void __launch_bounds__(kTraceBlock, DFC_TRACE_MIN_BLOCKS) k_trace_batch_records(TraceArgs a) { trace_rays<true, true>(a); }

}  // namespace dfc
