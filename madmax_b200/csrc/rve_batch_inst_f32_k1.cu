// rve_batch_inst_f32_k1.cu -- instantiations of the batched kernel (rve_batch_kernel.cuh),
// split over several translation units so they compile in parallel.
#include "rve_batch_kernel.cuh"

namespace sp {
SP_BATCH_SHAPES(SP_BATCH_DEFINE, float, 1)
}  // namespace sp
