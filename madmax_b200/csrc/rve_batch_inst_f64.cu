// rve_batch_inst_f64.cu -- instantiations of the batched kernel (rve_batch_kernel.cuh),
// split over several translation units so they compile in parallel.
#include "rve_batch_kernel.cuh"

namespace sp {
SP_BATCH_SHAPES_FP64(SP_BATCH_DEFINE, double, 1)
SP_BATCH_SHAPES_FP64(SP_BATCH_DEFINE, double, 6)
SP_BATCH_SHAPES_FP64(SP_BATCH_DEFINE, double, 8)
}  // namespace sp
