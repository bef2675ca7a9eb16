// Batched step kernel: float32 fields, float32 Krylov vectors inside the FP64 defect
// correction, 16 values per thread, row-transform shape chosen per scenario at run time.
// Own translation unit so it compiles in parallel with the single-solve kernels.
#include "fb_step.cuh"

namespace fb {

void *step_kernel_batch_f32m() { return reinterpret_cast<void *>(&step_kernel_batch<float, float, 16, 0>); }

}  // namespace fb
