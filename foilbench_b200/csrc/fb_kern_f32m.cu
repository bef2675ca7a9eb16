// Step-kernel instantiations for velocity type float and Krylov type float, one per
// row-transform shape (values per thread, first-pass radix) that a grid can need. Kept in
// its own translation unit so the precisions compile in parallel.
#include "fb_step.cuh"

namespace fb {

void *step_kernel_f32m(int vpt, int r0) {
  switch (vpt * 16 + r0) {
    case 16 * 16 + 2: return reinterpret_cast<void *>(&step_kernel<float, float, 16, 2>);
    case 16 * 16 + 4: return reinterpret_cast<void *>(&step_kernel<float, float, 16, 4>);
    case 16 * 16 + 8: return reinterpret_cast<void *>(&step_kernel<float, float, 16, 8>);
    case 16 * 16 + 16: return reinterpret_cast<void *>(&step_kernel<float, float, 16, 16>);
    case 32 * 16 + 4: return reinterpret_cast<void *>(&step_kernel<float, float, 32, 4>);
    default: return nullptr;
  }
}

}  // namespace fb
