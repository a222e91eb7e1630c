// FP32 instantiation of the NUFFT building blocks.
#include "nufft_kernels.cuh"

namespace fb {
FB_INSTANTIATE_NUFFT(float)
}  // namespace fb
