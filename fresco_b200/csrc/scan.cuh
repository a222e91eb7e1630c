// Exclusive prefix sum of n ints in three launches (block scan, scan of the
// block sums in one block, add).  out may alias nothing; tmp holds
// ceil(n / 1024) ints.
#pragma once

#include "common.cuh"

namespace fb {

__global__ void __launch_bounds__(1024) scan_block_kernel(const int* __restrict__ in, int* out, int* block_sums,
                                                          int64_t n);
__global__ void __launch_bounds__(1024) scan_sums_kernel(int* block_sums, int nb);
__global__ void scan_add_kernel(int* out, const int* __restrict__ block_sums, int64_t n);

inline int64_t scan_tmp_size(int64_t n) { return ceil_div(std::max<int64_t>(n, 1), 1024); }

inline void exclusive_scan(const int* in, int* out, int* tmp, int64_t n, cudaStream_t s) {
  const int nb = int(scan_tmp_size(n));
  scan_block_kernel<<<nb, 1024, 0, s>>>(in, out, tmp, n);
  scan_sums_kernel<<<1, 1024, 0, s>>>(tmp, nb);
  scan_add_kernel<<<nb, 1024, 0, s>>>(out, tmp, n);
  FB_LAUNCH_CHECK();
}

}  // namespace fb
