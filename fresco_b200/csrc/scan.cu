// Prefix-sum kernels (see scan.cuh).
#include "scan.cuh"

namespace fb {

namespace {

// Inclusive scan of v over the 1024 threads of the block (warp shuffles, then
// the 32 warp totals); *total gets the block sum.
__device__ __forceinline__ int block_inclusive_scan_1024(int v, int* total) {
  __shared__ int warp_tot[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) warp_tot[wid] = v;
  __syncthreads();
  if (wid == 0) {
    int w = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  const int r = v + (wid > 0 ? warp_tot[wid - 1] : 0);
  *total = warp_tot[31];
  __syncthreads();
  return r;
}

}  // namespace

__global__ void __launch_bounds__(1024) scan_block_kernel(const int* __restrict__ in, int* out, int* block_sums,
                                                          int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * 1024 + threadIdx.x;
  const int v = i < n ? in[i] : 0;
  int tot;
  const int inc = block_inclusive_scan_1024(v, &tot);
  if (i < n) out[i] = inc - v;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(int* block_sums, int nb) {
  int carry = 0;
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? block_sums[i] : 0;
    int tot;
    const int inc = block_inclusive_scan_1024(v, &tot);
    if (i < nb) block_sums[i] = carry + inc - v;
    carry += tot;
  }
}

__global__ void scan_add_kernel(int* out, const int* __restrict__ block_sums, int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * 1024 + threadIdx.x;
  if (i < n) out[i] += block_sums[blockIdx.x];
}

}  // namespace fb
