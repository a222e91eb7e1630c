// Prefix-sum kernels (see scan.cuh).
#include "scan.cuh"

namespace fb {

__global__ void __launch_bounds__(1024) scan_block_kernel(const int* __restrict__ in, int* out, int* block_sums,
                                                          int64_t n) {
  __shared__ int s[1024];
  const int64_t i = int64_t(blockIdx.x) * 1024 + threadIdx.x;
  const int v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) block_sums[blockIdx.x] = s[1023];
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(int* block_sums, int nb) {
  __shared__ int s[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? block_sums[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) block_sums[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += s[1023];
    __syncthreads();
  }
}

__global__ void scan_add_kernel(int* out, const int* __restrict__ block_sums, int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * 1024 + threadIdx.x;
  if (i < n) out[i] += block_sums[blockIdx.x];
}

}  // namespace fb
