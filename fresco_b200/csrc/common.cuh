// Shared helpers for the fresco_b200 CUDA library: error handling, status
// words, reductions and small device math.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace fb {

// Error classes thrown inside the library and turned into C status codes at
// the C-ABI boundary (capi.cu).  They mirror the reference's exception types:
// std::invalid_argument -> ValueError and std::runtime_error -> RuntimeError
// in the Cython layer (fresco/potentials/nuwu.pxd:9-11).
struct InvalidArgument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    throw CudaError(std::string(what) + " failed: " + cudaGetErrorString(e) + " at " + file + ":" +
                    std::to_string(line));
  }
}
inline void cufft_check(cufftResult r, const char* what, const char* file, int line) {
  if (r != CUFFT_SUCCESS) {
    throw CudaError(std::string(what) + " failed with cufftResult " + std::to_string(int(r)) + " at " +
                    file + ":" + std::to_string(line));
  }
}
#define FB_CUDA(x) ::fb::cuda_check((x), #x, __FILE__, __LINE__)
#define FB_CUFFT(x) ::fb::cufft_check((x), #x, __FILE__, __LINE__)
#define FB_LAUNCH_CHECK() ::fb::cuda_check(cudaPeekAtLastError(), "kernel launch", __FILE__, __LINE__)

// Sticky status bits a kernel can raise; read back by the host after a call.
enum StatusBits : int {
  STATUS_NONFINITE_INPUT = 1,  // a coordinate was NaN or +-inf
  STATUS_OVERFLOW = 2,         // a bounded buffer was too small (kernel skipped the excess)
  STATUS_TIMEOUT = 4,          // a bounded wait gave up: the evaluation's energy and gradient are NaN
  STATUS_TILE_RETRY = 8,       // a tile copy outlasted its first bounded wait and was waited for again
                               // (informational: the results are complete)
  STATUS_EXACT_FALLBACK = 16,  // a point outside a type-3 plan's window: exact sums served the
                               // evaluation (informational: the results are complete)
};

// A potential's status block holds two words: [0] the flags of the current
// evaluation (cleared when it starts) and [1] the flags accumulated since the
// host last read them.
__device__ inline void raise_status(int* st, int bit) {
  atomicOr(st, bit);
  atomicOr(st + 1, bit);
}

// Nanoseconds of the GPU's global timer (bounds for waits).
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier for cooperative launches (every block resident at once).
constexpr uint64_t kGridBarrierNs = 2000000000ull;

// Waits until all blocks of this launch have arrived: launch k's blocks take
// the tickets [k n, (k + 1) n) of the counter, which only grows.  Returns false
// if the wait gave up after kGridBarrierNs.
__device__ __forceinline__ bool grid_barrier(unsigned long long* bar, unsigned nblocks) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned long long ticket = atomicAdd(bar, 1ull);
    const unsigned long long target = (ticket / nblocks + 1) * nblocks;
    const uint64_t t0 = global_ns();
    int ok = 1;
    for (;;) {
      unsigned long long v;
      asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(bar) : "memory");
      if (v >= target) break;
      if (global_ns() - t0 > kGridBarrierNs) {
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// RAII device buffer (cudaMalloc'ed once at set-up, never on the evaluation path).
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) FB_CUDA(cudaMalloc(&p, count * sizeof(T)));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

template <typename T> struct Complex;
template <> struct Complex<float> { using type = float2; };
template <> struct Complex<double> { using type = double2; };
template <typename T> using cplx_t = typename Complex<T>::type;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Warp + block reduction of a double, then one atomicAdd per block.
__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Linear thread index and thread count of the block (any block shape whose
// x extent is a multiple of 32 when y or z exceed 1).
__device__ __forceinline__ int block_tid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
__device__ __forceinline__ int block_threads() { return blockDim.x * blockDim.y * blockDim.z; }

// Adds the block-wide sum of v into *out (one atomic per block).  Every
// thread of the block must call it.
__device__ inline void block_sum_atomic(double v, double* out) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int lane = block_tid() & 31, wid = block_tid() >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    const int nw = (block_threads() + 31) >> 5;
    double s = lane < nw ? red[lane] : 0.0;
    s = warp_sum(s);
    if (lane == 0 && s != 0.0) atomicAdd(out, s);
  }
  __syncthreads();
}

// Same, for several accumulators at once (k <= 4).
template <int K>
__device__ inline void block_sum_atomic_k(double (&v)[K], double* out) {
  __shared__ double red[K][32];
  const int lane = block_tid() & 31, wid = block_tid() >> 5;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    double s = warp_sum(v[i]);
    if (lane == 0) red[i][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = (block_threads() + 31) >> 5;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      double s = lane < nw ? red[i][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) atomicAdd(out + i, s);
    }
  }
  __syncthreads();
}

// Number of SMs of the current device (cached per process for device 0..15).
int sm_count();

// Raises `kernel`'s dynamic shared-memory limit on the current device to at
// least `bytes`.  The limit belongs to the function, which every object that
// launches it shares, so it only ever grows: an object with a smaller need
// never lowers the limit under another's captured or later launches.
void ensure_dynamic_smem(const void* kernel, size_t bytes);
template <typename K>
inline void ensure_dynamic_smem(K* kernel, size_t bytes) {
  ensure_dynamic_smem(reinterpret_cast<const void*>(kernel), bytes);
}

}  // namespace fb
