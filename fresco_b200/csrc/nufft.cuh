// Non-uniform FFT building blocks on sm_100a: point binning (counting sort
// with block-local histograms), subproblem table, ES-kernel spreading into
// shared-memory tiles flushed to the fine grid with atomics, and
// interpolation from the fine grid.
//
// The method (bin-sort, spread, FFT, deconvolve / pre-correct, FFT,
// interpolate) is the one of Barnett, Magland & af Klinteberg (SIAM J. Sci.
// Comput. 41(5), 2019), which FINUFFT v2.2.0 implements for the reference
// (source/fresco/nuwu.hpp:256-258 setpts/execute; :291-309 type-2 calls).
//
// Layout conventions (all arrays in HBM):
//  * fine grid: nf[0] x nf[1] x nf[2], dimension 0 fastest (cuFFT row-major
//    with the dims passed slowest first);
//  * sorted points: one packed record per point (Rec<D,T>: absolute fine
//    cell, per-dimension fractional offset inside the cell, original index),
//    grouped by bin (a tile of `tile[]` fine cells).  Keeping the fractional
//    offset rather than the coordinate keeps full phase accuracy in FP32.
#pragma once

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "es.cuh"

namespace fb {

// Points per spreading/interpolation subproblem at most: a bin is cut into
// equal parts of at most kMaxSub points.  Each tile block stages its
// subproblem in shared memory, so kMaxSub also sets how many blocks share an
// SM; 640 gives the 2D tile kernels seven (FP32 spreading) and about two
// subproblems per bin at the benchmark's density, close to two full waves.
constexpr int kMaxSub = 640;
constexpr int kMaxBins = 32768;   // bins per geometry (block-local histograms live in shared memory)
constexpr int kTile2D = 64;       // 2D tile edge (phased spreading needs a multiple of the sub-block edge)

struct Geom {
  int D = 2;
  int w = 7;
  int nf[3] = {1, 1, 1};
  int tile[3] = {1, 1, 1};
  int nb[3] = {1, 1, 1};
  int tw[3] = {1, 1, 1};  // shared tile width per dim: tile + w (1 for unused dims)
  int pad = 3;            // w / 2
  __host__ __device__ int64_t G() const { return int64_t(nf[0]) * nf[1] * nf[2]; }
  __host__ __device__ int64_t nbins() const { return int64_t(nb[0]) * nb[1] * nb[2]; }
  __host__ __device__ int64_t tile_cells() const { return int64_t(tw[0]) * tw[1] * tw[2]; }
};

// Builds the geometry for fine sizes nf[0..D-1] and kernel width w; tiles
// grow (doubling) until there are at most kMaxBins bins.
Geom make_geom(int D, const int64_t* nf, int w, const int* tile_pref);

// How raw input coordinates become fine-grid coordinates u in [0, nf).
//  kind 0 (NUwU map, source/fresco/nuwu.hpp:216-250):
//        x = (p - round(p / L)) * 2 pi / L, u = x * nf / (2 pi)
//  kind 1 (scaled points, uwnu.hpp:243-276): x = p * 2 pi / L
struct MapParams {
  int kind = 0;
  double L[3] = {1, 1, 1};
  int stride = 2;  // doubles between consecutive points (interleaved layout)
  double scale[3] = {1, 1, 1};  // fine-grid cells per unit length, nf / L (set by the sort)
  double invL[3] = {1, 1, 1};   // 1 / L (set by the sort)
};

// Packed sorted-point records (16 or 32 bytes, read with one vector load).
template <int D, typename T> struct Rec;
template <> struct alignas(16) Rec<1, float> { uint32_t cell; float f[1]; uint32_t idx; uint32_t pad_; };
template <> struct alignas(16) Rec<2, float> { uint32_t cell; float f[2]; uint32_t idx; };
template <> struct alignas(16) Rec<3, float> { uint32_t cell; float f[3]; uint32_t idx; uint32_t pad_[3]; };
template <> struct alignas(16) Rec<1, double> { uint32_t cell; uint32_t idx; double f[1]; };
template <> struct alignas(16) Rec<2, double> { uint32_t cell; uint32_t idx; double f[2]; };
template <> struct alignas(16) Rec<3, double> { uint32_t cell; uint32_t idx; double f[3]; };

inline size_t rec_bytes(int D, bool f32) {
  if (f32) return D == 3 ? 32 : 16;
  return D == 1 ? 16 : 32;
}

struct SortBufs {
  int NB = 1;            // sort blocks (each owns a contiguous chunk of points)
  int64_t chunk = 1;     // points per sort block
  DevBuf<int> bin_total; // nbins point counts; zero between sorts (the plan pass clears it)
  DevBuf<int> blk_off;   // NB * nbins: each block's offset inside each bin (block-major)
  DevBuf<int> bin_start; // nbins + 1: first record of each bin
  DevBuf<int> sub_bin, sub_start, sub_count, num_sub;
  DevBuf<unsigned char> unsorted;  // N records in input order (written by the counting pass)
  DevBuf<unsigned> done;           // blocks of the scattering pass that finished (reset by the last one)
  int64_t max_sub = 0;
  // one-pass sort (a cooperative launch whose blocks keep their points in
  // shared memory across a grid-wide barrier): blocks and points per block,
  // decided at the first sort (one_blocks 0: the two-pass sort is used)
  int one_blocks = -1;
  int64_t one_N = -1, one_chunk = 0;
  size_t one_smem = 0;
  DevBuf<unsigned long long> bar;  // grid barrier arrivals (monotonic)
};

// Packing of an absolute fine cell (c0, c1, c2) into 32 bits.
__host__ __device__ inline uint32_t pack_cell(int D, int c0, int c1, int c2) {
  if (D == 1) return uint32_t(c0);
  if (D == 2) return uint32_t(c0) | (uint32_t(c1) << 16);
  return uint32_t(c0) | (uint32_t(c1) << 11) | (uint32_t(c2) << 22);
}
__host__ __device__ inline void unpack_cell(int D, uint32_t v, int& c0, int& c1, int& c2) {
  if (D == 1) { c0 = int(v); c1 = 0; c2 = 0; }
  else if (D == 2) { c0 = int(v & 0xffffu); c1 = int(v >> 16); c2 = 0; }
  else { c0 = int(v & 0x7ffu); c1 = int((v >> 11) & 0x7ffu); c2 = int(v >> 22); }
}

// Allocates the sort buffers for N points on geometry g.
void alloc_sort(SortBufs& sb, int64_t N, const Geom& g);

// Sorts the points into packed records (device buffer of N * rec_bytes).
template <typename T>
void bin_sort(const double* pts, int64_t N, const MapParams& mp, const Geom& g, SortBufs& sb, void* recs, int* status,
              cudaStream_t s);

// `poly` holds the kernel-tap polynomial coefficients (es_poly_coefficients).

// Spreads real strengths (weights[idx], or `uniform` when weights is null)
// onto a real fine grid (accumulated into; the caller zeroes it).
template <typename T>
void spread_real(const void* recs, const T* weights, T uniform, const SortBufs& sb, const Geom& g,
                 const std::vector<double>& poly, T* grid, cudaStream_t s);

// Spreads complex strengths (original point order) onto a complex fine grid.
template <typename T>
void spread_cplx(const void* recs, const cplx_t<T>* strengths, const SortBufs& sb, const Geom& g,
                 const std::vector<double>& poly, cplx_t<T>* grid, cudaStream_t s);

// Interpolation epilogues.
enum InterpOut : int {
  INTERP_GRAD = 0,  // grad[idx*D + a] (+)= w_idx * component, components (Re f0, Im f0, Re f1)
  INTERP_CPLX = 1,  // out2[idx] = value of field 0 (double2)
};

// Per-dimension factors applied to INTERP_GRAD outputs.
struct GradScale {
  double s[3] = {1.0, 1.0, 1.0};
};

// Interpolates `nfields` complex fine grids (field stride G) at the sorted points.
// fail_energy (may be null): the evaluation's energy, set to NaN if a tile
// copy of the 2D kernel never completes (STATUS_TIMEOUT).
template <typename T>
void interp(const void* recs, int64_t N, const T* weights, T uniform, const SortBufs& sb, const Geom& g,
            const std::vector<double>& poly, const cplx_t<T>* fields, int nfields, int mode, double* grad,
            double2* out2, int accumulate, const int* status, cudaStream_t s, GradScale gs = GradScale(),
            double* fail_energy = nullptr);

// Mbarrier polls of the first wait for an interpolation tile copy, used by
// launches from now on (< 0 restores the default, kTileWaitPolls; 0 makes
// the first wait run out at once).  Tests lower it to exercise the second,
// time-bounded wait.
constexpr int kTileWaitPolls = 1 << 22;
void set_tile_wait_polls(int polls);
int& tile_wait_polls_setting();

}  // namespace fb
