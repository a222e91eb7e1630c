// Non-uniform FFT building blocks on sm_100a: point binning (counting sort),
// subproblem table, ES-kernel spreading into shared-memory tiles flushed to
// the fine grid with atomics, and interpolation from the fine grid.
//
// The method (bin-sort, spread, FFT, deconvolve / pre-correct, FFT,
// interpolate) is the one of Barnett, Magland & af Klinteberg (SIAM J. Sci.
// Comput. 41(5), 2019), which FINUFFT v2.2.0 implements for the reference
// (source/fresco/nuwu.hpp:256-258 setpts/execute; :291-309 type-2 calls).
//
// Layout conventions (all arrays in HBM):
//  * fine grid: nf[0] x nf[1] x nf[2], dimension 0 fastest (cuFFT row-major
//    with the dims passed slowest first);
//  * points are sorted by bin (a tile of `tile[]` fine cells); within the
//    sorted order each point carries its packed absolute fine cell, its
//    fractional offset inside the cell per dimension (so FP32 keeps full
//    phase accuracy), its strength and its original index.
#pragma once

#include "common.cuh"
#include "es.cuh"

namespace fb {

constexpr int kMaxSub = 1024;      // points per spreading subproblem
constexpr int kSortThreads = 256;

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

// Builds the geometry for fine sizes nf[0..D-1] and kernel width w.
Geom make_geom(int D, const int64_t* nf, int w, const int* tile_pref);

// How raw input coordinates become fine-grid coordinates u in [0, nf).
//  kind 0 (NUwU map, source/fresco/nuwu.hpp:216-250):
//        x = (p - round(p / L)) * 2 pi / L, u = x * nf / (2 pi)
//  kind 1 (scaled points, uwnu.hpp:243-276): x = p * 2 pi / L
struct MapParams {
  int kind = 0;
  double L[3] = {1, 1, 1};
  int stride = 2;  // doubles between consecutive points (interleaved layout)
};

struct SortBufs {
  DevBuf<int> bin_count, bin_start;
  DevBuf<int> sub_bin, sub_start, sub_count, num_sub;
  DevBuf<uint32_t> rank;
  int64_t max_sub = 0;
};

template <typename T>
struct SortedPts {
  uint32_t* cell = nullptr;  // packed absolute fine cell
  T* frac[3] = {nullptr, nullptr, nullptr};
  T* cw = nullptr;           // strength (real), sorted order
  uint32_t* idx = nullptr;   // original point index
};

template <typename T>
struct SortedStore {
  DevBuf<uint32_t> cell, idx;
  DevBuf<T> frac[3];
  DevBuf<T> cw;
  void alloc(int64_t n, int D) {
    cell.alloc(n);
    idx.alloc(n);
    for (int a = 0; a < D; ++a) frac[a].alloc(n);
    cw.alloc(n);
  }
  SortedPts<T> view() {
    SortedPts<T> v;
    v.cell = cell.p;
    v.idx = idx.p;
    for (int a = 0; a < 3; ++a) v.frac[a] = frac[a].p;
    v.cw = cw.p;
    return v;
  }
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

// Host driver for the binning sort.  `pts` are device doubles; `weights`
// (device, original order) may be null, in which case every strength is
// `uniform_weight`.
template <typename T>
void bin_sort(const double* pts, int64_t N, const MapParams& mp, const Geom& g, const double* weights,
              double uniform_weight, SortBufs& sb, SortedStore<T>& out, int* status, cudaStream_t s);

// Allocates the sort buffers for N points on geometry g.
void alloc_sort(SortBufs& sb, int64_t N, const Geom& g);

// Spreads real strengths of the sorted points onto a real fine grid (grid is
// accumulated into; the caller zeroes it).
template <typename T>
void spread_real(const SortedPts<T>& sp, const SortBufs& sb, const Geom& g, double beta, T* grid,
                 cudaStream_t s);

// Spreads complex strengths (given in ORIGINAL point order, cplx) onto a
// complex fine grid.
template <typename T>
void spread_cplx(const SortedPts<T>& sp, const SortBufs& sb, const Geom& g, double beta,
                 const cplx_t<T>* strengths, cplx_t<T>* grid, cudaStream_t s);

// Interpolation epilogues.
enum InterpOut : int {
  INTERP_GRAD = 0,   // NUwU gradient from packed fields (see nuwu.cu)
  INTERP_CPLX = 1,   // complex value per point, original order, written as double2
};

// Interpolates `nfields` complex fine grids (field stride G) at the sorted
// points.  INTERP_GRAD: grad[idx*D + a] (+)= cw * component, components
// (Re f0, Im f0, Re f1) for a = 0, 1, 2.  INTERP_CPLX: out2[idx] = value.
template <typename T>
void interp(const SortedPts<T>& sp, int64_t N, const Geom& g, double beta, const cplx_t<T>* fields,
            int nfields, int mode, double* grad, double2* out2, int accumulate, const int* status,
            cudaStream_t s);

}  // namespace fb
