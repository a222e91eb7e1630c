// Batched 2D NUwU ensemble (ensemble.cuh): the single-pattern pipeline of
// nuwu.cu (source/fresco/nuwu.hpp:210-317) with a pattern dimension added
// to every stage.
//
// Per group of patterns sharing a mode grid (and so a fine grid nf x nf):
//   sort     segmented bin sort: each sort block owns a chunk of ONE pattern,
//            histograms that pattern's bins in shared memory and reserves its
//            segments with one atomic per bin; the scatter blocks scan their
//            pattern's bin totals, the first block of each pattern writes its
//            bin starts and subproblem table at fixed per-pattern offsets;
//   spread   per pattern either the tiled kernel (64 x 64-cell tiles in
//            shared memory, the same body as the single-pattern kernel) or,
//            for patterns too sparse to fill tiles, a direct kernel (thread
//            per point, global atomics into the L2-resident grid); the split
//            is tuned per group by timing (tune());
//   R2C      one batched cuFFT plan over the group's grids;
//   modes    the NUwU mode pass of every pattern (its own V, S0, weights);
//   C2C      one batched cuFFT plan over the packed type-2 fields;
//            groups whose fine grid is N x N with N a power of two in
//            512..8192 and whose active modes lie in a narrow band replace
//            these three by the batched band transforms (band_fft.cuh), which
//            only touch the columns |k_x| <= Kx the loss reads;
//   interp   tiled or direct, as for the spread.
#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "band_fft.cuh"
#include "ensemble.cuh"
#include "es.cuh"
#include "nufft_kernels.cuh"
#include "nuwu_modes.cuh"

namespace fb {

Ensemble::~Ensemble() {
  for (auto& en : graphs_)
    if (en.exec) cudaGraphExecDestroy(en.exec);
  if (capture_stream_) cudaStreamDestroy(capture_stream_);
}

void Ensemble::invalidate_graphs() {
  for (auto& en : graphs_)
    if (en.exec) cudaGraphExecDestroy(en.exec);
  graphs_.clear();
  ++version_;
}

void Ensemble::eval_graph(const double* x, double* g, double* e, cudaStream_t s) {
  for (auto& en : graphs_) {
    if (en.x != x || en.g != g || en.e != e) continue;
    if (!en.exec) {
      if (!capture_stream_) FB_CUDA(cudaStreamCreateWithFlags(&capture_stream_, cudaStreamNonBlocking));
      cudaGraph_t graph = nullptr;
      FB_CUDA(cudaStreamBeginCapture(capture_stream_, cudaStreamCaptureModeRelaxed));
      try {
        eval(x, g, e, capture_stream_);
      } catch (...) {
        cudaStreamEndCapture(capture_stream_, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      FB_CUDA(cudaStreamEndCapture(capture_stream_, &graph));
      const cudaError_t ie = cudaGraphInstantiate(&en.exec, graph, 0);
      cudaGraphDestroy(graph);
      FB_CUDA(ie);
    }
    FB_CUDA(cudaGraphLaunch(en.exec, s));
    return;
  }
  if (graphs_.size() >= 8) invalidate_graphs();
  graphs_.push_back(GraphEntry{x, g, e, nullptr});
  eval(x, g, e, s);
}

namespace {

constexpr int kEnsSortThreads = 512;
constexpr int kEnsSortChunk = 2048;  // points per sort block
constexpr int kDirectPts = 256;      // points per block of the direct spread / interpolation
// Subproblem sizes (points per tile block) the tuner tries, smallest first;
// the subproblem slots are sized for the smallest.
constexpr int kSubCaps[3] = {kMaxSub / 4, kMaxSub / 2, kMaxSub};

// Per pattern of a group (device copy read with one load per block).
struct alignas(16) PatInfo {
  int64_t pt_base;   // first global point index
  double invN;       // 1 / N
  double uniform;    // weight when the ensemble has no per-point weights
  int rec_base;      // first record in the group's record arrays
  int npts;
  int first_item;    // first sort block
  int n_items;       // sort blocks
  int sub_base;      // first subproblem slot
  int max_sub;       // subproblem slots
  int pid;           // pattern index in the ensemble
  int mode_base;     // first active mode in the group's mode table
  int n_active;      // active modes
  int sub_cap;       // points per subproblem at most (<= kMaxSub; tuned per group)
};

struct SortItem {
  int64_t j0, j1;  // global point range
  int l, pad_;     // pattern of the group
};

struct PointItem {
  int start, count, l, pad_;  // record range of pattern l (direct kernels)
};

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

template <typename T>
__global__ void __launch_bounds__(kEnsSortThreads) ens_sort_count_kernel(
    const double* __restrict__ x, const SortItem* __restrict__ items, const PatInfo* __restrict__ pats, MapParams mp,
    Geom g, int* bin_total, int* blk_off, Rec<2, T>* unsorted, int* cur_status, int* sticky) {
  extern __shared__ int hist[];
  const int nbins = int(g.nbins());
  const SortItem it = items[blockIdx.x];
  const PatInfo pi = pats[it.l];
  for (int i = threadIdx.x; i < nbins; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  bool bad = false;
  for (int64_t j = it.j0 + threadIdx.x; j < it.j1; j += blockDim.x) {
    const double p[2] = {x[2 * j], x[2 * j + 1]};
    int c[3] = {0, 0, 0};
    double f[3] = {0, 0, 0};
    bool ok;
    const int bin = point_bin<2>(p, mp, g, c, f, ok);
    bad |= !ok;
    atomicAdd(&hist[bin], 1);
    Rec<2, T> r;
    r.cell = pack_cell(2, c[0], c[1], 0);
    r.f[0] = T(f[0]);
    r.f[1] = T(f[1]);
    r.idx = uint32_t(j);
    unsorted[pi.rec_base + (j - pi.pt_base)] = r;
  }
  if (bad) {
    atomicOr(cur_status + pi.pid, STATUS_NONFINITE_INPUT);
    atomicOr(sticky + pi.pid, STATUS_NONFINITE_INPUT);
  }
  __syncthreads();
  int* my = blk_off + int64_t(blockIdx.x) * nbins;
  int* tot = bin_total + int64_t(it.l) * nbins;
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
    const int cnt = hist[b];
    if (cnt) my[b] = atomicAdd(&tot[b], cnt);
  }
}

template <typename T>
__global__ void __launch_bounds__(kEnsSortThreads) ens_sort_scatter_kernel(
    const Rec<2, T>* __restrict__ unsorted, const SortItem* __restrict__ items, const PatInfo* __restrict__ pats,
    Geom g, int* bin_total, const int* __restrict__ blk_off, int* bin_start, int* sub_bin, int* sub_start,
    int* sub_count, int* num_sub, unsigned* done, Rec<2, T>* out, int* sticky) {
  extern __shared__ int sh_cur[];
  __shared__ int s_warp[32];
  __shared__ bool s_last;
  const int nbins = int(g.nbins());
  const int tid = threadIdx.x;
  const SortItem it = items[blockIdx.x];
  const int l = it.l;
  const PatInfo pi = pats[l];
  int* tot = bin_total + int64_t(l) * nbins;
  const int* my_off = blk_off + int64_t(blockIdx.x) * nbins;
  int* bs = bin_start + int64_t(l) * (nbins + 1);
  const bool first = int(blockIdx.x) == pi.first_item;
  const int per = (nbins + int(blockDim.x) - 1) / int(blockDim.x);
  const int b0 = min(nbins, tid * per), b1 = min(nbins, b0 + per);
  int npts = 0, nsub = 0;
  for (int b = b0; b < b1; ++b) {
    const int c = tot[b];
    npts += c;
    nsub += (c + pi.sub_cap - 1) / pi.sub_cap;
  }
  int tot_pts;
  int run = block_exclusive_scan(npts, &tot_pts, s_warp);
  const int first_start = run;
  for (int b = b0; b < b1; ++b) {
    sh_cur[b] = pi.rec_base + run + my_off[b];  // stale for bins without points of this block; never used
    if (first) bs[b] = pi.rec_base + run;
    run += tot[b];
  }
  if (first) {
    int tot_sub;
    int sbase = block_exclusive_scan(nsub, &tot_sub, s_warp);
    int st = pi.rec_base + first_start;
    for (int b = b0; b < b1; ++b) {
      const int c = tot[b];
      const int parts = (c + pi.sub_cap - 1) / pi.sub_cap;  // equal parts of at most sub_cap points
      for (int q = 0; q < parts; ++q) {
        if (sbase < pi.max_sub) {
          const int si = pi.sub_base + sbase;
          const int lo = int(int64_t(q) * c / parts), hi = int(int64_t(q + 1) * c / parts);
          sub_bin[si] = b;
          sub_start[si] = st + lo;
          sub_count[si] = hi - lo;
        }
        ++sbase;
      }
      st += c;
    }
    if (tid == 0) {
      bs[nbins] = pi.rec_base + tot_pts;
      num_sub[l] = min(tot_sub, pi.max_sub);
    }
  }
  __syncthreads();
  for (int64_t j = it.j0 + tid; j < it.j1; j += blockDim.x) {
    const Rec<2, T> r = unsorted[pi.rec_base + (j - pi.pt_base)];
    int c[3] = {0, 0, 0};
    unpack_cell(2, r.cell, c[0], c[1], c[2]);
    const int dest = atomicAdd(&sh_cur[bin_of_cell<2>(c, g)], 1);
    if (dest < pi.rec_base || dest >= pi.rec_base + pi.npts) {
      atomicOr(sticky + pi.pid, STATUS_OVERFLOW);
      continue;
    }
    out[dest] = r;
  }
  // every block of the pattern has read its bin totals before it counts itself done
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(done + l, 1u) == unsigned(pi.n_items - 1);
  }
  __syncthreads();
  if (s_last) {
    for (int b = tid; b < nbins; b += blockDim.x) tot[b] = 0;
    if (tid == 0) done[l] = 0u;
  }
}

// Block b of the tiled kernels handles subproblem slot tab[b].y of pattern
// tab[b].x of the group; the pattern's grid starts at pattern x G.
template <typename T>
struct EnsTileMap {
  const PatInfo* __restrict__ pats;
  const int2* __restrict__ tab;
  const int* __restrict__ sub_bin;
  const int* __restrict__ sub_start;
  const int* __restrict__ sub_count;
  const int* __restrict__ num_sub;
  const int* __restrict__ bin_start;
  const int* __restrict__ cur_status;
  int64_t G;
  __device__ __forceinline__ bool fetch(const Geom& g, TileWork<T>& w) const {
    const int2 bt = tab[blockIdx.x];
    if (bt.y >= num_sub[bt.x]) return false;
    const PatInfo& pi = pats[bt.x];
    const int si = pi.sub_base + bt.y;
    const int bin = sub_bin[si];
    w.start = sub_start[si];
    w.cnt = sub_count[si];
    w.org0 = (bin % g.nb[0]) * kTile2D;
    w.org1 = (bin / g.nb[0]) * kTile2D;
    w.bin_range = bin_start + int64_t(bt.x) * (g.nbins() + 1) + bin;
    w.grid_off = int64_t(bt.x) * G;
    w.uniform = T(pi.uniform);
    return true;
  }
  __device__ __forceinline__ bool nonfinite(const TileWork<T>&) const {
    return (cur_status[pats[tab[blockIdx.x].x].pid] & STATUS_NONFINITE_INPUT) != 0;
  }
  // tiles are read with plain loads (one grid per pattern)
  __device__ __forceinline__ const CUtensorMap* tile_tmap() const { return nullptr; }
  __device__ __forceinline__ int* err_status() const { return nullptr; }
  __device__ __forceinline__ int wait_polls() const { return 0; }
  __device__ __forceinline__ double* fail_energy() const { return nullptr; }
};

// Direct spreading for sparse patterns: thread per sorted point, the w x w
// taps added to the grid with global atomics.
template <int W, typename T>
__global__ void __launch_bounds__(kDirectPts) ens_spread_direct_kernel(const Rec<2, T>* __restrict__ recs,
                                                                       const T* __restrict__ weights,
                                                                       const PatInfo* __restrict__ pats,
                                                                       const PointItem* __restrict__ items, Geom g,
                                                                       const EsPoly<W, T> poly, T* grid, int64_t G) {
  const PointItem it = items[blockIdx.x];
  if (int(threadIdx.x) >= it.count) return;
  const Rec<2, T> r = recs[it.start + threadIdx.x];
  const T wgt = weights ? weights[r.idx] : T(pats[it.l].uniform);
  int c0, c1, c2;
  unpack_cell(2, r.cell, c0, c1, c2);
  T k0[W], k1[W];
  const int s0 = es_taps<W, T>(r.f[0], poly, k0);
  const int s1 = es_taps<W, T>(r.f[1], poly, k1);
  const int nf0 = g.nf[0], nf1 = g.nf[1];
  int ix[W];
#pragma unroll
  for (int m = 0; m < W; ++m) ix[m] = wrap_index(c0 + s0 + m, nf0);
  T* gp = grid + int64_t(it.l) * G;
#pragma unroll
  for (int m1 = 0; m1 < W; ++m1) {
    T* row = gp + int64_t(wrap_index(c1 + s1 + m1, nf1)) * nf0;
    const T wy = wgt * k1[m1];
#pragma unroll
    for (int m0 = 0; m0 < W; ++m0) atomicAdd(row + ix[m0], wy * k0[m0]);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) ens_modes_kernel(const PatInfo* __restrict__ pats,
                                                        const int* __restrict__ mode_idx,
                                                        const ModeCoef* __restrict__ coef, int n, int K,
                                                        const cplx_t<T>* __restrict__ bhat, int nh0, int64_t GH,
                                                        int nf, const double* __restrict__ corr, cplx_t<T>* hgrid,
                                                        int64_t G, double* energy, const int* __restrict__ cur_status,
                                                        int want_grad) {
  const int l = blockIdx.y;
  const PatInfo pi = pats[l];
  double phi = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < pi.n_active; i += gridDim.x * blockDim.x) {
    const int mi = pi.mode_base + i;
    phi += nuwu_mode_term<2, T>(mode_idx[mi], n, K, coef[mi], bhat + int64_t(l) * GH, nh0, nf, nf, 1, corr, corr,
                                corr, pi.invN, hgrid + int64_t(l) * G, G, want_grad != 0);
  }
  block_sum_atomic(phi, energy + pi.pid);
  if (blockIdx.x == 0 && threadIdx.x == 0 && (cur_status[pi.pid] & STATUS_NONFINITE_INPUT))
    atomicAdd(energy + pi.pid, __longlong_as_double(0x7ff8000000000000ULL));
}

template <int W, typename T>
__global__ void __launch_bounds__(kDirectPts) ens_interp_direct_kernel(
    const Rec<2, T>* __restrict__ recs, const T* __restrict__ weights, const PatInfo* __restrict__ pats,
    const PointItem* __restrict__ items, Geom g, const EsPoly<W, T> poly, const cplx_t<T>* __restrict__ field,
    int64_t G, double* grad, const int* __restrict__ cur_status) {
  const PointItem it = items[blockIdx.x];
  if (int(threadIdx.x) >= it.count) return;
  const PatInfo pi = pats[it.l];
  const Rec<2, T> r = recs[it.start + threadIdx.x];
  int c0, c1, c2;
  unpack_cell(2, r.cell, c0, c1, c2);
  T k0[W], k1[W];
  const int s0 = es_taps<W, T>(r.f[0], poly, k0);
  const int s1 = es_taps<W, T>(r.f[1], poly, k1);
  const int nf0 = g.nf[0], nf1 = g.nf[1];
  int ix[W];
#pragma unroll
  for (int m = 0; m < W; ++m) ix[m] = wrap_index(c0 + s0 + m, nf0);
  const cplx_t<T>* fp = field + int64_t(it.l) * G;
  T vr = 0, vi = 0;
#pragma unroll
  for (int m1 = 0; m1 < W; ++m1) {
    const cplx_t<T>* row = fp + int64_t(wrap_index(c1 + s1 + m1, nf1)) * nf0;
    T rr = 0, ri = 0;
#pragma unroll
    for (int m0 = 0; m0 < W; ++m0) {
      const cplx_t<T> a = __ldg(row + ix[m0]);
      rr += a.x * k0[m0];
      ri += a.y * k0[m0];
    }
    vr += k1[m1] * rr;
    vi += k1[m1] * ri;
  }
  const T wgt = weights ? weights[r.idx] : T(pi.uniform);
  const bool bad = (cur_status[pi.pid] & STATUS_NONFINITE_INPUT) != 0;
  interp_store<2, T>(INTERP_GRAD, r.idx, wgt, vr, vi, T(0), bad, grad, nullptr, 0, GradScale());
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

#define FB_ENS_W(T, X)                                                               \
  switch (es_.w) {                                                                   \
    case 2: X(2); break;                                                             \
    case 3: X(3); break;                                                             \
    case 4: X(4); break;                                                             \
    case 5: X(5); break;                                                             \
    case 6: X(6); break;                                                             \
    case 7: X(7); break;                                                             \
    case 8: X(8); break;                                                             \
    case 9: X(9); break;                                                             \
    case 10: X(10); break;                                                           \
    case 11: X(FB_WCLAMP(T, 11)); break;                                             \
    case 12: X(FB_WCLAMP(T, 12)); break;                                             \
    case 13: X(FB_WCLAMP(T, 13)); break;                                             \
    case 14: X(FB_WCLAMP(T, 14)); break;                                             \
    case 15: X(FB_WCLAMP(T, 15)); break;                                             \
    case 16: X(FB_WCLAMP(T, 16)); break;                                             \
    default: throw InvalidArgument("unsupported kernel width");                      \
  }

template <typename T>
class NUwUEnsembleImpl final : public Ensemble {
  struct Group {
    int n = 1, K = 0, P = 0;
    Geom geom;
    int nbins = 1, nh0 = 1;
    int64_t G = 1, GH = 1, NG = 0;
    std::vector<PatInfo> pats_h;
    int sub_cap = kMaxSub;  // points per subproblem (tune())
    DevBuf<PatInfo> pats;
    int n_items = 0;
    DevBuf<SortItem> items;
    DevBuf<int> bin_total, blk_off, bin_start, sub_bin, sub_start, sub_count, num_sub;
    DevBuf<unsigned> done;
    DevBuf<unsigned char> unsorted, recs;
    DevBuf<T> spread;
    DevBuf<cplx_t<T>> bhat, hgrid, ggrid;
    DevBuf<double> corr;
    DevBuf<int> mode_idx;
    DevBuf<ModeCoef> coef;
    int max_active = 0;
    // spreading / interpolation split (tune())
    std::vector<char> direct;  // per pattern
    double ratio = 1.0;
    DevBuf<int2> tab;
    int n_tab = 0;
    DevBuf<PointItem> pitems;
    int n_pitems = 0;
    cufftHandle r2c = 0, c2c = 0;
    // band transforms
    bool band = false;
    int Kx = 0, Ky = 0;
    DevBuf<cplx_t<T>> tw, band1, band2;
    DevBuf<ModeCoef> coef_box;
    DevBuf<double> invN;
    DevBuf<int> pid;
    size_t smem_rows = 0, smem_modes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;
  };

 public:
  NUwUEnsembleImpl(int P, const int64_t* n_points, const double* radii, const int64_t* n_modes, const double* sk,
                   const double* v, const double* L, double eps) {
    if (P < 1) throw InvalidArgument("an ensemble needs at least one pattern");
    L_[0] = L[0];
    L_[1] = L[1];
    if (!(L_[0] > 0.0) || !(L_[1] > 0.0)) throw InvalidArgument("box lengths must be positive");
    es_ = es_params(eps, sizeof(T) == 4 ? 10 : 16);
    poly_ = es_poly_coefficients(es_, es_.w);
    P_ = P;
    dof_off_.assign(P + 1, 0);
    std::vector<int64_t> mode_off(P + 1, 0);
    std::vector<int> nper(P);
    for (int p = 0; p < P; ++p) {
      if (n_points[p] < 1) throw InvalidArgument("every pattern needs at least one point");
      dof_off_[p + 1] = dof_off_[p] + 2 * n_points[p];
      mode_off[p + 1] = mode_off[p] + n_modes[p];
      // nuwu.hpp:54-79: K = int((sqrt(len V) - 1) / 2)
      const int kk = int((std::sqrt(double(n_modes[p])) - 1) / 2);
      nper[p] = 2 * kk + 1;
      if (int64_t(nper[p]) * nper[p] > n_modes[p]) throw InvalidArgument("V too short for its mode grid");
    }
    if (dof_off_[P] / 2 >= (int64_t(1) << 32)) throw InvalidArgument("too many points in one ensemble");
    // weights, nuwu.hpp:125-149, normalised per pattern
    std::vector<double> c(size_t(dof_off_[P] / 2), 1.0);
    std::vector<double> uni(P, 1.0);
    bool all_uniform = true;
    for (int p = 0; p < P; ++p) {
      const int64_t b = dof_off_[p] / 2, np = n_points[p];
      double sum = 0.0;
      for (int64_t i = 0; i < np; ++i) {
        double ci = 1.0;
        for (int a = 0; a < 2; ++a) ci = ci * M_PI * radii[b + i] * radii[b + i];
        c[b + i] = ci;
        sum += ci;
      }
      bool u = true;
      for (int64_t i = 0; i < np; ++i) {
        c[b + i] *= double(np) / sum;
        if (c[b + i] != c[b]) u = false;
      }
      uni[p] = c[b];
      all_uniform &= u;
    }
    if (!all_uniform) {
      std::vector<T> ct(c.begin(), c.end());
      weights_.alloc(ct.size());
      FB_CUDA(cudaMemcpy(weights_.p, ct.data(), sizeof(T) * ct.size(), cudaMemcpyHostToDevice));
    }
    cur_status_.alloc(P);
    sticky_.alloc(P);
    FB_CUDA(cudaMemset(cur_status_.p, 0, cur_status_.bytes()));
    FB_CUDA(cudaMemset(sticky_.p, 0, sticky_.bytes()));
    FB_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));

    std::map<int, std::vector<int>> by_n;
    for (int p = 0; p < P; ++p) by_n[nper[p]].push_back(p);
    for (auto& kv : by_n) {
      groups_.emplace_back(new Group);
      build_group(*groups_.back(), kv.first, kv.second, n_points, mode_off, sk, v, uni);
    }
    FB_CUDA(cudaDeviceSynchronize());
  }

  ~NUwUEnsembleImpl() override {
    for (auto& gp : groups_) {
      if (gp->r2c) cufftDestroy(gp->r2c);
      if (gp->c2c) cufftDestroy(gp->c2c);
      if (gp->stream) cudaStreamDestroy(gp->stream);
      if (gp->join) cudaEventDestroy(gp->join);
    }
    if (fork_) cudaEventDestroy(fork_);
  }

  void eval(const double* x, double* g, double* e, cudaStream_t s) override {
    FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double) * P_, s));
    FB_CUDA(cudaMemsetAsync(cur_status_.p, 0, cur_status_.bytes(), s));
    FB_CUDA(cudaEventRecord(fork_, s));
    for (auto& gp : groups_) {
      FB_CUDA(cudaStreamWaitEvent(gp->stream, fork_, 0));
      run_group(*gp, x, g, e, gp->stream);
      FB_CUDA(cudaEventRecord(gp->join, gp->stream));
      FB_CUDA(cudaStreamWaitEvent(s, gp->join, 0));
    }
  }

  void read_and_clear_status(int* out, cudaStream_t s) override {
    FB_CUDA(cudaMemcpyAsync(out, sticky_.p, sticky_.bytes(), cudaMemcpyDeviceToHost, s));
    FB_CUDA(cudaMemsetAsync(sticky_.p, 0, sticky_.bytes(), s));
    FB_CUDA(cudaStreamSynchronize(s));
  }

  void tune(const double* x, double* g, double* e, cudaStream_t s) override {
    invalidate_graphs();
    FB_CUDA(cudaDeviceSynchronize());  // no launch may still read the split tables
    cudaEvent_t t0, t1;
    FB_CUDA(cudaEventCreate(&t0));
    FB_CUDA(cudaEventCreate(&t1));
    FB_CUDA(cudaMemsetAsync(e, 0, sizeof(double) * P_, s));
    FB_CUDA(cudaMemsetAsync(cur_status_.p, 0, cur_status_.bytes(), s));
    for (auto& gp : groups_) {
      Group& gr = *gp;
      double best_ms = 1e300, best_ratio = gr.ratio;
      int best_cap = gr.sub_cap;
      for (int cap : kSubCaps) {  // points per subproblem x direct/tiled split
        set_cap(gr, cap);
        for (double r : {0.0, 0.0625, 0.25, 1.0, 4.0, 16.0, 1e30}) {
          set_split(gr, r);
          run_group(gr, x, g, e, s);  // warm-up
          FB_CUDA(cudaEventRecord(t0, s));
          for (int rep = 0; rep < 3; ++rep) run_group(gr, x, g, e, s);
          FB_CUDA(cudaEventRecord(t1, s));
          FB_CUDA(cudaEventSynchronize(t1));
          float ms = 0.f;
          FB_CUDA(cudaEventElapsedTime(&ms, t0, t1));
          if (ms < best_ms) {
            best_ms = ms;
            best_ratio = r;
            best_cap = cap;
          }
        }
      }
      gr.ratio = best_ratio;
      set_cap(gr, best_cap);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    FB_CUDA(cudaStreamSynchronize(s));
  }

  void set_split(double ratio) override {
    invalidate_graphs();
    FB_CUDA(cudaDeviceSynchronize());  // no launch may still read the split tables
    for (auto& gp : groups_) set_split(*gp, ratio);
  }

  void set_subproblem_cap(int cap) override {
    if (cap < kSubCaps[0] || cap > kMaxSub)
      throw InvalidArgument("the subproblem size must lie in [" + std::to_string(kSubCaps[0]) + ", " +
                            std::to_string(kMaxSub) + "]");
    invalidate_graphs();
    FB_CUDA(cudaDeviceSynchronize());  // no launch may still read the split tables
    for (auto& gp : groups_) set_cap(*gp, cap);
  }

  std::string describe() const override {
    std::string out = "NUwU ensemble precision=" + std::string(sizeof(T) == 4 ? "fp32" : "fp64") +
                      " patterns=" + std::to_string(P_) + " w=" + std::to_string(es_.w) +
                      " groups=" + std::to_string(groups_.size());
    for (const auto& gp : groups_) {
      int nd = 0;
      for (char d : gp->direct) nd += d ? 1 : 0;
      out += " [modes/dim=" + std::to_string(gp->n) + " nf=" + std::to_string(gp->geom.nf[0]) +
             " patterns=" + std::to_string(gp->P) + " points=" + std::to_string(gp->NG) +
             " direct=" + std::to_string(nd) + " subproblem<=" + std::to_string(gp->sub_cap) +
             (gp->band ? " fft=band|kx|<=" + std::to_string(gp->Kx) + ",|ky|<=" + std::to_string(gp->Ky)
                       : std::string(" fft=cufft")) + "]";
    }
    return out;
  }

 private:
  void build_group(Group& gr, int n, const std::vector<int>& pids, const int64_t* n_points,
                   const std::vector<int64_t>& mode_off, const double* sk, const double* v,
                   const std::vector<double>& uni) {
    gr.n = n;
    gr.K = n / 2;
    gr.P = int(pids.size());
    const int64_t nf = fine_grid_size(n, es_.w);
    const int64_t nfs[3] = {nf, nf, 1};
    const int tile[3] = {kTile2D, kTile2D, 1};
    gr.geom = make_geom(2, nfs, es_.w, tile);
    gr.nbins = int(gr.geom.nbins());
    gr.G = nf * nf;
    gr.nh0 = int(nf / 2 + 1);
    gr.GH = int64_t(gr.nh0) * nf;
    if (int64_t(gr.P) * gr.G >= (int64_t(1) << 31)) throw InvalidArgument("too many patterns of one grid size");
    std::vector<SortItem> items;
    std::vector<int> midx;
    std::vector<ModeCoef> mcoef;
    int rec = 0, sub = 0;
    for (int l = 0; l < gr.P; ++l) {
      const int p = pids[l];
      PatInfo pi{};
      pi.pt_base = dof_off_[p] / 2;
      pi.npts = int(n_points[p]);
      pi.invN = 1.0 / double(n_points[p]);
      pi.uniform = uni[p];
      pi.rec_base = rec;
      pi.first_item = int(items.size());
      for (int64_t j = 0; j < pi.npts; j += kEnsSortChunk)
        items.push_back(SortItem{pi.pt_base + j, pi.pt_base + std::min<int64_t>(pi.npts, j + kEnsSortChunk), l, 0});
      pi.n_items = int(items.size()) - pi.first_item;
      pi.sub_base = sub;
      pi.max_sub = int(gr.nbins + ceil_div(pi.npts, kSubCaps[0]));
      pi.sub_cap = gr.sub_cap;
      pi.pid = p;
      std::vector<int> idx;
      std::vector<ModeCoef> cf;
      nuwu_mode_table(2, n, v + mode_off[p], sk + mode_off[p], idx, cf);
      pi.mode_base = int(midx.size());
      pi.n_active = int(idx.size());
      gr.max_active = std::max(gr.max_active, pi.n_active);
      midx.insert(midx.end(), idx.begin(), idx.end());
      mcoef.insert(mcoef.end(), cf.begin(), cf.end());
      rec += pi.npts;
      sub += pi.max_sub;
      gr.pats_h.push_back(pi);
    }
    gr.NG = rec;
    gr.n_items = int(items.size());
    gr.pats.alloc(gr.P);
    FB_CUDA(cudaMemcpy(gr.pats.p, gr.pats_h.data(), sizeof(PatInfo) * gr.P, cudaMemcpyHostToDevice));
    gr.items.alloc(items.size());
    FB_CUDA(cudaMemcpy(gr.items.p, items.data(), sizeof(SortItem) * items.size(), cudaMemcpyHostToDevice));
    gr.bin_total.alloc(int64_t(gr.P) * gr.nbins);
    FB_CUDA(cudaMemset(gr.bin_total.p, 0, gr.bin_total.bytes()));
    gr.blk_off.alloc(int64_t(gr.n_items) * gr.nbins);
    gr.bin_start.alloc(int64_t(gr.P) * (gr.nbins + 1));
    gr.sub_bin.alloc(sub);
    gr.sub_start.alloc(sub);
    gr.sub_count.alloc(sub);
    gr.num_sub.alloc(gr.P);
    FB_CUDA(cudaMemset(gr.num_sub.p, 0, gr.num_sub.bytes()));
    gr.done.alloc(gr.P);
    FB_CUDA(cudaMemset(gr.done.p, 0, gr.done.bytes()));
    const size_t rb = rec_bytes(2, sizeof(T) == 4);
    gr.unsorted.alloc(size_t(gr.NG) * rb);
    gr.recs.alloc(size_t(gr.NG) * rb);
    gr.spread.alloc(size_t(gr.P) * gr.G);
    FB_CUDA(cudaMemset(gr.spread.p, 0, gr.spread.bytes()));
    gr.ggrid.alloc(size_t(gr.P) * gr.G);
    setup_band(gr, midx, mcoef);
    if (!gr.band) {
      gr.bhat.alloc(size_t(gr.P) * gr.GH);
      gr.hgrid.alloc(size_t(gr.P) * gr.G);
      FB_CUDA(cudaMemset(gr.hgrid.p, 0, gr.hgrid.bytes()));
    }
    const std::vector<double> pc = es_correction(es_, nf, -gr.K, n);
    gr.corr.alloc(n);
    FB_CUDA(cudaMemcpy(gr.corr.p, pc.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    if (!midx.empty()) {
      gr.mode_idx.alloc(midx.size());
      gr.coef.alloc(mcoef.size());
      FB_CUDA(cudaMemcpy(gr.mode_idx.p, midx.data(), sizeof(int) * midx.size(), cudaMemcpyHostToDevice));
      FB_CUDA(cudaMemcpy(gr.coef.p, mcoef.data(), sizeof(ModeCoef) * mcoef.size(), cudaMemcpyHostToDevice));
    }
    // split tables at their largest size; set_split fills them
    gr.tab.alloc(std::max(sub, 1));
    int64_t npi = 0;
    for (const PatInfo& pi : gr.pats_h) npi += ceil_div(pi.npts, kDirectPts);
    gr.pitems.alloc(std::max<int64_t>(npi, 1));
    gr.direct.assign(gr.P, 0);
    set_split(gr, 1.0);
    if (!gr.band) {  // batched cuFFT plans (rows of nf, dims slowest first)
      const bool f32 = sizeof(T) == 4;
      int dims[2] = {int(nf), int(nf)};
      int emb_r[2] = {int(nf), int(nf)}, emb_h[2] = {int(nf), gr.nh0};
      FB_CUFFT(cufftPlanMany(&gr.r2c, 2, dims, emb_r, 1, int(gr.G), emb_h, 1, int(gr.GH),
                             f32 ? CUFFT_R2C : CUFFT_D2Z, gr.P));
      FB_CUFFT(cufftPlanMany(&gr.c2c, 2, dims, emb_r, 1, int(gr.G), emb_r, 1, int(gr.G),
                             f32 ? CUFFT_C2C : CUFFT_Z2Z, gr.P));
    }
    FB_CUDA(cudaStreamCreateWithFlags(&gr.stream, cudaStreamNonBlocking));
    FB_CUDA(cudaEventCreateWithFlags(&gr.join, cudaEventDisableTiming));
    smem_attrs();
  }

  // Band transforms for the group when its grid and active modes allow them
  // (the same conditions as the single-pattern potential).
  void setup_band(Group& gr, const std::vector<int>& midx, const std::vector<ModeCoef>& mcoef) {
    gr.band = false;
    const int nf = gr.geom.nf[0];
    if (midx.empty() || nf < 512 || nf > 8192 || (nf & (nf - 1)) != 0) return;
    if (3 * size_t(fft_padded(nf)) * sizeof(cplx_t<T>) > 200 * 1024) return;
    int kxm = 0, kym = 0;
    for (int m : midx) {
      kxm = std::max(kxm, std::abs(m % gr.n - gr.K));
      kym = std::max(kym, std::abs(m / gr.n - gr.K));
    }
    if (2 * kxm + 1 > nf / 2) return;
    gr.Kx = kxm;
    gr.Ky = kym;
    const int NX = 2 * kxm + 1, NY = 2 * kym + 1;
    std::vector<ModeCoef> box(size_t(gr.P) * NX * NY, ModeCoef{0.0, 0.0, 0.0, 0.0});
    std::vector<double> invn(gr.P);
    std::vector<int> pid(gr.P);
    for (int l = 0; l < gr.P; ++l) {
      const PatInfo& pi = gr.pats_h[l];
      invn[l] = pi.invN;
      pid[l] = pi.pid;
      for (int i = 0; i < pi.n_active; ++i) {
        const int m = midx[size_t(pi.mode_base) + i];
        const int kx = m % gr.n - gr.K, ky = m / gr.n - gr.K;
        box[size_t(l) * NX * NY + size_t(kx + kxm) * NY + (ky + kym)] = mcoef[size_t(pi.mode_base) + i];
      }
    }
    gr.coef_box.alloc(box.size());
    FB_CUDA(cudaMemcpy(gr.coef_box.p, box.data(), sizeof(ModeCoef) * box.size(), cudaMemcpyHostToDevice));
    gr.invN.alloc(gr.P);
    FB_CUDA(cudaMemcpy(gr.invN.p, invn.data(), sizeof(double) * gr.P, cudaMemcpyHostToDevice));
    gr.pid.alloc(gr.P);
    FB_CUDA(cudaMemcpy(gr.pid.p, pid.data(), sizeof(int) * gr.P, cudaMemcpyHostToDevice));
    const std::vector<double> t = fft_twiddles(nf);
    std::vector<cplx_t<T>> h(nf);
    for (int j = 0; j < nf; ++j) {
      h[j].x = T(t[2 * size_t(j)]);
      h[j].y = T(t[2 * size_t(j) + 1]);
    }
    gr.tw.alloc(nf);
    FB_CUDA(cudaMemcpy(gr.tw.p, h.data(), sizeof(cplx_t<T>) * nf, cudaMemcpyHostToDevice));
    gr.band1.alloc(size_t(gr.P) * (kxm + 1) * nf);
    gr.band2.alloc(size_t(gr.P) * nf * NX);
    gr.smem_rows = 2 * size_t(fft_padded(nf)) * sizeof(cplx_t<T>);
    gr.smem_modes = 3 * size_t(fft_padded(nf)) * sizeof(cplx_t<T>);
    switch (nf) {
      case 512: band_attrs<512>(gr); break;
      case 1024: band_attrs<1024>(gr); break;
      case 2048: band_attrs<2048>(gr); break;
      case 4096: band_attrs<4096>(gr); break;
      default: band_attrs<8192>(gr); break;
    }
    gr.band = true;
  }

  template <int N>
  void band_attrs(const Group& gr) {
    ensure_dynamic_smem(band_rows_r2c_kernel<T, N>, gr.smem_rows);
    ensure_dynamic_smem(band_rows_c2c_kernel<T, N>, gr.smem_rows);
    ensure_dynamic_smem(band_modes_kernel<T, N>, gr.smem_modes);
  }

  template <int N>
  void run_band_n(Group& gr, double* g, double* e, cudaStream_t s) {
    const dim3 blk(N / 16, 2);
    const int NX = 2 * gr.Kx + 1, NY = 2 * gr.Ky + 1;
    const BandBatch<T> bb{gr.spread.p, gr.G,         gr.band1.p,           int64_t(gr.Kx + 1) * N,
                          gr.band2.p,  int64_t(N) * NX, gr.ggrid.p,        gr.G,
                          gr.coef_box.p, int64_t(NX) * NY, gr.invN.p,      0.0,
                          e,           cur_status_.p, gr.pid.p};
    band_rows_r2c_kernel<T, N><<<dim3(N / 4, gr.P), blk, gr.smem_rows, s>>>(gr.spread.p, gr.G, gr.tw.p, gr.Kx + 1,
                                                                           gr.band1.p, int64_t(gr.Kx + 1) * N);
    FB_LAUNCH_CHECK();
    band_modes_kernel<T, N><<<dim3(gr.Kx + 1, gr.P), blk, gr.smem_modes, s>>>(bb, gr.tw.p, gr.Kx, gr.Ky, gr.K,
                                                                              gr.corr.p, gr.corr.p, g != nullptr);
    FB_LAUNCH_CHECK();
    if (!g) return;
    band_rows_c2c_kernel<T, N><<<dim3(N / 2, gr.P), blk, gr.smem_rows, s>>>(bb, gr.Kx, gr.tw.p);
    FB_LAUNCH_CHECK();
  }

  void run_band(Group& gr, double* g, double* e, cudaStream_t s) {
    switch (gr.geom.nf[0]) {
      case 512: run_band_n<512>(gr, g, e, s); break;
      case 1024: run_band_n<1024>(gr, g, e, s); break;
      case 2048: run_band_n<2048>(gr, g, e, s); break;
      case 4096: run_band_n<4096>(gr, g, e, s); break;
      default: run_band_n<8192>(gr, g, e, s); break;
    }
  }

  // Subproblems of at most cap points (bins cut into equal parts), then the
  // split tables for them.
  void set_cap(Group& gr, int cap) {
    gr.sub_cap = cap;
    for (PatInfo& pi : gr.pats_h) pi.sub_cap = cap;
    FB_CUDA(cudaMemcpy(gr.pats.p, gr.pats_h.data(), sizeof(PatInfo) * gr.P, cudaMemcpyHostToDevice));
    set_split(gr, gr.ratio);
  }

  // Patterns whose tap work N w^2 is below ratio x (tile cells of all bins)
  // take the direct kernels.
  void set_split(Group& gr, double ratio) {
    gr.ratio = ratio;
    const double tile_work = double(gr.nbins) * double(kTile2D + es_.w) * double(kTile2D + es_.w);
    std::vector<int2> tab;
    std::vector<PointItem> pit;
    for (int l = 0; l < gr.P; ++l) {
      const PatInfo& pi = gr.pats_h[l];
      const bool d = double(pi.npts) * es_.w * es_.w < ratio * tile_work;
      gr.direct[l] = d ? 1 : 0;
      if (d) {
        for (int s = 0; s < pi.npts; s += kDirectPts)
          pit.push_back(PointItem{pi.rec_base + s, std::min(kDirectPts, pi.npts - s), l, 0});
      } else {  // slots for this cap's subproblems
        const int slots = int(std::min<int64_t>(pi.max_sub, gr.nbins + ceil_div(pi.npts, gr.sub_cap)));
        for (int s = 0; s < slots; ++s) tab.push_back(make_int2(l, s));
      }
    }
    gr.n_tab = int(tab.size());
    gr.n_pitems = int(pit.size());
    if (!tab.empty()) FB_CUDA(cudaMemcpy(gr.tab.p, tab.data(), sizeof(int2) * tab.size(), cudaMemcpyHostToDevice));
    if (!pit.empty())
      FB_CUDA(cudaMemcpy(gr.pitems.p, pit.data(), sizeof(PointItem) * pit.size(), cudaMemcpyHostToDevice));
  }

  template <int W>
  void smem_attrs_w() {
    constexpr size_t ss = spread2d_smem_bytes<W, T, false>();
    constexpr size_t si = interp2d_smem_bytes<W, T>();
    ensure_dynamic_smem(spread2d_tile_kernel<W, T, false, EnsTileMap<T>>, ss);
    ensure_dynamic_smem(interp2d_tile_kernel<W, T, EnsTileMap<T>>, si);
  }
  void smem_attrs() {
#define FB_X(WW) smem_attrs_w<WW>()
    FB_ENS_W(T, FB_X)
#undef FB_X
    int most = 0;
    for (const auto& gp : groups_) most = std::max(most, gp->nbins);
    const int sb = int(sizeof(int)) * most;
    ensure_dynamic_smem(ens_sort_count_kernel<T>, size_t(sb));
    ensure_dynamic_smem(ens_sort_scatter_kernel<T>, size_t(sb));
  }

  template <int W>
  void run_group_w(Group& gr, const double* x, double* g, double* e, cudaStream_t s) {
    const Geom& geo = gr.geom;
    MapParams mp;
    mp.kind = 0;
    mp.stride = 2;
    for (int a = 0; a < 2; ++a) {
      mp.L[a] = L_[a];
      mp.scale[a] = double(geo.nf[a]) / L_[a];
      mp.invL[a] = 1.0 / L_[a];
    }
    const size_t hs = sizeof(int) * size_t(gr.nbins);
    Rec<2, T>* uns = reinterpret_cast<Rec<2, T>*>(gr.unsorted.p);
    Rec<2, T>* recs = reinterpret_cast<Rec<2, T>*>(gr.recs.p);
    ens_sort_count_kernel<T><<<gr.n_items, kEnsSortThreads, hs, s>>>(x, gr.items.p, gr.pats.p, mp, geo,
                                                                    gr.bin_total.p, gr.blk_off.p, uns, cur_status_.p,
                                                                    sticky_.p);
    FB_LAUNCH_CHECK();
    ens_sort_scatter_kernel<T><<<gr.n_items, kEnsSortThreads, hs, s>>>(
        uns, gr.items.p, gr.pats.p, geo, gr.bin_total.p, gr.blk_off.p, gr.bin_start.p, gr.sub_bin.p, gr.sub_start.p,
        gr.sub_count.p, gr.num_sub.p, gr.done.p, recs, sticky_.p);
    FB_LAUNCH_CHECK();
    if (!gr.band) FB_CUDA(cudaMemsetAsync(gr.spread.p, 0, gr.spread.bytes(), s));  // the band row pass re-zeroes
    const EsPoly<W, T> poly = make_es_poly<W, T>(poly_);
    const EnsTileMap<T> map{gr.pats.p,     gr.tab.p,       gr.sub_bin.p, gr.sub_start.p, gr.sub_count.p,
                            gr.num_sub.p, gr.bin_start.p, cur_status_.p, gr.G};
    if (gr.n_tab) {
      bool done = false;
      if constexpr (sizeof(T) == 4 && W >= 4 && W <= 8) {
        if (geo.nf[0] % 4 == 0) {  // thread per point, fixed-point shared atomics
          spread2d_tpp_kernel<W, EnsTileMap<float>><<<gr.n_tab, Tpp2D<W>::NT, spread2d_tpp_smem_bytes<W>(), s>>>(
              recs, weights_.p, map, geo, poly, gr.spread.p);
          FB_LAUNCH_CHECK();
          done = true;
        }
      }
      if (!done) {
        constexpr size_t ss = spread2d_smem_bytes<W, T, false>();
        spread2d_tile_kernel<W, T, false, EnsTileMap<T>><<<gr.n_tab, Tile2D<W>::THREADS, ss, s>>>(
            recs, weights_.p, nullptr, map, geo, poly, gr.spread.p, nullptr);
        FB_LAUNCH_CHECK();
      }
    }
    if (gr.n_pitems) {
      ens_spread_direct_kernel<W, T><<<gr.n_pitems, kDirectPts, 0, s>>>(recs, weights_.p, gr.pats.p, gr.pitems.p,
                                                                        geo, poly, gr.spread.p, gr.G);
      FB_LAUNCH_CHECK();
    }
    if (gr.band) {
      run_band(gr, g, e, s);
      if (!g) return;
    } else {
      FB_CUFFT(cufftSetStream(gr.r2c, s));
      if (sizeof(T) == 4) {
        FB_CUFFT(cufftExecR2C(gr.r2c, reinterpret_cast<cufftReal*>(gr.spread.p),
                              reinterpret_cast<cufftComplex*>(gr.bhat.p)));
      } else {
        FB_CUFFT(cufftExecD2Z(gr.r2c, reinterpret_cast<cufftDoubleReal*>(gr.spread.p),
                              reinterpret_cast<cufftDoubleComplex*>(gr.bhat.p)));
      }
      const int gx = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(gr.max_active, 256), 64)));
      ens_modes_kernel<T><<<dim3(gx, gr.P), 256, 0, s>>>(gr.pats.p, gr.mode_idx.p, gr.coef.p, gr.n, gr.K, gr.bhat.p,
                                                         gr.nh0, gr.GH, geo.nf[0], gr.corr.p, gr.hgrid.p, gr.G, e,
                                                         cur_status_.p, g != nullptr);
      FB_LAUNCH_CHECK();
      if (!g) return;
      FB_CUFFT(cufftSetStream(gr.c2c, s));
      if (sizeof(T) == 4) {
        FB_CUFFT(cufftExecC2C(gr.c2c, reinterpret_cast<cufftComplex*>(gr.hgrid.p),
                              reinterpret_cast<cufftComplex*>(gr.ggrid.p), CUFFT_FORWARD));
      } else {
        FB_CUFFT(cufftExecZ2Z(gr.c2c, reinterpret_cast<cufftDoubleComplex*>(gr.hgrid.p),
                              reinterpret_cast<cufftDoubleComplex*>(gr.ggrid.p), CUFFT_FORWARD));
      }
    }
    if (gr.n_tab) {
      constexpr size_t si = interp2d_smem_bytes<W, T>();
      interp2d_tile_kernel<W, T, EnsTileMap<T>><<<gr.n_tab, 256, si, s>>>(recs, weights_.p, map, geo, poly, gr.ggrid.p,
                                                                          INTERP_GRAD, g, nullptr, 0, GradScale());
      FB_LAUNCH_CHECK();
    }
    if (gr.n_pitems) {
      ens_interp_direct_kernel<W, T><<<gr.n_pitems, kDirectPts, 0, s>>>(recs, weights_.p, gr.pats.p, gr.pitems.p, geo,
                                                                        poly, gr.ggrid.p, gr.G, g, cur_status_.p);
      FB_LAUNCH_CHECK();
    }
  }

  void run_group(Group& gr, const double* x, double* g, double* e, cudaStream_t s) {
#define FB_X(WW) run_group_w<WW>(gr, x, g, e, s)
    FB_ENS_W(T, FB_X)
#undef FB_X
  }

  int P_ = 0;
  double L_[2] = {1, 1};
  ESParams es_;
  std::vector<double> poly_;
  DevBuf<T> weights_;
  DevBuf<int> cur_status_, sticky_;
  std::vector<std::unique_ptr<Group>> groups_;
  cudaEvent_t fork_ = nullptr;
};

}  // namespace

EnsemblePtr make_nuwu_ensemble(int n_patterns, const int64_t* n_points, const double* radii, const int64_t* n_modes,
                               const double* sk, const double* v, const double* L, int ndim, double eps,
                               int precision) {
  if (ndim != 2) throw InvalidArgument("NUwU ensembles are two-dimensional");
  if (precision == 1) return EnsemblePtr(new NUwUEnsembleImpl<float>(n_patterns, n_points, radii, n_modes, sk, v, L, eps));
  return EnsemblePtr(new NUwUEnsembleImpl<double>(n_patterns, n_points, radii, n_modes, sk, v, L, eps));
}

}  // namespace fb
