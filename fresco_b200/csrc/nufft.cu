// Precision-independent NUFFT set-up: geometry and sort buffers.
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "nufft.cuh"
#include "scan.cuh"

namespace fb {

int& tile_wait_polls_setting() {
  static int polls = kTileWaitPolls;
  return polls;
}

void set_tile_wait_polls(int polls) { tile_wait_polls_setting() = polls >= 0 ? polls : kTileWaitPolls; }

int sm_count() {
  static int cache[16] = {0};
  int dev = 0;
  FB_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 16 && cache[dev]) return cache[dev];
  int n = 0;
  FB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  if (dev >= 0 && dev < 16) cache[dev] = n;
  return n;
}

void ensure_dynamic_smem(const void* kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return;  // within the default limit
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> limit;
  int dev = 0;
  FB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limit[{kernel, dev}];
  if (bytes <= cur) return;
  FB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  cur = bytes;
}

Geom make_geom(int D, const int64_t* nf, int w, const int* tile_pref) {
  if (D < 1 || D > 3) throw InvalidArgument("Invalid dimension: " + std::to_string(D));
  Geom g;
  g.D = D;
  g.w = w;
  g.pad = w / 2;
  const int64_t lim[3][3] = {{int64_t(1) << 31, 1, 1}, {65536, 65536, 1}, {2048, 2048, 1024}};
  int tile[3] = {1, 1, 1};
  for (int a = 0; a < D; ++a) {
    if (nf[a] > lim[D - 1][a]) throw InvalidArgument("fine grid too large for dimension " + std::to_string(D));
    g.nf[a] = int(nf[a]);
    // 2D uses fixed 64-cell tiles (phased spreading); other dimensions clamp to the grid
    tile[a] = (D == 2) ? kTile2D : std::max(1, std::min(tile_pref[a], g.nf[a]));
  }
  for (;;) {
    int64_t nb = 1;
    for (int a = 0; a < D; ++a) nb *= ceil_div(g.nf[a], tile[a]);
    if (nb <= kMaxBins || D == 2) break;
    // grow the smallest tile edge that is still below its grid edge
    int best = -1;
    for (int a = 0; a < D; ++a)
      if (tile[a] < g.nf[a] && (best < 0 || tile[a] < tile[best])) best = a;
    if (best < 0) break;
    tile[best] = std::min(2 * tile[best], g.nf[best]);
  }
  for (int a = 0; a < 3; ++a) {
    if (a < D) {
      g.tile[a] = tile[a];
      g.nb[a] = int(ceil_div(g.nf[a], g.tile[a]));
      g.tw[a] = g.tile[a] + w;
    } else {
      g.nf[a] = g.tile[a] = g.nb[a] = g.tw[a] = 1;
    }
  }
  if (g.nbins() > kMaxBins) throw InvalidArgument("fine grid needs too many bins for the block-local sort");
  return g;
}

void alloc_sort(SortBufs& sb, int64_t N, const Geom& g) {
  const int64_t nb = g.nbins();
  const int sms = sm_count();
  sb.NB = int(std::max<int64_t>(1, std::min<int64_t>(2 * sms, ceil_div(std::max<int64_t>(N, 1), 1024))));
  sb.chunk = ceil_div(std::max<int64_t>(N, 1), sb.NB);
  sb.bin_total.alloc(nb);
  FB_CUDA(cudaMemset(sb.bin_total.p, 0, sizeof(int) * nb));
  sb.blk_off.alloc(nb * sb.NB);
  sb.bin_start.alloc(nb + 1);
  sb.max_sub = nb + ceil_div(std::max<int64_t>(N, 1), kMaxSub);
  sb.sub_bin.alloc(sb.max_sub);
  sb.sub_start.alloc(sb.max_sub);
  sb.sub_count.alloc(sb.max_sub);
  sb.num_sub.alloc(1);
  sb.unsorted.alloc(std::max<int64_t>(N, 1) * 32);  // the largest record is 32 bytes
  sb.done.alloc(1);
  FB_CUDA(cudaMemset(sb.done.p, 0, sizeof(unsigned)));
  sb.bar.alloc(1);
  FB_CUDA(cudaMemset(sb.bar.p, 0, sizeof(unsigned long long)));
}

}  // namespace fb
