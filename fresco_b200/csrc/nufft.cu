// Precision-independent NUFFT set-up: geometry and sort buffers.
#include <algorithm>
#include <string>

#include "nufft.cuh"

namespace fb {

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

Geom make_geom(int D, const int64_t* nf, int w, const int* tile_pref) {
  if (D < 1 || D > 3) throw InvalidArgument("Invalid dimension: " + std::to_string(D));
  Geom g;
  g.D = D;
  g.w = w;
  g.pad = w / 2;
  const int64_t lim[3][3] = {{int64_t(1) << 31, 1, 1}, {65536, 65536, 1}, {2048, 2048, 1024}};
  for (int a = 0; a < 3; ++a) {
    if (a < D) {
      if (nf[a] > lim[D - 1][a]) throw InvalidArgument("fine grid too large for dimension " + std::to_string(D));
      g.nf[a] = int(nf[a]);
      g.tile[a] = std::max(1, std::min(tile_pref[a], g.nf[a]));
      g.nb[a] = int(ceil_div(g.nf[a], g.tile[a]));
      g.tw[a] = g.tile[a] + w;
    } else {
      g.nf[a] = g.tile[a] = g.nb[a] = g.tw[a] = 1;
    }
  }
  if (g.nbins() > (int64_t(1) << 30)) throw InvalidArgument("too many bins");
  return g;
}

void alloc_sort(SortBufs& sb, int64_t N, const Geom& g) {
  const int64_t nb = g.nbins();
  sb.bin_count.alloc(nb);
  sb.bin_start.alloc(nb);
  sb.max_sub = nb + ceil_div(std::max<int64_t>(N, 1), kMaxSub);
  sb.sub_bin.alloc(sb.max_sub);
  sb.sub_start.alloc(sb.max_sub);
  sb.sub_count.alloc(sb.max_sub);
  sb.num_sub.alloc(1);
  sb.rank.alloc(std::max<int64_t>(N, 1));
}

}  // namespace fb
