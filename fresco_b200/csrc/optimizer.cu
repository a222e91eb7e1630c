// Device-resident LBFGS and modified FIRE (see optimizer.cuh).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <vector>

#include "optimizer.cuh"

namespace fb {

namespace {

constexpr int kThreads = 512;  // streaming kernels: more loads in flight per block

// Sum of P block partials, the same value on every thread (fixed order).
__device__ double sum_parts(const double* __restrict__ part, int P) {
  __shared__ double sh[32];
  __shared__ double result;
  double v = 0.0;
  for (int i = threadIdx.x; i < P; i += blockDim.x) v += part[i];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    s = warp_sum(s);
    if (threadIdx.x == 0) result = s;
  }
  __syncthreads();
  const double r = result;
  __syncthreads();
  return r;
}

// Writes the block sums of v[0..K-1] to part[slot[k] * P + blockIdx.x].
template <int K>
__device__ void block_partials(double (&v)[K], double* part, int P, const int (&slot)[K]) {
  __shared__ double red[K][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double s = warp_sum(v[k]);
    if (lane == 0) red[k][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = lane < nw ? red[k][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) part[int64_t(slot[k]) * P + blockIdx.x] = s;
    }
  }
  __syncthreads();
}

#define GRID_LOOP(i, n) \
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

// ---------------------------------------------------------------------------
// shared kernels
// ---------------------------------------------------------------------------

__global__ void dot_kernel(const double* __restrict__ a, const double* __restrict__ b, int64_t n, double* part, int P,
                           int slot) {
  double v[1] = {0.0};
  GRID_LOOP(i, n) v[0] += a[i] * b[i];
  const int sl[1] = {slot};
  block_partials<1>(v, part, P, sl);
}

// ---------------------------------------------------------------------------
// LBFGS (source/lbfgs.cpp)
// ---------------------------------------------------------------------------

struct LbState {
  double f, fnew, rms, H0, stepnorm, factor;
  double inv_sqrt_n, maxstep, max_f_rise;
  int k, nred, accepted, rel, M;
  int fault;  // a grid barrier of the fused direction kernel gave up (the iteration is void)
};

enum LbSlot { S_IN = 0, S_OUT = 1, S_SG = 2, S_SS = 3, S_GG = 4, S_YS = 5, S_YY = 6, S_TMP = 7, S_NSLOT = 8 };

// k == 0 (lbfgs.cpp:109-124): step = -H0 * gn * g with gn = 1/|g| if |g| > 1 else |g|.
__global__ void lb_first_step(const double* __restrict__ g, double* __restrict__ step, int64_t n, LbState* st,
                              double* part, int P) {
  double gnorm = sqrt(sum_parts(part + int64_t(S_GG) * P, P));
  if (gnorm > 1.0) gnorm = 1.0 / gnorm;
  const double pref = -gnorm * st->H0;
  double v[2] = {0.0, 0.0};
  GRID_LOOP(i, n) {
    const double s = pref * g[i];
    step[i] = s;
    v[0] += s * g[i];
    v[1] += s * s;
  }
  const int sl[2] = {S_SG, S_SS};
  block_partials<2>(v, part, P, sl);
}

// step = g and the first backward dot s_i . g.
__global__ void lb_start(const double* __restrict__ g, double* __restrict__ step, const double* __restrict__ s_i,
                         int64_t n, double* part, int P) {
  double v[1] = {0.0};
  GRID_LOOP(i, n) {
    const double gi = g[i];
    step[i] = gi;
    v[0] += s_i[i] * gi;
  }
  const int sl[1] = {S_IN};
  block_partials<1>(v, part, P, sl);
}

// One two-loop update (lbfgs.cpp:136-169).
//  backward: a = rho_i (s_i . step); step -= a y_i; [last: step *= -H0]
//  forward : b = -rho_i (y_i . step); step -= (alpha_i - b) s_i
// followed by the next dot product (dnext . step), or for the final forward
// update the line-search dots (step . g, step . step).
// The incoming dot product is in slot in_slot, the next one goes to out_slot
// (the two alternate between consecutive updates).
__global__ void lb_update(int forward, int last, double* __restrict__ step, const double* __restrict__ vec,
                          const double* __restrict__ dnext, const double* __restrict__ g, int64_t n, LbState* st,
                          double* rho, double* alpha, int mi, double* part, int P, int in_slot, int out_slot) {
  const double dotin = sum_parts(part + int64_t(in_slot) * P, P);
  double coef;
  if (!forward) {
    coef = rho[mi] * dotin;
    if (blockIdx.x == 0 && threadIdx.x == 0) alpha[mi] = coef;
  } else {
    const double beta = -rho[mi] * dotin;
    coef = alpha[mi] - beta;
  }
  const double h0 = -st->H0;
  const bool scale = !forward && last;
  const bool ls = forward && last;
  double v[2] = {0.0, 0.0};
  GRID_LOOP(i, n) {
    double s = step[i] - coef * vec[i];
    if (scale) s *= h0;
    step[i] = s;
    if (ls) {
      v[0] += s * g[i];
      v[1] += s * s;
    } else {
      v[0] += dnext[i] * s;
    }
  }
  if (ls) {
    const int sl[2] = {S_SG, S_SS};
    block_partials<2>(v, part, P, sl);
  } else {
    double w[1] = {v[0]};
    const int sl[1] = {out_slot};
    block_partials<1>(w, part, P, sl);
  }
}

// The whole two-loop recursion of an iteration with stored pairs (k > 0,
// lbfgs.cpp:126-169) in one cooperative launch.  Block b keeps its slice
// [b chunk, (b + 1) chunk) of the step in shared memory from the copy of g
// to the final scaling, so the step is neither re-read nor re-written
// between the updates; each memory vector is read once in each loop.  Every
// dot product is the sum of the blocks' partials, taken after a grid barrier
// in block order, so all blocks use the same coefficient; the element-wise
// updates are those of lb_start / lb_update.  At the end the step goes to
// HBM and the line-search dots step.g, step.step are left in their slots,
// padded with zeros to the P partials that lb_trial sums.  A barrier that
// gives up sets st->fault.
constexpr int kDirThreads = 1024;

__global__ void __launch_bounds__(kDirThreads, 1) lb_direction_kernel(
    const double* __restrict__ g, const double* __restrict__ sm, const double* __restrict__ ym, int64_t n,
    int64_t chunk, int k, int M, LbState* st, const double* __restrict__ rho, double* alpha, double* part, int P,
    unsigned long long* bar, double* __restrict__ step) {
  extern __shared__ __align__(16) double q[];  // this block's slice of the step
  __shared__ double alph[64];                   // alpha_i of the backward loop (M <= 64)
  const int B = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
  const int64_t e0 = int64_t(b) * chunk, e1 = min(n, e0 + chunk);
  const int cnt = e1 > e0 ? int(e1 - e0) : 0;
  const int jmin = max(0, k - M), jmax = k, m = jmax - jmin;
  bool ok = true;
  // the sum over the blocks of slot `slot` (fixed order; same value in every block)
  auto total = [&](int slot) { return sum_parts(part + int64_t(slot) * P, B); };
  auto partial = [&](double v, int slot) {
    double w[1] = {v};
    const int sl[1] = {slot};
    block_partials<1>(w, part, P, sl);
  };
  // lb_start: step = g, first backward dot s_i0 . g
  {
    const double* s0 = sm + int64_t((jmax - 1) % M) * n + e0;
    double v = 0.0;
    for (int i = tid; i < cnt; i += blockDim.x) {
      const double gi = g[e0 + i];
      q[i] = gi;
      v += s0[i] * gi;
    }
    partial(v, S_IN);
  }
  ok &= grid_barrier(bar, B);
  int in_slot = S_IN, out_slot = S_OUT;
  for (int t = 0; t < m; ++t) {  // backward loop, newest pair first
    const int j = jmax - 1 - t, mi = j % M;
    const bool last = t == m - 1;
    const double coef = rho[mi] * total(in_slot);
    if (tid == 0) alph[t] = coef;
    if (b == 0 && tid == 0) alpha[mi] = coef;
    const double* y = ym + int64_t(mi) * n + e0;
    const double* dn = (last ? ym + int64_t(jmin % M) * n : sm + int64_t((j - 1) % M) * n) + e0;
    const double h0 = -st->H0;
    double v = 0.0;
    for (int i = tid; i < cnt; i += blockDim.x) {
      double sv = q[i] - coef * y[i];
      if (last) sv *= h0;
      q[i] = sv;
      v += dn[i] * sv;
    }
    partial(v, out_slot);
    ok &= grid_barrier(bar, B);
    const int tmp = in_slot;
    in_slot = out_slot;
    out_slot = tmp;
  }
  __syncthreads();
  for (int t = 0; t < m; ++t) {  // forward loop, oldest pair first
    const int j = jmin + t, mi = j % M;
    const bool last = t == m - 1;
    const double beta = -rho[mi] * total(in_slot);
    const double coef = alph[m - 1 - t] - beta;
    const double* sv_ = sm + int64_t(mi) * n + e0;
    if (!last) {
      const double* dn = ym + int64_t((j + 1) % M) * n + e0;
      double v = 0.0;
      for (int i = tid; i < cnt; i += blockDim.x) {
        const double sv = q[i] - coef * sv_[i];
        q[i] = sv;
        v += dn[i] * sv;
      }
      partial(v, out_slot);
      ok &= grid_barrier(bar, B);
      const int tmp = in_slot;
      in_slot = out_slot;
      out_slot = tmp;
    } else {
      double v[2] = {0.0, 0.0};
      for (int i = tid; i < cnt; i += blockDim.x) {
        const double sv = q[i] - coef * sv_[i];
        step[e0 + i] = sv;
        v[0] += sv * g[e0 + i];
        v[1] += sv * sv;
      }
      const int sl[2] = {S_SG, S_SS};
      block_partials<2>(v, part, P, sl);
    }
  }
  // lb_trial sums P partials: the slots of the blocks this launch does not have are zero
  if (b == 0)
    for (int i = B + tid; i < P; i += blockDim.x) {
      part[int64_t(S_SG) * P + i] = 0.0;
      part[int64_t(S_SS) * P + i] = 0.0;
    }
  if (!ok && tid == 0) st->fault = 1;
}

// Trial point of the backtracking line search (lbfgs.cpp:176-204).
__global__ void lb_trial(const double* __restrict__ xold, const double* __restrict__ step, double* __restrict__ xnew,
                         int64_t n, LbState* st, double* part, int P) {
  const double dsg = sum_parts(part + int64_t(S_SG) * P, P);
  const double ss = sum_parts(part + int64_t(S_SS) * P, P);
  const double sgn = dsg > 0.0 ? -1.0 : 1.0;
  const double stepnorm = sqrt(ss);
  double factor = 1.0;
  if (factor * stepnorm > st->maxstep) factor = st->maxstep / stepnorm;
  for (int r = 0; r < st->nred; ++r) factor *= 0.5;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->stepnorm = stepnorm;
    st->factor = factor;
  }
  GRID_LOOP(i, n) xnew[i] = xold[i] + factor * (sgn * step[i]);
}

// s = xnew - xold, y = gnew - gold into memory slot; |g|^2, y.s, y.y (lbfgs.cpp:74-84).
__global__ void lb_post(const double* __restrict__ xnew, const double* __restrict__ xold,
                        const double* __restrict__ gnew, const double* __restrict__ gold, double* __restrict__ s_k,
                        double* __restrict__ y_k, int64_t n, double* part, int P) {
  double v[3] = {0.0, 0.0, 0.0};
  GRID_LOOP(i, n) {
    const double gi = gnew[i];
    const double yi = gi - gold[i];
    const double si = xnew[i] - xold[i];
    y_k[i] = yi;
    s_k[i] = si;
    v[0] += gi * gi;
    v[1] += yi * si;
    v[2] += yi * yi;
  }
  const int sl[3] = {S_GG, S_YS, S_YY};
  block_partials<3>(v, part, P, sl);
}

// Accept test and memory update (lbfgs.cpp:206-245, 86-104).  One block.
// out: [accepted, f, rms, H0, printed step norm, fnew]
__global__ void lb_finalize(LbState* st, const double* __restrict__ fnew_dev, double* rho, int kl, double* part, int P,
                            double* out) {
  const double gg = sum_parts(part + int64_t(S_GG) * P, P);
  double ys = sum_parts(part + int64_t(S_YS) * P, P);
  double yy = sum_parts(part + int64_t(S_YY) * P, P);
  if (threadIdx.x != 0) return;
  const double fnew = *fnew_dev;
  double df = fnew - st->f;
  if (st->rel) {
    double absf = 1e-100;
    if (st->f != 0) absf = fabs(st->f);
    df /= absf;
  }
  const bool ok = df < st->max_f_rise;
  const bool accept = ok || st->nred >= 9;
  double printed = st->stepnorm * st->factor;
  if (!ok) printed *= 0.5;
  st->fnew = fnew;
  if (accept) {
    st->f = fnew;
    st->rms = sqrt(gg) * st->inv_sqrt_n;
    if (ys == 0.0) ys = 1.0;
    rho[kl] = 1.0 / ys;
    if (yy == 0.0) yy = 1.0;
    st->H0 = ys / yy;
    st->k += 1;
    st->nred = 0;
    st->accepted = 1;
  } else {
    st->nred += 1;
    st->accepted = 0;
  }
  out[0] = accept ? 1.0 : 0.0;
  out[1] = st->f;
  out[2] = st->rms;
  out[3] = st->H0;
  out[4] = printed;
  out[5] = fnew;
  out[6] = st->fault;
}

// Initial f, rms (optimizer.hpp:203-210: rms = sqrt(|g|^2 / n)).
__global__ void lb_init_fin(LbState* st, const double* __restrict__ e, double inv_n, double* part, int P, double* out) {
  const double gg = sum_parts(part + int64_t(S_GG) * P, P);
  if (threadIdx.x != 0) return;
  st->f = *e;
  st->rms = sqrt(gg * inv_n);
  out[1] = st->f;
  out[2] = st->rms;
  out[3] = st->H0;
}

__global__ void lb_set_h0(LbState* st, double h0) { st->H0 = h0; }

__global__ void lb_set_scalars(LbState* st, double f, double rms, int reset_k, int set_h0, double h0) {
  st->f = f;
  st->rms = rms;
  if (reset_k) {
    st->k = 0;
    st->nred = 0;
  }
  if (set_h0) st->H0 = h0;
}

// ---------------------------------------------------------------------------
// FIRE (source/fresco/modified_fire.hpp)
// ---------------------------------------------------------------------------

struct FiState {
  double f, dt, a, ifnorm, vnorm, rms, P, sqrtN;
  double dtmax, maxstep, finc, fdec, fa, astart;
  int fire_iter, Nmin, stepback, restore;
  // graph-captured loop only (FireGraph): the loop state on the device; cur is
  // the buffer parity holding the current point, guard bounds the loop
  double tol;
  int active, iter, stop_iter, nfev, cur, guard, guard_limit;
};

enum FiSlot { F_DD = 0, F_PV = 1, F_GG = 2, F_VV = 3, F_NSLOT = 4 };

// v = -g dt and the norms (modified_fire.cpp:313-324).
__global__ void fi_init_v(const double* __restrict__ g, double* __restrict__ v, int64_t n, FiState* st, double* part,
                          int P) {
  const double dt = st->dt;
  double acc[2] = {0.0, 0.0};
  GRID_LOOP(i, n) {
    const double vi = -g[i] * dt;
    v[i] = vi;
    acc[0] += g[i] * g[i];
    acc[1] += vi * vi;
  }
  const int sl[2] = {F_GG, F_VV};
  block_partials<2>(acc, part, P, sl);
}

__global__ void fi_init_fin(FiState* st, const double* __restrict__ e, double* part, int P, double* out) {
  const double gg = sum_parts(part + int64_t(F_GG) * P, P);
  const double vv = sum_parts(part + int64_t(F_VV) * P, P);
  if (threadIdx.x != 0) return;
  st->f = *e;
  st->ifnorm = 1.0 / sqrt(gg);
  st->vnorm = sqrt(vv);
  st->rms = 1.0 / (st->ifnorm * st->sqrtN);
  out[0] = st->f;
  out[1] = st->rms;
  out[2] = st->dt;
  out[3] = st->a;
  out[4] = 0.0;
  out[5] = st->vnorm;
  out[6] = double(st->fire_iter);
}

// Inertial mixing and the forward-Euler velocity update (modified_fire.hpp:172-174, 141-144).
// GRAPH: part of a captured iteration, a no-op once the loop has stopped.
template <bool GRAPH>
__global__ void fi_mix(double* __restrict__ v, const double* __restrict__ g, int64_t n, FiState* st, double* part,
                       int P) {
  if (GRAPH && !st->active) return;  // uniform over the grid
  const double a = st->a, ifn = st->ifnorm, vn = st->vnorm, dt = st->dt;
  double acc[1] = {0.0};
  GRID_LOOP(i, n) {
    double vi = (1.0 - a) * v[i] - a * g[i] * ifn * vn;
    vi -= dt * g[i];
    v[i] = vi;
    const double dx = dt * vi;
    acc[0] += dx * dx;
  }
  const int sl[1] = {F_DD};
  block_partials<1>(acc, part, P, sl);
}

// x_new = x + dx * factor (modified_fire.hpp:146-155), written to the other
// coordinate buffer: x and its gradient stay where they are for a step back.
__global__ void fi_step(const double* __restrict__ x, double* __restrict__ xnew, const double* __restrict__ v,
                        int64_t n, FiState* st, double* part, int P) {
  const double normdx = sqrt(sum_parts(part + int64_t(F_DD) * P, P));
  double factor = 1.0;
  if (normdx > st->maxstep) factor = st->maxstep / normdx;
  const double dt = st->dt;
  GRID_LOOP(i, n) {
    const double dx = dt * v[i];
    xnew[i] = x[i] + dx * factor;
  }
}

template <bool GRAPH>
__global__ void fi_post(const double* __restrict__ v, const double* __restrict__ g, int64_t n, double* part, int P,
                        const FiState* st) {
  if (GRAPH && !st->active) return;
  double acc[3] = {0.0, 0.0, 0.0};
  GRID_LOOP(i, n) {
    acc[0] += v[i] * g[i];
    acc[1] += g[i] * g[i];
    acc[2] += v[i] * v[i];
  }
  const int sl[3] = {F_PV, F_GG, F_VV};
  block_partials<3>(acc, part, P, sl);
}

// modified_fire.hpp:180-216.  out: [f, rms, dt, a, P, vnorm, fire_iter]
// GRAPH: also the loop bookkeeping of GradientOptimizer::run (optimizer.hpp:
// 97-112): evaluation and iteration counts, and whether to continue.
template <bool GRAPH>
__global__ void fi_fin(FiState* st, const double* __restrict__ e, double* part, int P, double* out) {
  if (GRAPH && !st->active) {
    if (threadIdx.x == 0) st->restore = 0;
    return;
  }
  const double pv = sum_parts(part + int64_t(F_PV) * P, P);
  const double gg = sum_parts(part + int64_t(F_GG) * P, P);
  const double vv = sum_parts(part + int64_t(F_VV) * P, P);
  if (threadIdx.x != 0) return;
  st->fire_iter += 1;
  const double Pw = -pv;
  st->P = Pw;
  if (Pw > 0) {
    if (st->fire_iter > st->Nmin) {
      st->dt = fmin(st->dt * st->finc, st->dtmax);
      st->a *= st->fa;
    }
    st->ifnorm = 1.0 / sqrt(gg);
    st->vnorm = sqrt(vv);
    st->rms = 1.0 / (st->ifnorm * st->sqrtN);
    st->f = *e;
    st->restore = 0;
  } else {
    st->dt *= st->fdec;
    st->a = st->astart;
    st->fire_iter = 0;
    st->restore = 1;
    if (!st->stepback) st->f = *e;
  }
  if (GRAPH) {
    st->nfev += 1;
    st->iter += 1;
    st->active = !(st->rms <= st->tol) && (st->iter < st->stop_iter);
    if (Pw > 0 || !st->stepback) st->cur = 1 - st->cur;  // the trial point becomes current
  }
  out[0] = st->f;
  out[1] = st->rms;
  out[2] = st->dt;
  out[3] = st->a;
  out[4] = Pw;
  out[5] = st->vnorm;
  out[6] = double(st->fire_iter);
}

// run(niter) of the captured loop: niter more iterations while rms > tol (or
// exactly one with force, as one_iteration); the loop ends after niter + 2
// passes of its body whatever the state says.
__global__ void fi_set_stop(FiState* st, int niter, int iter, int nfev, int force) {
  st->iter = iter;
  st->nfev = nfev;
  st->stop_iter = iter + niter;
  st->active = (force || !(st->rms <= st->tol)) && (iter < st->stop_iter);
  st->guard = 0;
  st->guard_limit = niter + 2;
}

// End of a loop body pass: the next pass's switch value (the iteration from
// buffer parity cur, or none, 2, once stopped) and whether to continue, at
// most guard_limit passes.  The first pass of a launch runs no iteration (the
// switch starts at its default, 2) and only sets the value.
__global__ void fi_loop(FiState* st, cudaGraphConditionalHandle h_while, cudaGraphConditionalHandle h_switch) {
  st->guard += 1;
  const bool go = st->active && st->guard < st->guard_limit;
  cudaGraphSetConditional(h_switch, go ? unsigned(st->cur & 1) : 2u);
  cudaGraphSetConditional(h_while, go ? 1u : 0u);
}

// P <= 0: v = 0 (modified_fire.hpp:204-212); the step back to x_old, g_old
// is the host keeping the previous coordinate and gradient buffers.
__global__ void fi_restore(double* __restrict__ v, int64_t n, const FiState* st) {
  if (!st->restore) return;
  GRID_LOOP(i, n) v[i] = 0.0;
}

// ---------------------------------------------------------------------------
// host classes
// ---------------------------------------------------------------------------

// A loaded FIRE state keeps the loading optimiser's parameters.
void fire_keep_params(FiState& h, const FireParams& p, int64_t n) {
  h.sqrtN = std::sqrt(double(n));
  h.dtmax = p.dtmax;
  h.maxstep = p.maxstep;
  h.finc = p.finc;
  h.fdec = p.fdec;
  h.fa = p.fa;
  h.astart = p.astart;
  h.Nmin = p.Nmin;
  h.stepback = p.stepback ? 1 : 0;
  h.tol = p.tol;
}

class Lbfgs final : public Optimizer {
 public:
  Lbfgs(PotentialPtr pot, const double* x0, int64_t n, const LbfgsParams& p)
      : Optimizer(pot, n, p.tol, p.maxiter, p.iprint, p.verbosity), prm_(p) {
    if (p.M < 1) throw InvalidArgument("LBFGS memory M must be >= 1");
    const int64_t nn = std::max<int64_t>(n, 1);
    for (int b = 0; b < 2; ++b) {
      X_[b].alloc(nn);
      G_[b].alloc(nn);
    }
    step_.alloc(nn);
    sm_.alloc(nn * p.M);
    ym_.alloc(nn * p.M);
    rho_.alloc(p.M);
    alpha_.alloc(p.M);
    e_.alloc(1);
    st_.alloc(1);
    part_.alloc(int64_t(S_NSLOT) * P_);
    FB_CUDA(cudaMemsetAsync(rho_.p, 0, rho_.bytes(), s_));
    FB_CUDA(cudaMemsetAsync(alpha_.p, 0, alpha_.bytes(), s_));
    FB_CUDA(cudaMemsetAsync(part_.p, 0, part_.bytes(), s_));
    LbState h{};
    h.f = 0.0;
    h.rms = 1e10;
    h.H0 = p.H0;
    h.inv_sqrt_n = 1.0 / std::sqrt(double(n));
    h.maxstep = p.maxstep;
    h.max_f_rise = p.max_f_rise;
    h.rel = p.rel_energy ? 1 : 0;
    h.M = p.M;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    if (n > 0) FB_CUDA(cudaMemcpyAsync(X_[0].p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    h0_ = p.H0;
  }

  double* device_x() override { return X_[cur_].p; }
  double* device_g() override { return G_[cur_].p; }
  double h0() const override { return h0_; }

  // lbfgs.hpp:70-76: allowed at any time; after the first iteration with the
  // reference's warning.  The next step's scale is H0 until the next memory
  // update replaces it with y.s / y.y (lbfgs.cpp:101).
  void set_H0(double H0) override {
    if (iter_ > 0) std::printf("warning: setting H0 after the first iteration.\n");
    lb_set_h0<<<1, 1, 0, s_>>>(st_.p, H0);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaStreamSynchronize(s_));
    h0_ = H0;
  }

  void set_reducer(ReduceFn fn, void* ctx, int64_t global_ndof) override {
    if (global_ndof < n_) throw InvalidArgument("the global coordinate count is below this process's");
    if (iter_ > 0 || func_initialized_) throw InvalidArgument("set the reducer before the first evaluation");
    reducer_ = fn;
    reducer_ctx_ = ctx;
    global_n_ = global_ndof;
    LbState h{};
    FB_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(h), cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    h.inv_sqrt_n = 1.0 / std::sqrt(double(global_ndof));
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
  }

  void set_func_gradient(double f, const double* grad, int64_t n) override {
    if (n != n_) throw InvalidArgument("the gradient has the wrong size");
    if (reducer_) throw InvalidArgument("set_func_gradient is not supported over a sharded pattern");
    if (iter_ > 0) std::printf("warning: setting f and grad after the first iteration.  this is dangerous.\n");
    double gnorm = 0.0;
    for (int64_t i = 0; i < n; ++i) gnorm += grad[i] * grad[i];
    f_ = f;
    rms_ = std::sqrt(gnorm / double(n));
    FB_CUDA(cudaMemcpyAsync(G_[cur_].p, grad, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    lb_set_scalars<<<1, 1, 0, s_>>>(st_.p, f_, rms_, 0, 0, 0.0);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaStreamSynchronize(s_));
    func_initialized_ = true;
  }

  void reset(const double* x0, int64_t n) override {
    if (n != n_)
      throw InvalidArgument("The number of degrees of freedom (x0.size()) cannot change when calling reset()");
    k_ = 0;
    iter_ = 0;
    nfev_ = 0;
    FB_CUDA(cudaMemcpyAsync(X_[cur_].p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    lb_set_scalars<<<1, 1, 0, s_>>>(st_.p, f_, rms_, 1, 0, 0.0);
    FB_LAUNCH_CHECK();
    initialize_func_gradient();
  }

  void one_iteration() override {
    if (!func_initialized_) initialize_func_gradient();
    const int c = cur_, o = 1 - cur_;
    const double* g = G_[c].p;
    const int M = prm_.M;
    // compute_lbfgs_step (lbfgs.cpp:107-170)
    if (k_ == 0) {
      dot_kernel<<<P_, kThreads, 0, s_>>>(g, g, n_, part_.p, P_, S_GG);
      reduce(S_GG, 1);
      lb_first_step<<<P_, kThreads, 0, s_>>>(g, step_.p, n_, st_.p, part_.p, P_);
      reduce(S_SG, 2);
    } else if (!reducer_ && direction_setup()) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(unsigned(dir_blocks_));
      cfg.blockDim = dim3(kDirThreads);
      cfg.dynamicSmemBytes = size_t(dir_chunk_) * sizeof(double);
      cfg.stream = s_;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeCooperative;
      attr[0].val.cooperative = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      FB_CUDA(cudaLaunchKernelEx(&cfg, lb_direction_kernel, static_cast<const double*>(g),
                                 static_cast<const double*>(sm_.p), static_cast<const double*>(ym_.p), n_,
                                 dir_chunk_, k_, M, st_.p, static_cast<const double*>(rho_.p), alpha_.p, part_.p, P_,
                                 bar_.p, step_.p));
    } else {
      const int jmin = std::max(0, k_ - M), jmax = k_;
      const int m = jmax - jmin;
      int i0 = (jmax - 1) % M;
      lb_start<<<P_, kThreads, 0, s_>>>(g, step_.p, sm_.p + int64_t(i0) * n_, n_, part_.p, P_);
      reduce(S_IN, 1);
      for (int t = 0; t < m; ++t) {
        const int j = jmax - 1 - t;
        const int i = j % M;
        const bool last = (t == m - 1);
        const int inext = last ? (jmin % M) : ((j - 1) % M);
        const double* dnext = last ? ym_.p + int64_t(inext) * n_ : sm_.p + int64_t(inext) * n_;
        lb_update<<<P_, kThreads, 0, s_>>>(0, last, step_.p, ym_.p + int64_t(i) * n_, dnext, g, n_, st_.p, rho_.p,
                                           alpha_.p, i, part_.p, P_, t % 2 ? S_OUT : S_IN, t % 2 ? S_IN : S_OUT);
        reduce(t % 2 ? S_IN : S_OUT, 1);
      }
      for (int t = 0; t < m; ++t) {
        const int j = jmin + t;
        const int i = j % M;
        const bool last = (t == m - 1);
        const int inext = (j + 1) % M;
        const double* dnext = last ? nullptr : ym_.p + int64_t(inext) * n_;
        const int u = m + t;  // update index over both loops
        lb_update<<<P_, kThreads, 0, s_>>>(1, last, step_.p, sm_.p + int64_t(i) * n_, dnext, g, n_, st_.p, rho_.p,
                                           alpha_.p, i, part_.p, P_, u % 2 ? S_OUT : S_IN, u % 2 ? S_IN : S_OUT);
        if (last) reduce(S_SG, 2);  // the line-search dots
        else reduce(u % 2 ? S_IN : S_OUT, 1);
      }
    }
    FB_LAUNCH_CHECK();
    // backtracking_linesearch (lbfgs.cpp:172-245) + update_memory (:66-105)
    const int kl = k_ % M;
    double printed = 0.0;
    for (int nred = 0; nred < 10; ++nred) {
      lb_trial<<<P_, kThreads, 0, s_>>>(X_[c].p, step_.p, X_[o].p, n_, st_.p, part_.p, P_);
      FB_LAUNCH_CHECK();
      ++nfev_;
      eval(X_[o].p, G_[o].p, e_.p);
      lb_post<<<P_, kThreads, 0, s_>>>(X_[o].p, X_[c].p, G_[o].p, G_[c].p, sm_.p + int64_t(kl) * n_,
                                       ym_.p + int64_t(kl) * n_, n_, part_.p, P_);
      reduce(S_GG, 3);
      lb_finalize<<<1, 256, 0, s_>>>(st_.p, e_.p, rho_.p, kl, part_.p, P_, host_);
      FB_LAUNCH_CHECK();
      FB_CUDA(cudaStreamSynchronize(s_));
      if (host_[6] != 0.0) throw std::runtime_error("LBFGS: a grid barrier of the direction kernel timed out");
      if (verbosity_ > 2 && host_[0] == 0.0) {
        std::printf("energy increased by %.17g to %.17g from %.17g\n", host_[5] - f_, host_[5], f_);
      }
      if (host_[0] != 0.0) {
        printed = host_[4];
        if (nred == 9 && verbosity_ > 0 && !(host_[5] - f_ < prm_.max_f_rise))
          std::printf("warning: the line search backtracked too many times\n");
        break;
      }
    }
    cur_ = o;
    f_ = host_[1];
    rms_ = host_[2];
    h0_ = host_[3];
    k_ += 1;
    if (iprint_ > 0 && iter_ % iprint_ == 0) {
      std::printf("lbgs: %d E %.17g rms %.17g nfev %d step norm %.17g\n", iter_, f_, rms_, nfev_, printed);
      std::fflush(stdout);
    }
    iter_ += 1;
  }

 private:
  void initialize_func_gradient() override {
    ++nfev_;
    eval(X_[cur_].p, G_[cur_].p, e_.p);
    dot_kernel<<<P_, kThreads, 0, s_>>>(G_[cur_].p, G_[cur_].p, n_, part_.p, P_, S_GG);
    reduce(S_GG, 1);
    lb_init_fin<<<1, 256, 0, s_>>>(st_.p, e_.p, 1.0 / double(global_n_), part_.p, P_, host_);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaStreamSynchronize(s_));
    f_ = host_[1];
    rms_ = host_[2];
    func_initialized_ = true;
  }

  int family() const override { return 1; }
  int memory_length() const override { return prm_.M; }
  std::vector<Block> image_blocks() override {
    const int64_t n = n_, M = prm_.M;
    return {{st_.p, int64_t(sizeof(LbState))},
            {X_[cur_].p, n * 8},
            {G_[cur_].p, n * 8},
            {sm_.p, M * n * 8},
            {ym_.p, M * n * 8},
            {rho_.p, M * 8},
            {e_.p, 8}};
  }
  // the loaded state keeps this optimiser's parameters
  void after_load() override {
    LbState h{};
    FB_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(h), cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    h.inv_sqrt_n = 1.0 / std::sqrt(double(global_n_));
    h.maxstep = prm_.maxstep;
    h.max_f_rise = prm_.max_f_rise;
    h.rel = prm_.rel_energy ? 1 : 0;
    h.M = prm_.M;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    k_ = h.k;
    h0_ = h.H0;
  }

  // sums `count` partial-sum slots over the processes of a sharded pattern
  void reduce(int slot, int count) {
    if (!reducer_) return;
    FB_LAUNCH_CHECK();
    reducer_(part_.p + int64_t(slot) * P_, int64_t(count) * P_, s_, reducer_ctx_);
  }

  // Whether the fused direction kernel can run: a cooperative launch of at
  // most one 1024-thread block per SM (and no more than the P partial slots)
  // whose slice of the step fits in shared memory (config 2's 2^21
  // coordinates over 148 SMs: 14,170 doubles, 113 KB per block).
  bool direction_setup() {
    if (dir_blocks_ >= 0) return dir_blocks_ > 0;
    dir_blocks_ = 0;
    if (prm_.M > 64) return false;
    int dev = 0, coop = 0, smem_max = 0;
    FB_CUDA(cudaGetDevice(&dev));
    FB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    FB_CUDA(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (!coop) return false;
    const int blocks = int(std::min<int64_t>({int64_t(sm_count()), int64_t(P_), ceil_div(n_, kDirThreads)}));
    const int64_t chunk = ceil_div(n_, blocks);
    const size_t smem = size_t(chunk) * sizeof(double);
    if (smem + 2048 > size_t(smem_max)) return false;
    ensure_dynamic_smem(lb_direction_kernel, smem);
    int occ = 0;
    FB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, lb_direction_kernel, kDirThreads, smem));
    if (occ < 1 || blocks > occ * sm_count()) return false;
    bar_.alloc(1);
    FB_CUDA(cudaMemset(bar_.p, 0, sizeof(unsigned long long)));
    dir_blocks_ = blocks;
    dir_chunk_ = chunk;
    return true;
  }

  LbfgsParams prm_;
  DevBuf<double> X_[2], G_[2], step_, sm_, ym_, rho_, alpha_, e_;
  DevBuf<LbState> st_;
  DevBuf<unsigned long long> bar_;  // grid-barrier arrivals of the direction kernel
  int dir_blocks_ = -1;             // blocks of the direction kernel (0: the per-update kernels are used)
  int64_t dir_chunk_ = 0;
  int cur_ = 0;
  int k_ = 0;
  double h0_ = 0.1;
  ReduceFn reducer_ = nullptr;
  void* reducer_ctx_ = nullptr;
  int64_t global_n_ = n_;
};

class Fire final : public Optimizer {
 public:
  Fire(PotentialPtr pot, const double* x0, int64_t n, const FireParams& p)
      : Optimizer(pot, n, p.tol, p.maxiter, p.iprint, p.verbosity), prm_(p) {
    const int64_t nn = std::max<int64_t>(n, 1);
    for (int b = 0; b < 2; ++b) {
      X_[b].alloc(nn);
      G_[b].alloc(nn);
      FB_CUDA(cudaMemsetAsync(G_[b].p, 0, G_[b].bytes(), s_));
    }
    V_.alloc(nn);
    e_.alloc(1);
    st_.alloc(1);
    part_.alloc(int64_t(F_NSLOT) * P_);
    FB_CUDA(cudaMemsetAsync(V_.p, 0, V_.bytes(), s_));
    FB_CUDA(cudaMemsetAsync(part_.p, 0, part_.bytes(), s_));
    FiState h{};
    h.f = 0.0;
    h.dt = p.dtstart;
    h.a = p.astart;
    h.rms = 1e10;
    h.sqrtN = std::sqrt(double(n));
    h.dtmax = p.dtmax;
    h.maxstep = p.maxstep;
    h.finc = p.finc;
    h.fdec = p.fdec;
    h.fa = p.fa;
    h.astart = p.astart;
    h.Nmin = p.Nmin;
    h.stepback = p.stepback ? 1 : 0;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    if (n > 0) FB_CUDA(cudaMemcpyAsync(X_[0].p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
  }

  double* device_x() override { return X_[cur_].p; }
  double* device_g() override { return G_[cur_].p; }

  void set_func_gradient(double f, const double* grad, int64_t n) override {
    if (n != n_) throw InvalidArgument("the gradient has the wrong size");
    if (iter_ > 0) std::printf("warning: setting f and grad after the first iteration.  this is dangerous.\n");
    FB_CUDA(cudaMemcpyAsync(G_[cur_].p, grad, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaMemcpyAsync(e_.p, &f, sizeof(double), cudaMemcpyHostToDevice, s_));
    init_from_gradient();
  }

  void reset(const double* x0, int64_t n) override {
    if (n != n_) throw InvalidArgument("The number of degrees of freedom (x0.size()) cannot change when calling reset()");
    if (!func_initialized_) initialize_func_gradient();
    iter_ = 0;
    FB_CUDA(cudaMemcpyAsync(X_[cur_].p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    eval(X_[cur_].p, G_[cur_].p, e_.p);
    nfev_ = 1;
    FiState h{};
    FB_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(h), cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    h.fire_iter = 0;
    h.dt = prm_.dtstart;
    h.a = prm_.astart;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    init_from_gradient();
  }

  // As modified_fire.hpp:160-178, no initialisation here: before run() the
  // step starts from f = 0, g = 0 (LBFGS initialises, lbfgs.cpp:38-40).
  void one_iteration() override {
    ++nfev_;
    ++iter_;
    const int nxt = 1 - cur_;
    fi_mix<false><<<P_, kThreads, 0, s_>>>(V_.p, G_[cur_].p, n_, st_.p, part_.p, P_);
    fi_step<<<P_, kThreads, 0, s_>>>(X_[cur_].p, X_[nxt].p, V_.p, n_, st_.p, part_.p, P_);
    FB_LAUNCH_CHECK();
    eval(X_[nxt].p, G_[nxt].p, e_.p);
    fi_post<false><<<P_, kThreads, 0, s_>>>(V_.p, G_[nxt].p, n_, part_.p, P_, st_.p);
    fi_fin<false><<<1, 256, 0, s_>>>(st_.p, e_.p, part_.p, P_, host_);
    fi_restore<<<P_, kThreads, 0, s_>>>(V_.p, n_, st_.p);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaStreamSynchronize(s_));
    // the new point stays unless the step was uphill and the step back is on
    if (host_[4] > 0 || !prm_.stepback) cur_ = nxt;
    f_ = host_[0];
    rms_ = host_[1];
    if (verbosity_ > 1 && !(host_[4] > 0)) std::printf("warning: step direction was uphill.  inverting\n");
    if (iprint_ > 0 && iter_ % iprint_ == 0) {
      std::printf("fire: %d fire_iter_number %d dt %.17g a %.17g P %.17g vnorm %.17g E %.17g rms %.17g nfev %d\n",
                  iter_, int(host_[6]), host_[2], host_[3], host_[4], host_[5], f_, rms_, nfev_);
      std::fflush(stdout);
    }
  }

 private:
  void init_from_gradient() {
    fi_init_v<<<P_, kThreads, 0, s_>>>(G_[cur_].p, V_.p, n_, st_.p, part_.p, P_);
    fi_init_fin<<<1, 256, 0, s_>>>(st_.p, e_.p, part_.p, P_, host_);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaStreamSynchronize(s_));
    f_ = host_[0];
    rms_ = host_[1];
    func_initialized_ = true;
  }

  void initialize_func_gradient() override {
    ++nfev_;
    eval(X_[cur_].p, G_[cur_].p, e_.p);
    init_from_gradient();
  }

  int family() const override { return 2; }
  std::vector<Block> image_blocks() override {
    const int64_t n = n_;
    return {{st_.p, int64_t(sizeof(FiState))}, {X_[cur_].p, n * 8}, {G_[cur_].p, n * 8}, {V_.p, n * 8}, {e_.p, 8}};
  }
  void after_load() override {
    FiState h{};
    FB_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(h), cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    fire_keep_params(h, prm_, n_);
    h.cur = cur_;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
  }

  FireParams prm_;
  DevBuf<double> X_[2], G_[2];  // current point and its gradient in [cur_], the trial in the other
  int cur_ = 0;
  DevBuf<double> V_, e_;
  DevBuf<FiState> st_;
};

// Modified FIRE with the whole run(niter) loop on the device, one CUDA graph
// launch: a conditional WHILE node repeats a body whose SWITCH node, keyed by
// the device state, runs the iteration from coordinate buffer 0 or 1 (mixing,
// step into the other buffer, the potential's own kernels, the power test and
// the step back, which keeps the parity); a one-thread kernel after it picks
// the next pass's branch.  The loop control of
// GradientOptimizer::run (optimizer.hpp:97-112) is a device state word, so the
// loop stops on the iteration the host loop would, with no evaluation after it.
// Same iterations, evaluations and trajectory as Fire.
class FireGraph final : public Optimizer {
 public:
  FireGraph(PotentialPtr pot, const double* x0, int64_t n, const FireParams& p)
      : Optimizer(pot, n, p.tol, p.maxiter, p.iprint, p.verbosity), prm_(p) {
    const int64_t nn = std::max<int64_t>(n, 1);
    for (int b = 0; b < 2; ++b) {
      X_[b].alloc(nn);
      G_[b].alloc(nn);
      FB_CUDA(cudaMemsetAsync(G_[b].p, 0, G_[b].bytes(), s_));
    }
    V_.alloc(nn);
    e_.alloc(1);
    st_.alloc(1);
    part_.alloc(int64_t(F_NSLOT) * P_);
    FB_CUDA(cudaMemsetAsync(V_.p, 0, V_.bytes(), s_));
    FB_CUDA(cudaMemsetAsync(part_.p, 0, part_.bytes(), s_));
    FiState h{};
    h.f = 0.0;
    h.dt = p.dtstart;
    h.a = p.astart;
    h.rms = 1e10;
    h.sqrtN = std::sqrt(double(n));
    h.dtmax = p.dtmax;
    h.maxstep = p.maxstep;
    h.finc = p.finc;
    h.fdec = p.fdec;
    h.fa = p.fa;
    h.astart = p.astart;
    h.Nmin = p.Nmin;
    h.stepback = p.stepback ? 1 : 0;
    h.tol = p.tol;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    if (n > 0) FB_CUDA(cudaMemcpyAsync(X_[0].p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
  }
  ~FireGraph() override {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (cap_) cudaStreamDestroy(cap_);
  }

  double* device_x() override { return X_[cur_].p; }
  double* device_g() override { return G_[cur_].p; }

  void set_func_gradient(double f, const double* grad, int64_t n) override {
    if (n != n_) throw InvalidArgument("the gradient has the wrong size");
    FB_CUDA(cudaMemcpyAsync(G_[cur_].p, grad, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaMemcpyAsync(e_.p, &f, sizeof(double), cudaMemcpyHostToDevice, s_));
    init_from_gradient();
  }

  void reset(const double* x0, int64_t n) override {
    if (n != n_) throw InvalidArgument("The number of degrees of freedom (x0.size()) cannot change when calling reset()");
    if (!func_initialized_) initialize_func_gradient();
    iter_ = 0;
    FB_CUDA(cudaMemcpyAsync(X_[cur_].p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s_));
    eval(X_[cur_].p, G_[cur_].p, e_.p);
    nfev_ = 1;
    FiState h{};
    FB_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(h), cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    h.fire_iter = 0;
    h.dt = prm_.dtstart;
    h.a = prm_.astart;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    init_from_gradient();
  }

  // As Fire::one_iteration (modified_fire.hpp:160-178): no initialisation, and
  // one step even below the tolerance.
  void one_iteration() override { launch(1, true); }

  void run(int niter) override {
    if (!func_initialized_) initialize_func_gradient();
    if (niter <= 0) return;
    launch(niter, false);
  }

 private:
  void launch(int niter, bool force) {
    ensure_graph();
    fi_set_stop<<<1, 1, 0, s_>>>(st_.p, niter, iter_, nfev_, force ? 1 : 0);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaGraphLaunch(graph_, s_));
    FiState h{};
    FB_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(h), cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    f_ = h.f;
    rms_ = h.rms;
    iter_ = h.iter;
    nfev_ = h.nfev;
    cur_ = h.cur & 1;
  }

  // One iteration from buffer parity c into body (the trial point goes to 1 - c).
  void capture_body(cudaGraph_t body, int c) {
    const int t = 1 - c;
    FB_CUDA(cudaStreamBeginCaptureToGraph(cap_, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    cudaGraph_t g = nullptr;
    try {
      fi_mix<true><<<P_, kThreads, 0, cap_>>>(V_.p, G_[c].p, n_, st_.p, part_.p, P_);
      fi_step<<<P_, kThreads, 0, cap_>>>(X_[c].p, X_[t].p, V_.p, n_, st_.p, part_.p, P_);
      pot_->energy_gradient(X_[t].p, n_, G_[t].p, e_.p, false, cap_);  // the potential's own launches
      fi_post<true><<<P_, kThreads, 0, cap_>>>(V_.p, G_[t].p, n_, part_.p, P_, st_.p);
      fi_fin<true><<<1, 256, 0, cap_>>>(st_.p, e_.p, part_.p, P_, host_dev_.p);
      fi_restore<<<P_, kThreads, 0, cap_>>>(V_.p, n_, st_.p);
    } catch (...) {
      cudaStreamEndCapture(cap_, &g);
      throw;
    }
    FB_CUDA(cudaStreamEndCapture(cap_, &g));
  }

  // (re)builds the loop graph when the potential's gradient convention changed
  void ensure_graph() {
    if (graph_ && graph_mode_ == pot_->gradient_mode()) return;
    if (pot_->host_steps())
      throw InvalidArgument("the graph FIRE cannot capture a potential that exchanges between processes");
    if (graph_) {
      cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
    }
    // one evaluation outside the capture, so that the potential's lazy set-up
    // (plans, workspaces) is done; into the trial buffers, which the next
    // iteration writes before it reads them
    pot_->energy_gradient(X_[cur_].p, n_, G_[1 - cur_].p, e_.p, false, s_);
    FB_CUDA(cudaStreamSynchronize(s_));
    if (!cap_) FB_CUDA(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking));
    cudaGraph_t top = nullptr;
    FB_CUDA(cudaGraphCreate(&top, 0));
    try {
      cudaGraphConditionalHandle hw, hs;
      FB_CUDA(cudaGraphConditionalHandleCreate(&hw, top, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams wp{};
      wp.type = cudaGraphNodeTypeConditional;
      wp.conditional.handle = hw;
      wp.conditional.type = cudaGraphCondTypeWhile;
      wp.conditional.size = 1;
      cudaGraphNode_t wn;
      FB_CUDA(cudaGraphAddNode(&wn, top, nullptr, 0, &wp));
      cudaGraph_t loop = wp.conditional.phGraph_out[0];
      FB_CUDA(cudaGraphConditionalHandleCreate(&hs, loop, 2, cudaGraphCondAssignDefault));
      FiState* stp = st_.p;
      cudaGraphNodeParams sp{};
      sp.type = cudaGraphNodeTypeConditional;
      sp.conditional.handle = hs;
      sp.conditional.type = cudaGraphCondTypeSwitch;
      sp.conditional.size = 2;
      cudaGraphNode_t sw, kloop;
      FB_CUDA(cudaGraphAddNode(&sw, loop, nullptr, 0, &sp));
      capture_body(sp.conditional.phGraph_out[0], 0);
      capture_body(sp.conditional.phGraph_out[1], 1);
      void* loop_args[] = {&stp, &hw, &hs};
      cudaKernelNodeParams kp{};
      kp.func = reinterpret_cast<void*>(fi_loop);
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(1);
      kp.sharedMemBytes = 0;
      kp.kernelParams = loop_args;
      FB_CUDA(cudaGraphAddKernelNode(&kloop, loop, &sw, 1, &kp));
      FB_CUDA(cudaGraphInstantiate(&graph_, top, 0));
    } catch (...) {
      cudaGraphDestroy(top);
      throw;
    }
    cudaGraphDestroy(top);
    graph_mode_ = pot_->gradient_mode();
  }

  void init_from_gradient() {
    fi_init_v<<<P_, kThreads, 0, s_>>>(G_[cur_].p, V_.p, n_, st_.p, part_.p, P_);
    fi_init_fin<<<1, 256, 0, s_>>>(st_.p, e_.p, part_.p, P_, host_);
    FB_LAUNCH_CHECK();
    FB_CUDA(cudaStreamSynchronize(s_));
    f_ = host_[0];
    rms_ = host_[1];
    func_initialized_ = true;
  }

  void initialize_func_gradient() override {
    ++nfev_;
    eval(X_[cur_].p, G_[cur_].p, e_.p);
    init_from_gradient();
  }

  int family() const override { return 2; }
  std::vector<Block> image_blocks() override {
    const int64_t n = n_;
    return {{st_.p, int64_t(sizeof(FiState))}, {X_[cur_].p, n * 8}, {G_[cur_].p, n * 8}, {V_.p, n * 8}, {e_.p, 8}};
  }
  void after_load() override {
    FiState h{};
    FB_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(h), cudaMemcpyDeviceToHost, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
    fire_keep_params(h, prm_, n_);
    h.cur = cur_;
    FB_CUDA(cudaMemcpyAsync(st_.p, &h, sizeof(h), cudaMemcpyHostToDevice, s_));
    FB_CUDA(cudaStreamSynchronize(s_));
  }

  FireParams prm_;
  DevBuf<double> X_[2], G_[2];  // current point and its gradient in [cur_], the trial in the other
  int cur_ = 0;
  DevBuf<double> V_, e_;
  DevBuf<double> host_dev_{16};  // scalar mirror written by fi_fin inside the graph (not read)
  DevBuf<FiState> st_;
  cudaStream_t cap_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  int graph_mode_ = -1;
};

}  // namespace

Optimizer::Optimizer(PotentialPtr pot, int64_t n, double tol, int maxiter, int iprint, int verbosity)
    : pot_(std::move(pot)), n_(n), tol_(tol), maxiter_(maxiter), iprint_(iprint), verbosity_(verbosity) {
  if (!pot_) throw InvalidArgument("null potential");
  if (n <= 0) throw InvalidArgument("empty coordinate array");
  FB_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
  P_ = std::max(1, std::min(1024, 2 * sm_count()));
  FB_CUDA(cudaMallocHost(&host_, 16 * sizeof(double)));
  for (int i = 0; i < 16; ++i) host_[i] = 0.0;
}

Optimizer::~Optimizer() {
  if (s_) {
    cudaStreamSynchronize(s_);
    cudaStreamDestroy(s_);
  }
  if (host_) cudaFreeHost(host_);
}

void Optimizer::eval(const double* x, double* g, double* e) { pot_->eval(x, n_, g, e, false, s_); }

void Optimizer::run(int niter) {
  if (!func_initialized_) initialize_func_gradient();
  for (int i = 0; i < niter; ++i) {
    if (stop_criterion_satisfied()) break;
    one_iteration();
  }
}

void Optimizer::run() { run(maxiter_ - iter_); }

namespace {
struct ImageHeader {
  uint32_t magic = 0x54534246u;  // "FBST"
  uint32_t version = 1;
  int32_t family = 0, memory = 0;
  int64_t n = 0;
  int32_t iter = 0, nfev = 0, func_initialized = 0, pad = 0;
  double f = 0.0, rms = 0.0;
};
}  // namespace

int64_t Optimizer::state_bytes() const {
  int64_t b = sizeof(ImageHeader);
  for (const Block& k : const_cast<Optimizer*>(this)->image_blocks()) b += k.bytes;
  return b;
}

void Optimizer::save_state(uint8_t* buf) {
  ImageHeader h;
  h.family = family();
  h.memory = memory_length();
  h.n = n_;
  h.iter = iter_;
  h.nfev = nfev_;
  h.func_initialized = func_initialized_ ? 1 : 0;
  h.f = f_;
  h.rms = rms_;
  std::memcpy(buf, &h, sizeof(h));
  int64_t off = sizeof(h);
  for (const Block& k : image_blocks()) {
    FB_CUDA(cudaMemcpyAsync(buf + off, k.dev, k.bytes, cudaMemcpyDeviceToHost, s_));
    off += k.bytes;
  }
  FB_CUDA(cudaStreamSynchronize(s_));
}

void Optimizer::load_state(const uint8_t* buf, int64_t bytes) {
  if (bytes < int64_t(sizeof(ImageHeader))) throw InvalidArgument("optimiser state image too short");
  ImageHeader h;
  std::memcpy(&h, buf, sizeof(h));
  if (h.magic != ImageHeader().magic || h.version != 1) throw InvalidArgument("not an optimiser state image");
  if (h.family != family()) throw InvalidArgument("the state image is of another optimiser family");
  if (h.n != n_) throw InvalidArgument("the state image has another number of coordinates");
  if (h.memory != memory_length()) throw InvalidArgument("the state image has another memory length M");
  if (bytes != state_bytes()) throw InvalidArgument("optimiser state image has the wrong size");
  int64_t off = sizeof(h);
  for (const Block& k : image_blocks()) {
    FB_CUDA(cudaMemcpyAsync(k.dev, buf + off, k.bytes, cudaMemcpyHostToDevice, s_));
    off += k.bytes;
  }
  FB_CUDA(cudaStreamSynchronize(s_));
  iter_ = h.iter;
  nfev_ = h.nfev;
  func_initialized_ = h.func_initialized != 0;
  f_ = h.f;
  rms_ = h.rms;
  after_load();
}

bool Optimizer::stop_criterion_satisfied() {
  if (!func_initialized_) initialize_func_gradient();
  return rms_ <= tol_;
}

void Optimizer::get_state(double* x, double* g, double* f, double* rms, int* nfev, int* niter, int* maxiter,
                          double* H0) {
  if (x) FB_CUDA(cudaMemcpyAsync(x, device_x(), sizeof(double) * n_, cudaMemcpyDeviceToHost, s_));
  if (g) FB_CUDA(cudaMemcpyAsync(g, device_g(), sizeof(double) * n_, cudaMemcpyDeviceToHost, s_));
  FB_CUDA(cudaStreamSynchronize(s_));
  if (f) *f = f_;
  if (rms) *rms = rms_;
  if (nfev) *nfev = nfev_;
  if (niter) *niter = iter_;
  if (maxiter) *maxiter = maxiter_;
  if (H0) *H0 = h0();
}

std::unique_ptr<Optimizer> make_lbfgs(PotentialPtr pot, const double* x0, int64_t n, const LbfgsParams& p) {
  return std::unique_ptr<Optimizer>(new Lbfgs(std::move(pot), x0, n, p));
}

std::unique_ptr<Optimizer> make_fire(PotentialPtr pot, const double* x0, int64_t n, const FireParams& p) {
  return std::unique_ptr<Optimizer>(new Fire(std::move(pot), x0, n, p));
}

std::unique_ptr<Optimizer> make_fire_graph(PotentialPtr pot, const double* x0, int64_t n, const FireParams& p) {
  return std::unique_ptr<Optimizer>(new FireGraph(std::move(pot), x0, n, p));
}

}  // namespace fb
