// C-ABI entry points (include/fresco_b200.h): argument checks, exception ->
// status translation, and the host-buffer call forms.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fresco_b200.h"
#include "ensemble.cuh"
#include "nufft.cuh"
#include "optimizer.cuh"
#include "pointstats.cuh"
#include "potential.cuh"

struct fresco_potential_s {
  fb::PotentialPtr pot;
  cudaStream_t stream = nullptr;
  fb::DevBuf<double> dx, dg, de;
  int64_t cap = -1;
};

struct fresco_optimizer_s {
  std::unique_ptr<fb::Optimizer> opt;
  fresco_potential_s* pot = nullptr;  // borrowed; the Python layer keeps it alive
};

struct fresco_ensemble_s {
  fb::EnsemblePtr ens;
  cudaStream_t stream = nullptr;
  fb::DevBuf<double> dx, dg, de;
};

struct fresco_ensemble_lbfgs_s {
  std::unique_ptr<fb::EnsembleLbfgs> opt;
};

struct fresco_overlap_s {
  std::unique_ptr<fb::OverlapCheck> chk;
};

struct fresco_window_stats_s {
  std::unique_ptr<fb::WindowCounts> wc;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <typename F>
int guarded(F&& f) {
  try {
    g_last_error.clear();
    return f();
  } catch (const fb::InvalidArgument& e) {
    return fail(FRESCO_ERR_INVALID, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(FRESCO_ERR_INVALID, e.what());
  } catch (const std::exception& e) {
    return fail(FRESCO_ERR_RUNTIME, e.what());
  } catch (...) {
    return fail(FRESCO_ERR_RUNTIME, "unknown error");
  }
}

fresco_potential_s* wrap(fb::PotentialPtr p) {
  auto* h = new fresco_potential_s;
  h->pot = std::move(p);
  FB_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  return h;
}

void ensure_io(fresco_potential_s* h, int64_t n) {
  if (h->cap >= n && h->de.p) return;
  h->dx.alloc(std::max<int64_t>(n, 1));
  h->dg.alloc(std::max<int64_t>(n, 1));
  if (!h->de.p) h->de.alloc(1);
  h->cap = n;
}

void check_n(fresco_potential_s* h, int64_t n) {
  const int64_t want = h->pot->ndof();
  if (n < 0) throw fb::InvalidArgument("negative coordinate count");
  if (want >= 0 && n != want) {
    throw fb::InvalidArgument("the coordinate array has size " + std::to_string(n) + ", the potential expects " +
                              std::to_string(want));
  }
}

std::vector<double> vec(const double* p, int64_t n) {
  if (n < 0) throw fb::InvalidArgument("negative size");
  if (n > 0 && !p) throw fb::InvalidArgument("null array");
  return std::vector<double>(p, p + n);
}

}  // namespace

extern "C" {

const char* fresco_last_error(void) { return g_last_error.c_str(); }
int fresco_abi_version(void) { return 100; }

int fresco_nuwu_create(const double* radii, int64_t n_points, double K, const double* sk, const double* v,
                       int64_t n_sk, const double* L, int ndim, double eps, int precision, fresco_potential* out) {
  return guarded([&] {
    if (!out) throw fb::InvalidArgument("null output handle");
    if (ndim < 1 || ndim > 3) throw std::runtime_error("Invalid dimension: " + std::to_string(ndim));
    auto p = fb::make_nuwu(vec(radii, n_points), K, vec(sk, n_sk), vec(v, n_sk), vec(L, ndim), eps, precision);
    *out = wrap(p);
    return FRESCO_OK;
  });
}

int fresco_nuwu_shard_create(const double* radii_local, int64_t n_local, int64_t n_total, double weight_sum_total,
                             double K, const double* sk, const double* v, int64_t n_sk, const double* L, int ndim,
                             double eps, int precision, fresco_potential* out) {
  return guarded([&] {
    if (!out) throw fb::InvalidArgument("null output handle");
    if (ndim < 1 || ndim > 3) throw std::runtime_error("Invalid dimension: " + std::to_string(ndim));
    auto p = fb::make_nuwu_shard(vec(radii_local, n_local), n_total, weight_sum_total, K, vec(sk, n_sk),
                                 vec(v, n_sk), vec(L, ndim), eps, precision);
    *out = wrap(p);
    return FRESCO_OK;
  });
}

int fresco_nuwu_weight_sum(const double* radii, int64_t n, int ndim, double* out) {
  return guarded([&] {
    if (!out || (n > 0 && !radii) || n < 0) throw fb::InvalidArgument("null or negative argument");
    if (ndim < 1 || ndim > 3) throw std::runtime_error("Invalid dimension: " + std::to_string(ndim));
    *out = fb::nuwu_weight_factor_sum(radii, n, ndim);
    return FRESCO_OK;
  });
}

namespace {
fb::NUwUShard* shard_of(fresco_potential p) {
  auto* sh = p ? dynamic_cast<fb::NUwUShard*>(p->pot.get()) : nullptr;
  if (!sh) throw fb::InvalidArgument("not a sharded NUwU handle");
  return sh;
}
}  // namespace

int fresco_nuwu_shard_nrho(fresco_potential p, int64_t* n_rho) {
  return guarded([&] {
    if (!n_rho) throw fb::InvalidArgument("null argument");
    *n_rho = shard_of(p)->n_rho();
    return FRESCO_OK;
  });
}

int fresco_nuwu_shard_rho(fresco_potential p, const double* d_x, int64_t n, double* d_rho, void* stream) {
  return guarded([&] {
    auto* sh = shard_of(p);
    if ((n > 0 && !d_x) || (sh->n_rho() > 0 && !d_rho)) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    sh->shard_rho(d_x, d_rho, static_cast<cudaStream_t>(stream));
    return FRESCO_OK;
  });
}

int fresco_nuwu_shard_finish(fresco_potential p, const double* d_rho, double* d_grad, double* d_energy,
                             void* stream) {
  return guarded([&] {
    auto* sh = shard_of(p);
    if (!d_energy || (sh->n_rho() > 0 && !d_rho)) throw fb::InvalidArgument("null argument");
    sh->shard_finish(d_rho, d_grad, d_energy, static_cast<cudaStream_t>(stream));
    return FRESCO_OK;
  });
}

int fresco_uwu_create(const int* grid, int ndim, double K, const double* sk, const double* v, int64_t n_sk,
                      const double* L, double eps, int precision, fresco_potential* out) {
  return guarded([&] {
    if (!out || !grid) throw fb::InvalidArgument("null argument");
    std::vector<int> g(grid, grid + ndim);
    auto p = fb::make_uwu(g, K, vec(sk, n_sk), vec(v, n_sk), vec(L, ndim), eps, precision);
    *out = wrap(p);
    return FRESCO_OK;
  });
}

int fresco_uwnu_create(const int* grid, int ndim, const double* kpts, int64_t n_k, const double* sk,
                       const double* v, const double* L, double eps, int precision, fresco_potential* out) {
  return guarded([&] {
    if (!out || !grid) throw fb::InvalidArgument("null argument");
    std::vector<int> g(grid, grid + ndim);
    auto p = fb::make_uwnu(g, vec(kpts, n_k * ndim), vec(sk, n_k), vec(v, n_k), vec(L, ndim), eps, precision);
    *out = wrap(p);
    return FRESCO_OK;
  });
}

int fresco_nuwnu_create(const double* radii, int64_t n_points, const double* kpts, int64_t n_k, const double* sk,
                        const double* v, const double* L, int ndim, double eps, int precision,
                        fresco_potential* out) {
  return guarded([&] {
    if (!out) throw fb::InvalidArgument("null output handle");
    auto p = fb::make_nuwnu(vec(radii, n_points), vec(kpts, n_k * ndim), vec(sk, n_k), vec(v, n_k), vec(L, ndim),
                            eps, precision);
    *out = wrap(p);
    return FRESCO_OK;
  });
}

int fresco_inversepower_create(double a, double eps, const double* radii, int64_t n_points, const double* boxv,
                               int ndim, int periodic, int use_cell_lists, double ncellx_scale,
                               fresco_potential* out) {
  return guarded([&] {
    if (!out) throw fb::InvalidArgument("null output handle");
    auto p = fb::make_inversepower(a, eps, vec(radii, n_points), vec(boxv, ndim), periodic != 0,
                                   use_cell_lists != 0, ncellx_scale);
    *out = wrap(p);
    return FRESCO_OK;
  });
}

int fresco_combined_create(fresco_potential* out) {
  return guarded([&] {
    if (!out) throw fb::InvalidArgument("null output handle");
    *out = wrap(std::make_shared<fb::CombinedPotential>());
    return FRESCO_OK;
  });
}

int fresco_combined_add(fresco_potential combined, fresco_potential part) {
  return guarded([&] {
    if (!combined || !part) throw fb::InvalidArgument("null handle");
    auto* c = dynamic_cast<fb::CombinedPotential*>(combined->pot.get());
    if (!c) throw fb::InvalidArgument("not a CombinedPotential");
    c->add(part->pot);
    return FRESCO_OK;
  });
}

void fresco_potential_destroy(fresco_potential p) {
  if (!p) return;
  if (p->stream) {
    cudaStreamSynchronize(p->stream);
    cudaStreamDestroy(p->stream);
  }
  delete p;
}

int64_t fresco_potential_ndof(fresco_potential p) { return p ? p->pot->ndof() : -1; }

int fresco_potential_energy(fresco_potential p, const double* x, int64_t n, double* energy) {
  return guarded([&] {
    if (!p || !energy || (n > 0 && !x)) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    ensure_io(p, n);
    FB_CUDA(cudaMemcpyAsync(p->dx.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, p->stream));
    p->pot->eval(p->dx.p, n, nullptr, p->de.p, false, p->stream);
    p->pot->timer_collect();
    FB_CUDA(cudaMemcpyAsync(energy, p->de.p, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    FB_CUDA(cudaStreamSynchronize(p->stream));
    return FRESCO_OK;
  });
}

int fresco_potential_energy_gradient(fresco_potential p, const double* x, int64_t n, double* grad,
                                     double* energy) {
  return guarded([&] {
    if (!p || !energy || (n > 0 && (!x || !grad))) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    ensure_io(p, n);
    FB_CUDA(cudaMemcpyAsync(p->dx.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, p->stream));
    p->pot->eval(p->dx.p, n, p->dg.p, p->de.p, false, p->stream);
    p->pot->timer_collect();
    FB_CUDA(cudaMemcpyAsync(grad, p->dg.p, sizeof(double) * n, cudaMemcpyDeviceToHost, p->stream));
    FB_CUDA(cudaMemcpyAsync(energy, p->de.p, sizeof(double), cudaMemcpyDeviceToHost, p->stream));
    FB_CUDA(cudaStreamSynchronize(p->stream));
    return FRESCO_OK;
  });
}

int fresco_potential_energy_device(fresco_potential p, const double* d_x, int64_t n, double* d_energy,
                                   int accumulate, void* stream) {
  return guarded([&] {
    if (!p || !d_energy || (n > 0 && !d_x)) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    p->pot->eval(d_x, n, nullptr, d_energy, accumulate != 0, static_cast<cudaStream_t>(stream));
    return FRESCO_OK;
  });
}

int fresco_potential_energy_gradient_device(fresco_potential p, const double* d_x, int64_t n, double* d_grad,
                                            double* d_energy, int accumulate, void* stream) {
  return guarded([&] {
    if (!p || !d_energy || (n > 0 && (!d_x || !d_grad))) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    p->pot->eval(d_x, n, d_grad, d_energy, accumulate != 0, static_cast<cudaStream_t>(stream));
    return FRESCO_OK;
  });
}

int fresco_nuwnu_energy_gradient_noalloc(const double* d_x, int64_t n_points, int ndim, const double* d_weights,
                                         const double* d_kpts, const double* d_sk, const double* d_v, int64_t n_k,
                                         const double* L, int gradient_mode, double* d_grad, double* d_energy,
                                         int accumulate, void* stream) {
  return guarded([&] {
    fb::nuwnu_energy_gradient_noalloc(d_x, n_points, ndim, d_weights, d_kpts, d_sk, d_v, n_k, L, gradient_mode,
                                      d_grad, d_energy, accumulate != 0, static_cast<cudaStream_t>(stream));
    return FRESCO_OK;
  });
}

int fresco_export_structure(const double* x, int64_t n_points, int ndim, const double* L, int Nk, const double* radii,
                            double tol, double* sk, double* gr, double* s_radial, double* g_radial) {
  return guarded([&] {
    if (!x || !L || !sk || !gr || !s_radial || !g_radial) throw fb::InvalidArgument("null argument");
    fb::export_structure(x, n_points, ndim, L, Nk, radii, tol, sk, gr, s_radial, g_radial);
    return FRESCO_OK;
  });
}

int fresco_potential_set_reducer(fresco_potential p, fresco_reduce_fn fn, void* ctx) {
  return guarded([&] {
    if (!p || !fn) throw fb::InvalidArgument("null argument");
    p->pot->set_reducer(fn, ctx);
    return FRESCO_OK;
  });
}

int fresco_inversepower_shard_create(double a, double eps, const double* radii_all, int64_t n_total,
                                     const double* boxv, int ndim, int periodic, int64_t lo, int64_t hi,
                                     fresco_gather_fn gather, fresco_reduce_fn reduce, void* ctx,
                                     fresco_potential* out) {
  return guarded([&] {
    if (!out || !boxv || (n_total > 0 && !radii_all)) throw fb::InvalidArgument("null argument");
    if (ndim < 1 || ndim > 3) throw fb::InvalidArgument("InversePower: ndim must be 1, 2 or 3");
    *out = wrap(fb::make_inversepower_shard(a, eps, std::vector<double>(radii_all, radii_all + n_total),
                                            std::vector<double>(boxv, boxv + ndim), periodic != 0, lo, hi, gather,
                                            reduce, ctx));
    return FRESCO_OK;
  });
}

int fresco_inversepower_halo_create(double a, double eps, const double* radii_all, int64_t n_total,
                                    const double* boxv, int ndim, int64_t lo, int64_t hi, int rank, int nranks,
                                    fresco_gatherv_fn gatherv, fresco_reduce_fn reduce, void* ctx,
                                    fresco_potential* out) {
  return guarded([&] {
    if (!out || !boxv || (n_total > 0 && !radii_all)) throw fb::InvalidArgument("null argument");
    if (ndim < 1 || ndim > 3) throw fb::InvalidArgument("InversePower: ndim must be 1, 2 or 3");
    *out = wrap(fb::make_inversepower_halo(a, eps, std::vector<double>(radii_all, radii_all + n_total),
                                           std::vector<double>(boxv, boxv + ndim), lo, hi, rank, nranks, gatherv,
                                           reduce, ctx));
    return FRESCO_OK;
  });
}

int fresco_inversepower_halo_stats(fresco_potential p, int64_t* exported, int64_t* halo) {
  return guarded([&] {
    if (!p) throw fb::InvalidArgument("null argument");
    if (!p->pot->halo_stats(exported, halo)) throw fb::InvalidArgument("not a repulsion halo shard");
    return FRESCO_OK;
  });
}

int fresco_optimizer_set_reducer(fresco_optimizer o, fresco_reduce_fn fn, void* ctx, int64_t global_ndof) {
  return guarded([&] {
    if (!o || !fn) throw fb::InvalidArgument("null argument");
    o->opt->set_reducer(fn, ctx, global_ndof);
    return FRESCO_OK;
  });
}

int fresco_debug_set_tile_wait_polls(int polls) {
  return guarded([&] {
    fb::set_tile_wait_polls(polls);
    return FRESCO_OK;
  });
}

int fresco_potential_status(fresco_potential p, void* stream, int* status) {
  return guarded([&] {
    if (!p || !status) throw fb::InvalidArgument("null argument");
    *status = p->pot->read_and_clear_status(stream ? static_cast<cudaStream_t>(stream) : p->stream);
    return FRESCO_OK;
  });
}

int fresco_potential_set_gradient_mode(fresco_potential p, int mode) {
  return guarded([&] {
    if (!p) throw fb::InvalidArgument("null handle");
    if (mode != 0 && mode != 1) throw fb::InvalidArgument("gradient mode must be 0 (reference) or 1 (exact)");
    p->pot->set_gradient_mode(mode);
    return FRESCO_OK;
  });
}

int fresco_potential_gradient_mode(fresco_potential p, int* mode) {
  return guarded([&] {
    if (!p || !mode) throw fb::InvalidArgument("null argument");
    *mode = p->pot->gradient_mode();
    return FRESCO_OK;
  });
}

int fresco_potential_set_timing(fresco_potential p, int enabled) {
  return guarded([&] {
    if (!p) throw fb::InvalidArgument("null handle");
    auto& t = p->pot->timer;
    t.enabled = enabled != 0;
    t.used = 0;
    t.total_names.clear();
    t.total_ms.clear();
    t.count.clear();
    return FRESCO_OK;
  });
}

int fresco_potential_get_timing(fresco_potential p, int max_stages, char* names, int names_len, double* total_ms,
                                int* counts, int* n_stages) {
  return guarded([&] {
    if (!p || !n_stages) throw fb::InvalidArgument("null argument");
    p->pot->timer_collect();
    auto& t = p->pot->timer;
    int k = 0, pos = 0;
    for (size_t i = 0; i < t.total_names.size() && k < max_stages; ++i, ++k) {
      if (names) {
        const std::string& s = t.total_names[i];
        if (pos + int(s.size()) + 1 <= names_len) {
          std::memcpy(names + pos, s.c_str(), s.size() + 1);
          pos += int(s.size()) + 1;
        }
      }
      if (total_ms) total_ms[k] = t.total_ms[i];
      if (counts) counts[k] = t.count[i];
    }
    *n_stages = k;
    return FRESCO_OK;
  });
}

int fresco_potential_describe(fresco_potential p, char* buf, int buf_len) {
  return guarded([&] {
    if (!p || !buf || buf_len <= 0) throw fb::InvalidArgument("null argument");
    std::string s = p->pot->describe();
    std::strncpy(buf, s.c_str(), size_t(buf_len - 1));
    buf[buf_len - 1] = 0;
    return FRESCO_OK;
  });
}

// ---- optimisers ----------------------------------------------------------

int fresco_lbfgs_create(fresco_potential p, const double* x0, int64_t n, double tol, int M, double maxstep,
                        double max_f_rise, double H0, int rel_energy, int nsteps, int iprint, int verbosity,
                        fresco_optimizer* out) {
  return guarded([&] {
    if (!p || !out || (n > 0 && !x0)) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    fb::LbfgsParams prm;
    prm.tol = tol;
    prm.M = M;
    prm.maxstep = maxstep;
    prm.max_f_rise = max_f_rise;
    prm.H0 = H0;
    prm.rel_energy = rel_energy != 0;
    prm.maxiter = nsteps;
    prm.iprint = iprint;
    prm.verbosity = verbosity;
    auto* h = new fresco_optimizer_s;
    h->pot = p;
    h->opt = fb::make_lbfgs(p->pot, x0, n, prm);
    *out = h;
    return FRESCO_OK;
  });
}

namespace {
int fire_create(bool graph, fresco_potential p, const double* x0, int64_t n, double dtstart, double dtmax,
                double maxstep, int Nmin, double finc, double fdec, double fa, double astart, double tol,
                int stepback, int nsteps, int iprint, int verbosity, fresco_optimizer* out) {
  return guarded([&] {
    if (!p || !out || (n > 0 && !x0)) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    fb::FireParams prm;
    prm.dtstart = dtstart;
    prm.dtmax = dtmax;
    prm.maxstep = maxstep;
    prm.Nmin = Nmin;
    prm.finc = finc;
    prm.fdec = fdec;
    prm.fa = fa;
    prm.astart = astart;
    prm.tol = tol;
    prm.stepback = stepback != 0;
    prm.maxiter = nsteps;
    prm.iprint = iprint;
    prm.verbosity = verbosity;
    auto* h = new fresco_optimizer_s;
    h->pot = p;
    h->opt = graph ? fb::make_fire_graph(p->pot, x0, n, prm) : fb::make_fire(p->pot, x0, n, prm);
    *out = h;
    return FRESCO_OK;
  });
}
}  // namespace

int fresco_fire_graph_create(fresco_potential p, const double* x0, int64_t n, double dtstart, double dtmax,
                             double maxstep, int Nmin, double finc, double fdec, double fa, double astart, double tol,
                             int stepback, int nsteps, fresco_optimizer* out) {
  return fire_create(true, p, x0, n, dtstart, dtmax, maxstep, Nmin, finc, fdec, fa, astart, tol, stepback, nsteps, -1,
                     0, out);
}

int fresco_fire_create(fresco_potential p, const double* x0, int64_t n, double dtstart, double dtmax,
                       double maxstep, int Nmin, double finc, double fdec, double fa, double astart, double tol,
                       int stepback, int nsteps, int iprint, int verbosity, fresco_optimizer* out) {
  return fire_create(false, p, x0, n, dtstart, dtmax, maxstep, Nmin, finc, fdec, fa, astart, tol, stepback, nsteps,
                     iprint, verbosity, out);
}

int fresco_optimizer_set_func_gradient(fresco_optimizer o, double f, const double* grad, int64_t n) {
  return guarded([&] {
    if (!o || (n > 0 && !grad)) throw fb::InvalidArgument("null argument");
    o->opt->set_func_gradient(f, grad, n);
    return FRESCO_OK;
  });
}

int fresco_lbfgs_set_H0(fresco_optimizer o, double H0) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null handle");
    o->opt->set_H0(H0);
    return FRESCO_OK;
  });
}

int fresco_optimizer_run(fresco_optimizer o, int niter) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null handle");
    if (niter < 0) o->opt->run();
    else o->opt->run(niter);
    return FRESCO_OK;
  });
}

int fresco_optimizer_one_iteration(fresco_optimizer o) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null handle");
    o->opt->one_iteration();
    return FRESCO_OK;
  });
}

int fresco_optimizer_reset(fresco_optimizer o, const double* x0, int64_t n) {
  return guarded([&] {
    if (!o || (n > 0 && !x0)) throw fb::InvalidArgument("null argument");
    o->opt->reset(x0, n);
    return FRESCO_OK;
  });
}

int fresco_optimizer_stop_criterion_satisfied(fresco_optimizer o, int* out) {
  return guarded([&] {
    if (!o || !out) throw fb::InvalidArgument("null argument");
    *out = o->opt->stop_criterion_satisfied() ? 1 : 0;
    return FRESCO_OK;
  });
}

int fresco_optimizer_get_state(fresco_optimizer o, double* x, double* g, double* f, double* rms, int* nfev,
                               int* niter, int* maxiter, double* H0) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null handle");
    o->opt->get_state(x, g, f, rms, nfev, niter, maxiter, H0);
    return FRESCO_OK;
  });
}

int fresco_optimizer_state_bytes(fresco_optimizer o, int64_t* bytes) {
  return guarded([&] {
    if (!o || !bytes) throw fb::InvalidArgument("null argument");
    *bytes = o->opt->state_bytes();
    return FRESCO_OK;
  });
}

int fresco_optimizer_save_state(fresco_optimizer o, void* image) {
  return guarded([&] {
    if (!o || !image) throw fb::InvalidArgument("null argument");
    o->opt->save_state(static_cast<uint8_t*>(image));
    return FRESCO_OK;
  });
}

int fresco_optimizer_load_state(fresco_optimizer o, const void* image, int64_t bytes) {
  return guarded([&] {
    if (!o || !image) throw fb::InvalidArgument("null argument");
    o->opt->load_state(static_cast<const uint8_t*>(image), bytes);
    return FRESCO_OK;
  });
}

int fresco_optimizer_device_state(fresco_optimizer o, double** d_x, double** d_g) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null handle");
    if (d_x) *d_x = o->opt->device_x();
    if (d_g) *d_g = o->opt->device_g();
    return FRESCO_OK;
  });
}

void fresco_optimizer_destroy(fresco_optimizer o) { delete o; }


// ---- batched ensembles -----------------------------------------------------

int fresco_nuwu_ensemble_create(int n_patterns, const int64_t* n_points, const double* radii, const int64_t* n_modes,
                                const double* sk, const double* v, const double* L, int ndim, double eps,
                                int precision, fresco_ensemble* out) {
  return guarded([&] {
    if (!out || !n_points || !radii || !n_modes || !sk || !v || !L) throw fb::InvalidArgument("null argument");
    if (n_patterns < 1) throw fb::InvalidArgument("an ensemble needs at least one pattern");
    if (precision != 0 && precision != 1) throw fb::InvalidArgument("precision must be 0 (fp64) or 1 (fp32)");
    for (int p = 0; p < n_patterns; ++p)
      if (n_points[p] < 1 || n_modes[p] < 1) throw fb::InvalidArgument("empty pattern or mode grid");
    auto* h = new fresco_ensemble_s;
    try {
      h->ens = fb::make_nuwu_ensemble(n_patterns, n_points, radii, n_modes, sk, v, L, ndim, eps, precision);
      FB_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return FRESCO_OK;
  });
}

int fresco_ensemble_info(fresco_ensemble h, int* n_patterns, int64_t* ndof, int64_t* offsets) {
  return guarded([&] {
    if (!h) throw fb::InvalidArgument("null argument");
    if (n_patterns) *n_patterns = h->ens->n_patterns();
    if (ndof) *ndof = h->ens->ndof();
    if (offsets) {
      const auto& off = h->ens->dof_offsets();
      std::memcpy(offsets, off.data(), sizeof(int64_t) * off.size());
    }
    return FRESCO_OK;
  });
}

namespace {
void ensemble_io(fresco_ensemble_s* h, int64_t n) {
  if (n != h->ens->ndof())
    throw fb::InvalidArgument("the coordinate array has size " + std::to_string(n) + ", the ensemble expects " +
                              std::to_string(h->ens->ndof()));
  if (!h->dx.p) {
    h->dx.alloc(n);
    h->dg.alloc(n);
    h->de.alloc(h->ens->n_patterns());
  }
}
}  // namespace

int fresco_ensemble_energy_gradient(fresco_ensemble h, const double* x, int64_t n, double* grad, double* energies) {
  return guarded([&] {
    if (!h || !x || !energies) throw fb::InvalidArgument("null argument");
    ensemble_io(h, n);
    FB_CUDA(cudaMemcpyAsync(h->dx.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    h->ens->eval_graph(h->dx.p, grad ? h->dg.p : nullptr, h->de.p, h->stream);
    if (grad) FB_CUDA(cudaMemcpyAsync(grad, h->dg.p, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    FB_CUDA(cudaMemcpyAsync(energies, h->de.p, sizeof(double) * h->ens->n_patterns(), cudaMemcpyDeviceToHost,
                            h->stream));
    FB_CUDA(cudaStreamSynchronize(h->stream));
    return FRESCO_OK;
  });
}

int fresco_ensemble_energy_gradient_device(fresco_ensemble h, const double* d_x, int64_t n, double* d_grad,
                                           double* d_energies, void* stream) {
  return guarded([&] {
    if (!h || !d_x || !d_energies) throw fb::InvalidArgument("null argument");
    if (n != h->ens->ndof()) throw fb::InvalidArgument("the coordinate array has the wrong size");
    h->ens->eval_graph(d_x, d_grad, d_energies, static_cast<cudaStream_t>(stream));
    return FRESCO_OK;
  });
}

int fresco_ensemble_tune(fresco_ensemble h, const double* x, int64_t n) {
  return guarded([&] {
    if (!h || !x) throw fb::InvalidArgument("null argument");
    ensemble_io(h, n);
    FB_CUDA(cudaMemcpyAsync(h->dx.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    h->ens->tune(h->dx.p, h->dg.p, h->de.p, h->stream);
    return FRESCO_OK;
  });
}

int fresco_ensemble_set_split(fresco_ensemble h, double ratio) {
  return guarded([&] {
    if (!h) throw fb::InvalidArgument("null argument");
    if (!(ratio >= 0.0)) throw fb::InvalidArgument("the split ratio must be >= 0");
    h->ens->set_split(ratio);
    return FRESCO_OK;
  });
}

int fresco_ensemble_set_subproblem_cap(fresco_ensemble h, int cap) {
  return guarded([&] {
    if (!h) throw fb::InvalidArgument("null argument");
    h->ens->set_subproblem_cap(cap);
    return FRESCO_OK;
  });
}

int fresco_ensemble_status(fresco_ensemble h, int* status) {
  return guarded([&] {
    if (!h || !status) throw fb::InvalidArgument("null argument");
    h->ens->read_and_clear_status(status, h->stream);
    return FRESCO_OK;
  });
}

int fresco_ensemble_describe(fresco_ensemble h, char* buf, int buf_len) {
  return guarded([&] {
    if (!h || !buf || buf_len < 1) throw fb::InvalidArgument("null argument");
    const std::string d = h->ens->describe();
    std::strncpy(buf, d.c_str(), size_t(buf_len) - 1);
    buf[buf_len - 1] = '\0';
    return FRESCO_OK;
  });
}

void fresco_ensemble_destroy(fresco_ensemble h) {
  if (!h) return;
  if (h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  delete h;
}

int fresco_ensemble_lbfgs_create(fresco_ensemble h, const double* x0, int64_t n, double tol, int M, double maxstep,
                                 double max_f_rise, double H0, int rel_energy, fresco_ensemble_lbfgs* out) {
  return guarded([&] {
    if (!h || !x0 || !out) throw fb::InvalidArgument("null argument");
    fb::EnsembleLbfgsParams prm;
    prm.tol = tol;
    prm.M = M;
    prm.maxstep = maxstep;
    prm.max_f_rise = max_f_rise;
    prm.H0 = H0;
    prm.rel_energy = rel_energy != 0;
    auto* o = new fresco_ensemble_lbfgs_s;
    try {
      o->opt.reset(new fb::EnsembleLbfgs(h->ens, x0, n, prm));
    } catch (...) {
      delete o;
      throw;
    }
    *out = o;
    return FRESCO_OK;
  });
}

int fresco_lbfgs_graph_create(fresco_potential p, const double* x0, int64_t n, double tol, int M, double maxstep,
                              double max_f_rise, double H0, int rel_energy, fresco_ensemble_lbfgs* out) {
  return guarded([&] {
    if (!p || !x0 || !out) throw fb::InvalidArgument("null argument");
    check_n(p, n);
    fb::EnsembleLbfgsParams prm;
    prm.tol = tol;
    prm.M = M;
    prm.maxstep = maxstep;
    prm.max_f_rise = max_f_rise;
    prm.H0 = H0;
    prm.rel_energy = rel_energy != 0;
    auto* o = new fresco_ensemble_lbfgs_s;
    try {
      o->opt.reset(new fb::EnsembleLbfgs(fb::make_potential_ensemble(p->pot, n), x0, n, prm));
    } catch (...) {
      delete o;
      throw;
    }
    *out = o;
    return FRESCO_OK;
  });
}

int fresco_ensemble_lbfgs_run(fresco_ensemble_lbfgs o, int niter, int* steps_taken) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null argument");
    const int k = o->opt->run(niter);
    if (steps_taken) *steps_taken = k;
    return FRESCO_OK;
  });
}

int fresco_ensemble_lbfgs_steps(fresco_ensemble_lbfgs o, int n_steps) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null argument");
    o->opt->steps(n_steps);
    return FRESCO_OK;
  });
}

int fresco_ensemble_lbfgs_state(fresco_ensemble_lbfgs o, double* x, double* g, double* f, double* rms, int* niter,
                                int* nfev, int* active) {
  return guarded([&] {
    if (!o) throw fb::InvalidArgument("null argument");
    o->opt->get_state(x, g, f, rms, niter, nfev, active);
    return FRESCO_OK;
  });
}

void fresco_ensemble_lbfgs_destroy(fresco_ensemble_lbfgs o) { delete o; }

int fresco_overlap_create(const double* radii, int64_t n, const double* boxv, int ndim, int periodic,
                          fresco_overlap* out) {
  return guarded([&] {
    if (!out || !boxv || (n > 0 && !radii)) throw fb::InvalidArgument("null argument");
    if (ndim < 1 || ndim > 3) throw fb::InvalidArgument("CheckOverlap: ndim must be 1, 2 or 3");
    auto* h = new fresco_overlap_s;
    try {
      h->chk = fb::make_overlap_check(std::vector<double>(radii, radii + std::max<int64_t>(n, 0)),
                                      std::vector<double>(boxv, boxv + ndim), periodic != 0);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return FRESCO_OK;
  });
}

int fresco_overlap_find(fresco_overlap h, const double* x, int64_t ndof, const int64_t* changed, int64_t n_changed,
                        uint64_t* out, int64_t* count) {
  return guarded([&] {
    if (!h || !out || !count || (ndof > 0 && !x) || (n_changed > 0 && !changed))
      throw fb::InvalidArgument("null argument");
    *count = h->chk->find(x, ndof, changed, n_changed, out);
    return FRESCO_OK;
  });
}

void fresco_overlap_destroy(fresco_overlap h) { delete h; }

int fresco_window_stats_create(const double* x, int64_t n_points, int ndim, const double* boxv, const double* radii,
                               int n_radii, uint64_t seed, fresco_window_stats* out) {
  return guarded([&] {
    if (!out || !boxv || !radii || (n_points > 0 && !x)) throw fb::InvalidArgument("null argument");
    if (ndim < 1 || ndim > 3) throw fb::InvalidArgument("point pattern statistics: ndim must be 1, 2 or 3");
    if (n_radii < 1) throw fb::InvalidArgument("at least one window radius is needed");
    auto* h = new fresco_window_stats_s;
    try {
      h->wc = fb::make_window_counts(x, n_points, std::vector<double>(boxv, boxv + ndim),
                                     std::vector<double>(radii, radii + n_radii), seed);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return FRESCO_OK;
  });
}

int fresco_window_stats_run(fresco_window_stats h, int64_t n) {
  return guarded([&] {
    if (!h) throw fb::InvalidArgument("null handle");
    if (n < 0) throw fb::InvalidArgument("the number of windows must be non-negative");
    h->wc->run(n);
    return FRESCO_OK;
  });
}

int fresco_window_stats_set_seed(fresco_window_stats h, uint64_t seed) {
  return guarded([&] {
    if (!h) throw fb::InvalidArgument("null handle");
    h->wc->set_seed(seed);
    return FRESCO_OK;
  });
}

int fresco_window_stats_get(fresco_window_stats h, uint64_t* seed, double* mean, double* var, uint64_t* count) {
  return guarded([&] {
    if (!h) throw fb::InvalidArgument("null handle");
    if (seed) *seed = h->wc->seed();
    h->wc->moments(mean, var, count);
    return FRESCO_OK;
  });
}

void fresco_window_stats_destroy(fresco_window_stats h) { delete h; }

}  // extern "C"
