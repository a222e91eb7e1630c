// Reference repulsion (source/fresco/inversepower_potential.hpp + cell lists),
// CombinedPotential (combine_potentials.hpp), LBFGS (source/lbfgs.cpp) and
// modified FIRE (modified_fire.hpp / source/modified_fire.cpp), compiled
// unchanged, plus the generic evaluation entry points.
#include <omp.h>

#include <stdexcept>

#include "fresco/combine_potentials.hpp"
#include "fresco/inversepower_potential.hpp"
#include "fresco/lbfgs.hpp"
#include "fresco/modified_fire.hpp"
#include "ref_glue.h"

extern "C" {

void ref_set_threads(int n) { omp_set_num_threads(n); }
int ref_get_threads(void) { return omp_get_max_threads(); }

double ref_energy(void* h, const double* x, int64_t n) {
  return static_cast<RefPotential*>(h)->p->get_energy(ref_vec(x, n));
}

double ref_energy_gradient(void* h, const double* x, int64_t n, double* grad) {
  std::vector<double> g(n, 0.0);
  const double e = static_cast<RefPotential*>(h)->p->get_energy_gradient(ref_vec(x, n), g);
  for (int64_t i = 0; i < n; ++i) grad[i] = g[i];
  return e;
}

void ref_destroy(void* h) { delete static_cast<RefPotential*>(h); }

void* ref_combined_create(void) {
  return new RefPotential{std::shared_ptr<fresco::BasePotential>(new fresco::CombinedPotential())};
}

void ref_combined_add(void* c, void* part) {
  auto* cp = dynamic_cast<fresco::CombinedPotential*>(static_cast<RefPotential*>(c)->p.get());
  cp->add_potential(static_cast<RefPotential*>(part)->p);
}

void* ref_inversepower_create(double a, double eps, const double* radii, int64_t n, const double* boxv, int ndim,
                              int periodic, int cell_lists, double ncellx_scale) {
  std::vector<double> r = ref_vec(radii, n), b = ref_vec(boxv, ndim);
  fresco::BasePotential* p = nullptr;
  if (!periodic) {
    if (ndim == 2) p = new fresco::InversePowerCartesian<2>(a, eps, r);
    else if (ndim == 3) p = new fresco::InversePowerCartesian<3>(a, eps, r);
  } else if (cell_lists) {
    if (ndim == 2) p = new fresco::InversePowerPeriodicCellLists<2>(a, eps, r, b, ncellx_scale, true);
    else if (ndim == 3) p = new fresco::InversePowerPeriodicCellLists<3>(a, eps, r, b, ncellx_scale, true);
  } else {
    if (ndim == 2) p = new fresco::InversePowerPeriodic<2>(a, eps, r, b);
    else if (ndim == 3) p = new fresco::InversePowerPeriodic<3>(a, eps, r, b);
  }
  if (!p) return nullptr;
  return new RefPotential{std::shared_ptr<fresco::BasePotential>(p)};
}

struct RefOpt {
  std::shared_ptr<fresco::GradientOptimizer> o;
  bool lbfgs;
};

void* ref_lbfgs_create(void* pot, const double* x0, int64_t n, double tol, int M, double maxstep, double maxErise,
                       double H0, int rel, int nsteps) {
  auto* l = new fresco::LBFGS(static_cast<RefPotential*>(pot)->p, ref_vec(x0, n), tol, M);
  l->set_H0(H0);
  l->set_maxstep(maxstep);
  l->set_max_f_rise(maxErise);
  l->set_max_iter(nsteps);
  if (rel) l->set_use_relative_f(1);
  return new RefOpt{std::shared_ptr<fresco::GradientOptimizer>(l), true};
}

void* ref_fire_create(void* pot, const double* x0, int64_t n, double dtstart, double dtmax, double maxstep, int Nmin,
                      double finc, double fdec, double fa, double astart, double tol, int stepback, int nsteps) {
  std::vector<double> x = ref_vec(x0, n);
  auto* f = new fresco::MODIFIED_FIRE(static_cast<RefPotential*>(pot)->p, x, dtstart, dtmax, maxstep, size_t(Nmin),
                                      finc, fdec, fa, astart, tol, stepback != 0);
  f->set_max_iter(nsteps);
  return new RefOpt{std::shared_ptr<fresco::GradientOptimizer>(f), false};
}

void ref_lbfgs_set_H0(void* o, double H0) {
  auto* r = static_cast<RefOpt*>(o);
  if (r->lbfgs) static_cast<fresco::LBFGS*>(r->o.get())->set_H0(H0);
}

void ref_opt_run(void* o, int niter) { static_cast<RefOpt*>(o)->o->run(niter); }
void ref_opt_one_iteration(void* o) { static_cast<RefOpt*>(o)->o->one_iteration(); }

void ref_opt_state(void* o, double* x, double* g, double* f, double* rms, int* nfev, int* niter, double* H0) {
  auto* r = static_cast<RefOpt*>(o);
  std::vector<double> xv = r->o->get_x(), gv = r->o->get_g();
  for (size_t i = 0; i < xv.size(); ++i) {
    if (x) x[i] = xv[i];
    if (g) g[i] = gv[i];
  }
  *f = r->o->get_f();
  *rms = r->o->get_rms();
  *nfev = r->o->get_nfev();
  *niter = r->o->get_niter();
  *H0 = r->lbfgs ? static_cast<fresco::LBFGS*>(r->o.get())->get_H0() : 0.0;
}

void ref_opt_destroy(void* o) { delete static_cast<RefOpt*>(o); }

}  // extern "C"
