/*
 * FINUFFT v2.2.0 guru-interface declarations, restated for the oracle build
 * (test infrastructure only).  The reference includes "finufft.h" at
 * source/fresco/nuwu.hpp:6, uwnu.hpp:6 and nuwnu.hpp:6 and calls exactly
 * these four functions; this header lets those files compile unchanged
 * against oracle/shim/shim_impl.cpp, which implements the documented
 * semantics (exact direct sums, or an ES-kernel NUFFT restated from
 * Barnett, Magland & af Klinteberg 2019).  Types and argument order follow
 * FINUFFT's published API so the reference call sites type-check.
 */
#ifndef FRESCO_ORACLE_FINUFFT_SHIM_H
#define FRESCO_ORACLE_FINUFFT_SHIM_H

#include <complex>
#include <cstdint>

typedef struct finufft_opts {
  int modeord;   /* 0: CMCL increasing order (the only order the reference uses) */
  int debug;
  double upsampfac;
} finufft_opts;

typedef struct finufft_plan_s* finufft_plan;

void finufft_default_opts(finufft_opts* o);
int finufft_makeplan(int type, int dim, int64_t* n_modes, int iflag, int ntrans, double tol, finufft_plan* plan,
                     finufft_opts* o);
int finufft_setpts(finufft_plan plan, int64_t M, double* x, double* y, double* z, int64_t N, double* s, double* t,
                   double* u);
int finufft_execute(finufft_plan plan, std::complex<double>* weights, std::complex<double>* result);
int finufft_destroy(finufft_plan plan);

/* Oracle controls (not part of FINUFFT): 0 = auto, 1 = exact direct sums,
 * 2 = ES-kernel NUFFT at the plan tolerance. */
extern "C" void fresco_shim_set_mode(int mode);
// Per-stage seconds of the ES NUFFT (setpts, spread, FFT, modes, interpolation); reset != 0 clears them.
extern "C" void fresco_shim_profile(double* out, int reset);
extern "C" int fresco_shim_get_mode(void);

#endif
