/*
 * FFTW3 declarations used by the reference's UwU (source/fresco/uwu.hpp:10,
 * 45-49, 134, 164, 187), restated for the oracle build (test
 * infrastructure only).  Semantics: unnormalised multi-dimensional complex
 * DFT, row-major (last dimension fastest), exponent sign = `sign`.
 */
#ifndef FRESCO_ORACLE_FFTW3_SHIM_H
#define FRESCO_ORACLE_FFTW3_SHIM_H

#include <cstddef>

typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#endif
