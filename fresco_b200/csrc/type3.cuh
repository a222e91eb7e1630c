// Type-3 non-uniform FFT on sm_100a: non-uniform points to non-uniform
// frequencies,
//
//   f_v(t_k) = sum_j a_{v,j} exp(i sign t_k . x_j),   v < nvec,
//
// the transform FINUFFT's type 3 computes for the reference's NUwNU loss in
// both directions (source/fresco/nuwnu.hpp:77-78 plans, :165-166 forward,
// :231-282 adjoint).  Method (Barnett, Magland & af Klinteberg, SIAM J. Sci.
// Comput. 41(5), 2019, type 3), per dimension with the sources centred at C
// (half-width X) and the frequencies centred at Dc (half-width S):
//
//   1. a'_j = a_j exp(i sign Dc . (x_j - C)), spread with the ES kernel of
//      width w onto a grid of spacing h = pi / (2 S) and nf >= 2X/h + w
//      points (period P = nf h covers the sources and the kernel's reach, so
//      nothing wraps);
//   2. an inner type-2 NUFFT of that grid, read as nf Fourier modes, at
//      theta_k = (t_k - Dc) h (pre-correction, FFT of the upsampled grid,
//      interpolation);
//   3. f(t_k) = h^d exp(i sign t_k . C) / prod_a psi^(t_k,a - Dc_a) times that,
//      psi^ the kernel's Fourier transform at the spreading grid's scale.
//
// Sources and targets are each set once (set_sources / set_targets with
// fixed coordinates: sorted and their factors computed once) or before every
// execution.  Coordinates are read through an optional map: NUWNU_MAP applies
// the reference's x = (p - round(p/L) + L) 2 pi / L (nuwnu.hpp:134, 193).  A
// coordinate outside the window given at construction raises a device flag
// (window_flag()); the caller then uses another method for that evaluation.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <vector>

#include "nufft.cuh"

namespace fb {

enum Type3Map : int {
  TYPE3_IDENTITY = 0,  // coordinates used as given
  TYPE3_NUWNU_MAP = 1  // x = (p - round(p/L) + L) 2 pi / L per dimension
};

template <typename T>
class Type3 {
 public:
  // D dimensions; n_src sources in [src_lo, src_hi] and n_tgt targets in
  // [tgt_lo, tgt_hi] per dimension (after the coordinate maps); sign of the
  // exponent; tolerance eps; nvec strength vectors per execution.
  Type3(int D, int64_t n_src, int64_t n_tgt, const double* src_lo, const double* src_hi, const double* tgt_lo,
        const double* tgt_hi, int sign, double eps, int nvec);
  ~Type3();
  Type3(const Type3&) = delete;
  Type3& operator=(const Type3&) = delete;

  // Source coordinates (device, n_src x D interleaved) through `map` (L: box
  // per dimension for NUWNU_MAP): window check, centring phases, bin sort.
  void set_sources(const double* d_coords, int map, const double* L, cudaStream_t s);
  // Target coordinates (device, n_tgt x D): inner-grid sort and the output
  // factors h^d exp(i sign t . C) / psi^(t - Dc).
  void set_targets(const double* d_coords, int map, const double* L, cudaStream_t s);
  // out[v * n_tgt + k] = f_v(t_k) for strengths a[v * n_src + j] (device).
  // Real strengths (re, im null) or complex (re = double2 array).
  void execute_real(const double* a, double uniform, double2* out, cudaStream_t s);
  void execute_cplx(const double2* a, double2* out, cudaStream_t s);

  // Device word: non-zero after set_sources / set_targets met a coordinate
  // outside the construction window (cleared by the next set_sources).
  const int* window_flag() const { return flag_.p; }
  std::string describe() const;
  // Fine-grid and spreading-grid sizes per dimension.
  int nf(int a) const { return nf_[a]; }
  int nf2(int a) const { return gin_.nf[a]; }

 private:
  void run(const cplx_t<T>* strengths, double2* out, cudaStream_t s);
  void exec_fft(cplx_t<T>* in, cplx_t<T>* out, cudaStream_t s);

  int D_, sign_, nvec_;
  int64_t Ns_, Nt_;
  double C_[3] = {0, 0, 0}, X_[3] = {1, 1, 1};    // source centre, half-width
  double Dc_[3] = {0, 0, 0}, S_[3] = {1, 1, 1};   // target centre, half-width
  double h_[3] = {1, 1, 1}, alpha_[3] = {1, 1, 1}, P_[3] = {1, 1, 1};
  int nf_[3] = {1, 1, 1};
  ESParams es_;
  std::vector<double> poly_;
  Geom gout_;  // spreading grid (sources)
  Geom gin_;   // inner type-2 fine grid (targets)
  SortBufs sort_src_, sort_tgt_;
  DevBuf<unsigned char> rec_src_, rec_tgt_;
  DevBuf<double> xs_, xt_;           // sort coordinates of sources, targets
  DevBuf<double2> phase_src_;        // exp(i sign Dc . (x_j - C))
  DevBuf<double2> post_;             // output factor per target
  DevBuf<cplx_t<T>> str_;            // nvec x n_src strengths with their phases
  DevBuf<cplx_t<T>> grid_;           // nvec spreading grids
  DevBuf<cplx_t<T>> H_, F_;          // nvec inner fine grids: pre-corrected modes, transformed
  DevBuf<double> corr_[3];           // inner pre-correction per mode
  DevBuf<double> cheb_[3];           // psi^ Chebyshev coefficients per dimension
  int ncheb_[3] = {0, 0, 0};
  DevBuf<int> flag_, status_;
  cufftHandle plan_ = 0;
};

}  // namespace fb
