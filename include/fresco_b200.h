/*
 * fresco_b200 C ABI: the drop-in boundary of the B200 implementation of
 * FReSCo's loss-and-gradient path.
 *
 * The reference binds its C++ classes from Cython (fresco/potentials/*.pxd,
 * fresco/optimize/*.pyx).  Each entry point below replaces one C++ member
 * the Cython layer calls; the citation names the reference declaration (paths
 * relative to the reference project root).  Arguments are plain pointers and
 * sizes; "host" pointers are ordinary CPU memory, "device" pointers are CUDA
 * global memory on the handle's device.
 *
 * Return value: FRESCO_OK (0) or an error code; fresco_last_error() gives the
 * message for the calling thread.  FRESCO_ERR_INVALID corresponds to the
 * reference's std::invalid_argument (Python ValueError), the others to
 * std::runtime_error (Python RuntimeError).
 *
 * Threading: like the reference objects (which mutate plan and gradient
 * members), a handle is not re-entrant; calls on one handle must not overlap.
 */
#ifndef FRESCO_B200_H
#define FRESCO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct fresco_potential_s* fresco_potential;
typedef struct fresco_optimizer_s* fresco_optimizer;
typedef struct fresco_ensemble_s* fresco_ensemble;
typedef struct fresco_ensemble_lbfgs_s* fresco_ensemble_lbfgs;
typedef struct fresco_overlap_s* fresco_overlap;
/* Sums `count` doubles at device address `data` over the processes that share
 * one pattern, in place, ordered on the CUDA stream `stream` (an all-reduce
 * supplied by the caller, e.g. NCCL through torch.distributed). */
typedef void (*fresco_reduce_fn)(double* data, int64_t count, void* stream, void* ctx);
/* Concatenates the processes' local arrays (local_count doubles each) in
 * process order into the device array `full` (full_count doubles), ordered on
 * `stream` (an all-gather supplied by the caller). */
typedef void (*fresco_gather_fn)(const double* local, int64_t local_count, double* full, int64_t full_count,
                                 void* stream, void* ctx);
/* Concatenates the processes' local arrays, whose lengths differ, in process
 * order into the device array `full` (at most full_capacity doubles) and
 * writes process q's length to counts[q] (host memory), ordered on `stream`
 * (an all-gather of varying sizes supplied by the caller). */
typedef void (*fresco_gatherv_fn)(const double* local, int64_t local_count, double* full, int64_t full_capacity,
                                  int64_t* counts, void* stream, void* ctx);
typedef struct fresco_window_stats_s* fresco_window_stats;

enum {
  FRESCO_OK = 0,
  FRESCO_ERR_INVALID = 1,     /* bad argument (reference: std::invalid_argument) */
  FRESCO_ERR_RUNTIME = 2,     /* CUDA/cuFFT failure or other runtime error */
  FRESCO_ERR_NONFINITE = 3,   /* a coordinate was NaN/inf: energy and gradient are NaN */
};

enum { FRESCO_FP64 = 0, FRESCO_FP32 = 1 };

/* Message of the last error on this thread ("" if none). */
const char* fresco_last_error(void);
/* ABI version (major * 100 + minor). */
int fresco_abi_version(void);

/* ---- potentials: constructors ------------------------------------------ */

/* fresco::NUwU(radii, K, Sk, V, L, eps)  (source/fresco/nuwu.hpp:35-52;
 * Cython binding fresco/potentials/nuwu.pxd:9).  sk and v hold n_sk doubles
 * each (flattened, dimension 0 fastest); ndim = len(L).  precision selects
 * the FP64 form or the FP32 spread/FFT/interpolation form (FP64 reduction). */
int fresco_nuwu_create(const double* radii, int64_t n_points, double K, const double* sk, const double* v,
                       int64_t n_sk, const double* L, int ndim, double eps, int precision, fresco_potential* out);

/* One NUwU pattern split over processes (GPUs): the loss of
 * fresco::NUwU::get_energy_gradient (source/fresco/nuwu.hpp:210-317) for the
 * union of all shards' points, each shard holding radii_local[n_local].
 * n_total is the pattern's point count and weight_sum_total the sum over all
 * points of the per-point weight factor (fresco_nuwu_weight_sum of each shard,
 * summed), so that the weights are normalised as nuwu.hpp:125-149 does for the
 * whole pattern.  Per evaluation: fresco_nuwu_shard_rho on every shard, a sum
 * of the rho arrays over the shards (one all-reduce), then
 * fresco_nuwu_shard_finish on every shard.  The shard uses the cuFFT
 * transforms (the band path fuses the point where the sum happens). */
int fresco_nuwu_shard_create(const double* radii_local, int64_t n_local, int64_t n_total, double weight_sum_total,
                             double K, const double* sk, const double* v, int64_t n_sk, const double* L, int ndim,
                             double eps, int precision, fresco_potential* out);
/* Sum over radii[n] of NUwU's per-point weight factor, (pi r^2)^2 in 2D and
 * (4/3 pi r^3)^3 in 3D (the area factor applied once per dimension, nuwu.hpp:131-141). */
int fresco_nuwu_weight_sum(const double* radii, int64_t n, int ndim, double* out);
/* Complex values per rho array (the active modes): d_rho holds 2 * n_rho doubles. */
int fresco_nuwu_shard_nrho(fresco_potential p, int64_t* n_rho);
/* rho of this shard's points (d_x[n], device) at the active modes into d_rho
 * (device), enqueued on stream.  Sums over shards give the pattern's rho. */
int fresco_nuwu_shard_rho(fresco_potential p, const double* d_x, int64_t n, double* d_rho, void* stream);
/* With d_rho holding the sum over all shards: *d_energy = the pattern's loss
 * (the same on every shard) and, if d_grad is not NULL, d_grad[n] = this
 * shard's gradient.  Uses the points of the last fresco_nuwu_shard_rho call. */
int fresco_nuwu_shard_finish(fresco_potential p, const double* d_rho, double* d_grad, double* d_energy,
                             void* stream);

/* fresco::UwU(N, K, Sk, V, L, eps)  (source/fresco/uwu.hpp:34-50; uwu.pxd).
 * sk and v are already ifftshifted (natural FFT order, as uwu.pyx:14-15
 * passes them).  grid holds ndim ints, slowest first (FFTW row-major). */
int fresco_uwu_create(const int* grid, int ndim, double K, const double* sk, const double* v, int64_t n_sk,
                      const double* L, double eps, int precision, fresco_potential* out);

/* fresco::UwNU(N, K, Sk, V, L, eps)  (source/fresco/uwnu.hpp:231-282; uwnu.pxd).
 * kpts holds n_k*ndim doubles interleaved; grid holds ndim ints with
 * grid[0] the fastest dimension (FINUFFT's n_modes order). */
int fresco_uwnu_create(const int* grid, int ndim, const double* kpts, int64_t n_k, const double* sk,
                       const double* v, const double* L, double eps, int precision, fresco_potential* out);

/* fresco::NUwNU(radii, K, Sk, V, L, eps)  (source/fresco/nuwnu.hpp:36-79; nuwnu.pxd). */
int fresco_nuwnu_create(const double* radii, int64_t n_points, const double* kpts, int64_t n_k, const double* sk,
                        const double* v, const double* L, int ndim, double eps, int precision,
                        fresco_potential* out);

/* fresco::InversePowerPeriodicCellLists<ndim>(pow, eps, radii, boxv,
 * ncellx_scale, balance_omp) and InversePowerPeriodic / InversePowerCartesian
 * (source/fresco/inversepower_potential.hpp:80-124;
 * fresco/potentials/inversepower_potential.pyx:16-79).  periodic = 0 selects
 * the Cartesian distance. */
int fresco_inversepower_create(double a, double eps, const double* radii, int64_t n_points, const double* boxv,
                               int ndim, int periodic, int use_cell_lists, double ncellx_scale,
                               fresco_potential* out);

/* fresco::CombinedPotential() and add_potential()  (source/fresco/combine_potentials.hpp:
 * 28-37; fresco/potentials/_fresco.pxd:39-44).  The combined handle keeps a
 * reference to each part. */
int fresco_combined_create(fresco_potential* out);
int fresco_combined_add(fresco_potential combined, fresco_potential part);

void fresco_potential_destroy(fresco_potential p);
/* Coordinates expected by the potential (-1 when any size is accepted). */
int64_t fresco_potential_ndof(fresco_potential p);

/* ---- potentials: evaluation --------------------------------------------- */

/* BasePotential::get_energy(x)  (source/fresco/base_potential.hpp:28-31),
 * host buffers: x[n] in, *energy out.  Synchronous. */
int fresco_potential_energy(fresco_potential p, const double* x, int64_t n, double* energy);

/* BasePotential::get_energy_gradient(x, grad)  (base_potential.hpp:38-43),
 * host buffers: x[n] in, grad[n] and *energy out.  Synchronous. */
int fresco_potential_energy_gradient(fresco_potential p, const double* x, int64_t n, double* grad,
                                     double* energy);

/* Device-resident forms of the two calls above: d_x, d_grad, d_energy are
 * device pointers; the work is enqueued on `stream` (a cudaStream_t; NULL
 * selects the legacy default stream) and the call returns without waiting.
 * accumulate != 0 adds into d_grad / d_energy (BasePotential::
 * add_energy_gradient, base_potential.hpp:50-58). */
int fresco_potential_energy_device(fresco_potential p, const double* d_x, int64_t n, double* d_energy,
                                   int accumulate, void* stream);
int fresco_potential_energy_gradient_device(fresco_potential p, const double* d_x, int64_t n, double* d_grad,
                                            double* d_energy, int accumulate, void* stream);

/* Allocation-free NUwNU loss and gradient.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory at the point where they need
 * the loss: a host that hands the whole GPU to its own memory pool (so that
 * cudaMalloc would fail), or a time-stepping loop that must not call cudaFree
 * because it waits for all work on the device.  Every other entry point
 * allocates when its handle is created; this one takes no handle.  It
 * computes exactly what a NUwNU handle computes (fresco_nuwnu_create, then
 * fresco_potential_energy_gradient_device), reading only the caller's arrays:
 *   d_x        n_points*ndim coordinates (device),
 *   d_weights  n_points per-point weights c_j as the reference derives them
 *              from the radii ((pi r^2)^ndim in 2D, (4/3 pi r^3)^ndim in 3D,
 *              then scaled to sum to n_points; nuwnu.hpp:81-105), or NULL for
 *              equal radii (c_j = 1),
 *   d_kpts     n_k*ndim k-points, d_sk and d_v n_k values each (device),
 *   L          ndim box lengths (HOST array),
 *   d_grad     n_points*ndim gradient out (device; NULL: energy only),
 *   d_energy   one double out (device).
 * gradient_mode is 0 (reference convention) or 1 (exact derivative), as in
 * fresco_potential_set_gradient_mode; accumulate != 0 adds into the outputs.
 * The per-k-point sums live in a static device array of 128 KiB that the
 * library holds on every GPU it is loaded on until the process exits, so
 * n_k may not exceed 4096 (FRESCO_ERR_INVALID beyond that).  All calls share
 * that array: calls whose work overlaps on the GPU (two streams, or two host
 * threads on one device) race and give undefined results.  The first call in
 * a device's CUDA context looks up the array's device address (and may load
 * the library's device code there); make that first call before any stream
 * capture begins.  The address is cached per context: after cudaDeviceReset,
 * or with another context current, the next call looks it up again.
 * Works on the current device and enqueues on `stream` without waiting.  A
 * non-finite coordinate makes the energy and the gradient NaN. */
int fresco_nuwnu_energy_gradient_noalloc(const double* d_x, int64_t n_points, int ndim, const double* d_weights,
                                         const double* d_kpts, const double* d_sk, const double* d_v, int64_t n_k,
                                         const double* L, int gradient_mode, double* d_grad, double* d_energy,
                                         int accumulate, void* stream);

/* fresco.utils.export_structure(r, L, Nk, radii, tol) (fresco/utils/utils.py:16-52) with
 * radial_profile (utils.py:138-152), computed on the device.  Host arrays: x holds
 * n_points*ndim coordinates, L ndim box lengths, radii n_points values or NULL; sk and gr
 * receive Nk^ndim values (S(k) and g(r) in centred order, dimension 0 slowest),
 * s_radial and g_radial Nk/2 + 1 radial averages.  ndim is 2 or 3.  Synchronous. */
int fresco_export_structure(const double* x, int64_t n_points, int ndim, const double* L, int Nk, const double* radii,
                            double tol, double* sk, double* gr, double* s_radial, double* g_radial);

/* A NUwU shard (fresco_nuwu_shard_create) with a reducer evaluates the whole
 * pattern through the ordinary calls and optimisers: its rho, fn over the
 * active modes' rho (2 * n_rho doubles), the shared mode pass, its own
 * gradient.  Other potentials have no exchange step and refuse one.  No
 * reference counterpart (the reference evaluates a pattern in one process,
 * source/fresco/nuwu.hpp:210-317). */
int fresco_potential_set_reducer(fresco_potential p, fresco_reduce_fn fn, void* ctx);
/* InversePower (inversepower_potential.hpp:104-124, cell lists) over a
 * pattern split into index slabs: this process owns points [lo, hi) of the
 * n_total whose radii are given, and takes its slab's coordinates.  Each
 * evaluation gathers all slabs (gather), evaluates the whole pattern's
 * repulsion and keeps this slab's gradient; the energy is counted by the
 * process whose slab starts at point 0 and summed by reduce, so every process
 * holds the pattern's energy.  Combines with a NUwU shard in a
 * CombinedPotential. */
int fresco_inversepower_shard_create(double a, double eps, const double* radii_all, int64_t n_total,
                                     const double* boxv, int ndim, int periodic, int64_t lo, int64_t hi,
                                     fresco_gather_fn gather, fresco_reduce_fn reduce, void* ctx,
                                     fresco_potential* out);
/* InversePower (periodic box, cell lists: inversepower_potential.hpp:104-124,
 * cell_list_potential.hpp:442-465) over a pattern split into index slabs that
 * are spatially compact (points ordered along axis 0 before the split): this
 * process is process `rank` of `nranks` and owns points [lo, hi) of the
 * n_total whose radii are given.  Each evaluation gathers every process's
 * occupied columns (cells along axis 0) through gatherv, exports its points
 * next to another process's columns, gathers the exports (gatherv), keeps the
 * received points next to its own columns as a halo, evaluates its own
 * points' pairs over own + halo points and sums the energy with reduce:
 * every process holds the pattern's energy and its slab's gradient.  Needs
 * at least 3 cells per dimension (FRESCO_ERR_INVALID otherwise).  Combines
 * with a NUwU shard in a CombinedPotential. */
int fresco_inversepower_halo_create(double a, double eps, const double* radii_all, int64_t n_total,
                                    const double* boxv, int ndim, int64_t lo, int64_t hi, int rank, int nranks,
                                    fresco_gatherv_fn gatherv, fresco_reduce_fn reduce, void* ctx,
                                    fresco_potential* out);
/* Points this process exported and halo points it kept in the last
 * evaluation of a halo shard (FRESCO_ERR_INVALID for other potentials). */
int fresco_inversepower_halo_stats(fresco_potential p, int64_t* exported, int64_t* halo);

/* Sticky status bits raised since the last call: 1 non-finite input, 2 a
 * bounded buffer overflowed, 4 a bounded wait gave up (the evaluation's
 * energy and gradient are then NaN), 8 an interpolation tile copy outlasted
 * its first bounded wait and was waited for again (the results are
 * complete), 16 a point outside a type-3 NUFFT plan's window made NUwNU use
 * exact sums for that evaluation (the results are complete).  Synchronises
 * `stream`.  No reference counterpart (FINUFFT's
 * return codes are ignored at source/fresco/nuwu.hpp:191-192, 256-258). */
int fresco_potential_status(fresco_potential p, void* stream, int* status);

/* Mbarrier polls of the first bounded wait for a 2D interpolation tile copy,
 * for kernels launched (or graphs captured) from now on, process-wide; polls
 * < 0 restores the default (1 << 22), 0 makes the first wait run out at once.
 * A block whose polls run out raises status bit 8 and waits again, bounded by
 * two seconds, so 0 exercises that second wait without changing any result.
 * A diagnostic with no reference counterpart. */
int fresco_debug_set_tile_wait_polls(int polls);

/* Gradient convention of the handle: 0 (default) returns the reference's own
 * gradient formula (drop-in parity); 1 returns the exact derivative of the
 * energy with respect to the input coordinates, as automatic differentiation
 * needs.  No reference counterpart: the reference only has convention 0
 * (NUwU/NUwNU differentiate the 2 pi-scaled coordinate, nuwu.hpp:219; UwNU
 * divides by 2 pi, uwnu.hpp:352; NUwNU omits conj(c_j), nuwnu.hpp:269; UwU
 * halves the rho term and drops d(1/R), uwu.hpp:178). */
int fresco_potential_set_gradient_mode(fresco_potential p, int mode);
/* The handle's current gradient convention (0 or 1). */
int fresco_potential_gradient_mode(fresco_potential p, int* mode);

/* Per-stage device timing of the next evaluations (CUDA events). */
int fresco_potential_set_timing(fresco_potential p, int enabled);
/* Copies up to max_stages (name, total ms, count) triples; names are
 * written NUL-separated into names (capacity names_len). */
int fresco_potential_get_timing(fresco_potential p, int max_stages, char* names, int names_len, double* total_ms,
                                int* counts, int* n_stages);
/* Describes the NUFFT set-up of a NUwU/UwNU handle: kernel width, fine grid
 * per dimension, active modes, FFT precision bytes. */
int fresco_potential_describe(fresco_potential p, char* buf, int buf_len);

/* ---- optimisers ---------------------------------------------------------- */

/* fresco::LBFGS(potential, x0, tol, M) plus set_H0 / set_maxstep /
 * set_max_f_rise / set_max_iter / set_verbosity / set_iprint /
 * set_use_relative_f  (source/fresco/lbfgs.hpp:316-342;
 * fresco/optimize/_lbfgs_cpp.pyx:22-66).  All state lives on the device. */
int fresco_lbfgs_create(fresco_potential p, const double* x0, int64_t n, double tol, int M, double maxstep,
                        double max_f_rise, double H0, int rel_energy, int nsteps, int iprint, int verbosity,
                        fresco_optimizer* out);

/* fresco::MODIFIED_FIRE(potential, x0, dtstart, dtmax, maxstep, Nmin, finc,
 * fdec, fa, astart, tol, stepback)  (source/fresco/modified_fire.hpp:57-60;
 * fresco/optimize/_modified_fire_cpp.pyx:18-37). */
int fresco_fire_create(fresco_potential p, const double* x0, int64_t n, double dtstart, double dtmax,
                       double maxstep, int Nmin, double finc, double fdec, double fa, double astart, double tol,
                       int stepback, int nsteps, int iprint, int verbosity, fresco_optimizer* out);
/* The same modified FIRE (modified_fire.hpp:44-230) with each iteration one
 * CUDA graph launch: the step, the potential call and the accept/step-back
 * decision all run on the device, and run(niter) reads the iteration count
 * back once per batch of launches.  Same trajectory, iterations and nfev as
 * fresco_fire_create; no progress printing (iprint, verbosity).  Driven by
 * the fresco_optimizer_* calls below. */
int fresco_fire_graph_create(fresco_potential p, const double* x0, int64_t n, double dtstart, double dtmax,
                             double maxstep, int Nmin, double finc, double fdec, double fa, double astart, double tol,
                             int stepback, int nsteps, fresco_optimizer* out);

/* LBFGS over a pattern split between processes (each process's optimiser
 * holds its slab of x and its shard's potential): every dot product of
 * lbfgs.cpp:9-258 (two-loop recursion, step norm, accept test, rms) has its
 * block partial sums reduced by fn before use, and the rms is taken over
 * global_ndof coordinates.  Call before the first evaluation; each process
 * takes the same steps.  LBFGS handles only. */
int fresco_optimizer_set_reducer(fresco_optimizer o, fresco_reduce_fn fn, void* ctx, int64_t global_ndof);
/* GradientOptimizer::set_func_gradient(f, grad)  (source/fresco/optimizer.hpp:127-144). */
int fresco_optimizer_set_func_gradient(fresco_optimizer o, double f, const double* grad, int64_t n);
/* LBFGS::set_H0(H0)  (source/fresco/lbfgs.hpp:70-76; fresco/optimize/_lbfgs_cpp.pyx:72-74): the
 * initial inverse-Hessian scale used by the next step, until the next memory
 * update replaces it (lbfgs.cpp:101).  Prints the reference's warning when
 * called after the first iteration.  LBFGS handles only (FRESCO_ERR_INVALID
 * otherwise). */
int fresco_lbfgs_set_H0(fresco_optimizer o, double H0);
/* GradientOptimizer::run(niter) / run()  (optimizer.hpp:97-121); niter < 0 runs to maxiter. */
int fresco_optimizer_run(fresco_optimizer o, int niter);
/* one_iteration()  (lbfgs.cpp:36-64, modified_fire.hpp:160-230). */
int fresco_optimizer_one_iteration(fresco_optimizer o);
/* reset(x0)  (lbfgs.cpp:247-257, modified_fire.hpp:84-112). */
int fresco_optimizer_reset(fresco_optimizer o, const double* x0, int64_t n);
/* stop_criterion_satisfied()  (optimizer.hpp:174-180). */
int fresco_optimizer_stop_criterion_satisfied(fresco_optimizer o, int* out);
/* get_x / get_g / get_f / get_rms / get_nfev / get_niter / get_maxiter and
 * LBFGS::get_H0  (optimizer.hpp:160-168, lbfgs.hpp:345).  x and g may be NULL. */
int fresco_optimizer_get_state(fresco_optimizer o, double* x, double* g, double* f, double* rms, int* nfev,
                               int* niter, int* maxiter, double* H0);
/* Device pointers of the optimiser's x and g (valid until destroy). */
int fresco_optimizer_device_state(fresco_optimizer o, double** d_x, double** d_g);
/* Checkpoint for an exact resume (no reference counterpart: the reference
 * saves coordinates only, opt.pyx:42-54).  The image holds the optimiser's
 * device state (x, g, LBFGS memory pairs or FIRE velocities, step sizes) and
 * counters; *bytes receives its size.  An image loads into an optimiser of
 * the same family (LBFGS, or either FIRE form), coordinate count and memory
 * length M, which keeps its own parameters and continues the saved
 * trajectory. */
int fresco_optimizer_state_bytes(fresco_optimizer o, int64_t* bytes);
int fresco_optimizer_save_state(fresco_optimizer o, void* image);
int fresco_optimizer_load_state(fresco_optimizer o, const void* image, int64_t bytes);
void fresco_optimizer_destroy(fresco_optimizer o);

/* ---- batched ensembles ---------------------------------------------------- */

/* P independent 2D NUwU patterns evaluated together: the batched form of P
 * objects fresco.potentials.NUwU(radii_p, K, Sk_p, V_p, L, eps)
 * (fresco/potentials/nuwu.pyx:10-23, source/fresco/nuwu.hpp:35-149).
 * n_points[p] points and n_modes[p] = len(V_p) per pattern; radii holds the
 * sum of n_points values and sk, v the sum of n_modes values, pattern after
 * pattern; L (ndim = 2 values) is common.  Coordinates of all patterns are
 * concatenated, pattern p at doubles [offsets[p], offsets[p+1]). */
int fresco_nuwu_ensemble_create(int n_patterns, const int64_t* n_points, const double* radii, const int64_t* n_modes,
                                const double* sk, const double* v, const double* L, int ndim, double eps,
                                int precision, fresco_ensemble* out);
/* Number of patterns, total coordinate count and the P + 1 offsets (may be NULL). */
int fresco_ensemble_info(fresco_ensemble h, int* n_patterns, int64_t* ndof, int64_t* offsets);
/* get_energy_gradient of every pattern (host buffers; grad may be NULL for
 * energies only): energies[p], grad in the x layout. */
int fresco_ensemble_energy_gradient(fresco_ensemble h, const double* x, int64_t n, double* grad, double* energies);
/* Device-buffer form, asynchronous on stream, replayed as a CUDA graph when
 * the same buffers repeat. */
int fresco_ensemble_energy_gradient_device(fresco_ensemble h, const double* d_x, int64_t n, double* d_grad,
                                           double* d_energies, void* stream);
/* Times the tiled and direct spreading/interpolation split on x and keeps
 * the fastest per group of equal mode grids. */
int fresco_ensemble_tune(fresco_ensemble h, const double* x, int64_t n);
/* Sets the split by hand: patterns whose tap work N w^2 is below ratio x the
 * tile cells of their bins use the direct kernels (0: all tiled). */
int fresco_ensemble_set_split(fresco_ensemble h, double ratio);
/* Sets the largest subproblem of the tile kernels (points per block; each
 * bin is cut into equal parts of at most cap points), 160..640; tune picks it
 * per group of equal grids together with the split.  No reference
 * counterpart (FINUFFT's GPU spreader calls it maxsubprobsize). */
int fresco_ensemble_set_subproblem_cap(fresco_ensemble h, int cap);
/* Per-pattern status bits since the last call (P ints). */
int fresco_ensemble_status(fresco_ensemble h, int* status);
int fresco_ensemble_describe(fresco_ensemble h, char* buf, int buf_len);
void fresco_ensemble_destroy(fresco_ensemble h);

/* LBFGS_CPP(x0_p, NUwU_p, M=M, tol=tol, maxstep=..., maxErise=..., H0=...)
 * for every pattern at once (fresco/optimize/_lbfgs_cpp.pyx:22-66,
 * source/lbfgs.cpp:9-258); x0 in the ensemble's layout. */
int fresco_ensemble_lbfgs_create(fresco_ensemble h, const double* x0, int64_t n, double tol, int M, double maxstep,
                                 double max_f_rise, double H0, int rel_energy, fresco_ensemble_lbfgs* out);
/* LBFGS_CPP(x0, potential, ...) (fresco/optimize/_lbfgs_cpp.pyx:22-66,
 * source/lbfgs.cpp:9-258) for any single potential with its whole iteration
 * on the device: a one-pattern ensemble optimiser, driven by the
 * fresco_ensemble_lbfgs_* calls below (one CUDA graph launch per evaluation). */
int fresco_lbfgs_graph_create(fresco_potential p, const double* x0, int64_t n, double tol, int M, double maxstep,
                              double max_f_rise, double H0, int rel_energy, fresco_ensemble_lbfgs* out);
/* run(niter) of every pattern (optimizer.hpp:97-112); steps_taken (may be
 * NULL) receives the number of ensemble evaluations used. */
int fresco_ensemble_lbfgs_run(fresco_ensemble_lbfgs o, int niter, int* steps_taken);
/* Exactly n_steps ensemble steps (each pattern iterating at most n_steps times). */
int fresco_ensemble_lbfgs_steps(fresco_ensemble_lbfgs o, int n_steps);
/* x, g (ndof doubles) and per-pattern f, rms, iterations, evaluations and
 * whether the pattern is still iterating; any pointer may be NULL. */
int fresco_ensemble_lbfgs_state(fresco_ensemble_lbfgs o, double* x, double* g, double* f, double* rms, int* niter,
                                int* nfev, int* active);
void fresco_ensemble_lbfgs_destroy(fresco_ensemble_lbfgs o);

/* CheckOverlap(radii, boxv, use_cell_lists, ncellx_scale, method)
 * (fresco/distances/_check_overlap.pyx:29-110; check_overlap.hpp:24-130,
 * check_overlap_cell_lists.hpp:87-180): the hard-core overlap test on the
 * device, with cell lists whatever use_cell_lists says (the result does not
 * depend on it).  periodic: 1 for Distance.PERIODIC (minimum image in the box
 * boxv), 0 for Distance.CARTESIAN (boxv only gives ndim = 1, 2 or 3).  An
 * empty radius array raises, as the reference does. */
int fresco_overlap_create(const double* radii, int64_t n, const double* boxv, int ndim, int periodic,
                          fresco_overlap* out);
/* get_overlapping_particles(coords) (check_overlap.hpp:111-115) or, with
 * n_changed > 0, get_overlapping_particles_ca(coords, changed_atoms)
 * (:105-109): the particles i with |r_ij|^2 < (r_i + r_j)^2 for some j != i
 * (only pairs holding a changed atom with changed atoms).  x: ndof host
 * coordinates (ndof = n * ndim, else the reference's "illegal input" error);
 * out: room for n indices, written in ascending order (the reference's
 * unordered_set order is unspecified); *count: how many.  Synchronous. */
int fresco_overlap_find(fresco_overlap h, const double* x, int64_t ndof, const int64_t* changed, int64_t n_changed,
                        uint64_t* out, int64_t* count);
void fresco_overlap_destroy(fresco_overlap h);

/* PointPatternStatistics(coords, boxv, radius, rseed) (n_radii = 1;
 * point_pattern_statistics.hpp:36-111) and BatchPPS(coords, boxv, radii,
 * rseed) (batch_pointstats.hpp:29-150): number-variance window counts.
 * x: n_points * ndim host coordinates, copied; radii ascending.  Windows are
 * centred at the std::mt19937_64(rseed) stream's points, drawn as the
 * reference draws them. */
int fresco_window_stats_create(const double* x, int64_t n_points, int ndim, const double* boxv, const double* radii,
                               int n_radii, uint64_t seed, fresco_window_stats* out);
/* run(n): n more windows (point_pattern_statistics.hpp:66-70, batch_pointstats.hpp:73-125). */
int fresco_window_stats_run(fresco_window_stats h, int64_t n);
/* set_generator_seed(seed) (point_pattern_statistics.hpp:105-108). */
int fresco_window_stats_set_seed(fresco_window_stats h, uint64_t seed);
/* get_seed, and per radius get_mean / get_variance / get_count
 * (point_pattern_statistics.hpp:92-103); any pointer may be NULL. */
int fresco_window_stats_get(fresco_window_stats h, uint64_t* seed, double* mean, double* var, uint64_t* count);
void fresco_window_stats_destroy(fresco_window_stats h);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* FRESCO_B200_H */
