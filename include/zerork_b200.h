/*
 * zerork_b200.h -- C ABI of the sm_100a mechanism kernels (mechanism level).
 *
 * Plain pointers and sizes only.  Device arrays are species-major
 * (structure of arrays): x[item * ld + state], ld >= n, the layout of
 * zerork::mechanism_cuda's multi-reactor entry points
 * (src/zerork/mechanism_cuda.h:19-45, C[j * nReactors + k]).
 * Every function returns 0 on success and a nonzero zerork_b200 error code
 * otherwise; zrk_last_error() gives the message of the calling thread.
 */
#ifndef ZERORK_B200_H
#define ZERORK_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zrk_mech_impl *zrk_mech_t;

enum {
  ZRK_OK = 0,
  ZRK_ERR_INVALID_HANDLE = 1,
  ZRK_ERR_INVALID_POINTER = 2,
  ZRK_ERR_PARSE = 3,
  ZRK_ERR_CUDA = 4,
  ZRK_ERR_INVALID_ARGUMENT = 5,
  ZRK_ERR_NO_DEVICE = 6
};

/* Last error message of the calling thread (never NULL). */
const char *zrk_last_error(void);

/* Parse a CHEMKIN mechanism + thermo file pair and upload the tables to the
 * current CUDA device.  Replaces zerork::mechanism::mechanism(mech, therm,
 * log) (src/zerork/mechanism.h:23-27) plus mechanism_cuda's table upload
 * (src/zerork/mechanism_cuda.h:12-17).  Errors: ZRK_ERR_PARSE (unsupported
 * or malformed input), ZRK_ERR_NO_DEVICE, ZRK_ERR_CUDA. */
int zrk_mech_create(const char *mech_file, const char *therm_file, zrk_mech_t *out);
int zrk_mech_free(zrk_mech_t m);

/* Parse only (no device upload): the tables and Jacobian pattern can be
 * inspected, kernel entry points return ZRK_ERR_NO_DEVICE. */
int zrk_mech_parse(const char *mech_file, const char *therm_file, zrk_mech_t *out);

/* Sizes: getNumSpecies/getNumReactions/getNumSteps (mechanism.h:30-34) and
 * the Jacobian nonzero count of the (nsp+1)^2 reactor Jacobian
 * (applications/cfd_plugin/reactor_nvector_serial.cpp:214-232). */
int zrk_mech_sizes(zrk_mech_t m, int *nsp, int *nrxn, int *nstep, int *nnz);

/* Export one mechanism table by name (e.g. "mw", "arr_lnA", "reac_spc"),
 * the tables zerork::rate_const / info_net build internally
 * (src/zerork/rate_const.h:98-170).  *count receives the element count; data
 * is copied when out != NULL and capacity >= count.  is_double says whether
 * elements are double (1) or int32 (0). */
int zrk_mech_table(zrk_mech_t m, const char *name, void *out, long capacity, long *count,
                   int *is_double);

/* Species name (getSpeciesName, mechanism.h:55). */
const char *zrk_mech_species_name(zrk_mech_t m, int idx);

/* Fixed Jacobian pattern, compressed column over nsp+1 variables:
 * col_ptr[nsp+2], row_idx[nnz]; SetupSparseJacobianArrays
 * (applications/cfd_plugin/reactor_nvector_serial.cpp:122-281). */
int zrk_mech_jac_pattern(zrk_mech_t m, int *col_ptr, int *row_idx);

/* Options used by the kernels (defaults as the cfd_plugin,
 * zerork_reactor_manager.cpp:49-101): "reference_temperature" (1.0),
 * "min_mass_fraction" (1e-30), "step_limiter" (1e22). */
int zrk_mech_set_double_option(zrk_mech_t m, const char *name, double value);
int zrk_mech_get_double_option(zrk_mech_t m, const char *name, double *value);

/* Tile mapping of the rate kernel: ts states per tile (8/16/32), v states
 * per thread (1/2/4), warps per CTA (1..16; 32 with v = 1); flags bit 0
 * (ZRK_LAUNCH_GLOBAL_WS) puts the per-tile workspace in global scratch (grid
 * CTAs; 0 = one CTA per tile), bit 1 (ZRK_LAUNCH_STAGE_TABLES) copies the
 * mechanism tables the kernel reads into each CTA's shared memory beside
 * the workspace (rejected when the two do not fit), bit 2
 * (ZRK_LAUNCH_TWO_CTAS, up to 8 warps and 16 states per tile, tables not
 * staged) compiles the kernel for two resident CTAs per SM (at most 128
 * registers per thread).  ts = 0 restores the default mapping. */
#define ZRK_LAUNCH_GLOBAL_WS 1
#define ZRK_LAUNCH_STAGE_TABLES 2
#define ZRK_LAUNCH_TWO_CTAS 4
int zrk_mech_set_launch(zrk_mech_t m, int ts, int v, int warps, int flags, int grid);
int zrk_mech_get_launch(zrk_mech_t m, int *ts, int *v, int *warps, int *flags, int *grid);

/* Autotuner: times every valid (ts, v, warps) mapping on the caller's sample
 * (device arrays as for zrk_rates_jac_dev, outputs overwritten) and keeps the
 * fastest for later calls.  *best_ms (may be NULL) receives its time.  No
 * counterpart in the reference, whose launch shapes are fixed constants
 * (src/zerork/rate_const_cuda.cpp:583-629, "tuned on P100"). */
int zrk_mech_autotune(zrk_mech_t m, int n, int ld, const double *T, const double *P,
                      const double *Y, double *wdot, double *jac, void *stream, float *best_ms);

/* Net production rates + reactor Jacobian at independent (T, P, Y) states,
 * all device pointers on the current device, species-major with leading
 * dimension ld.  Per state: inverse density from (T, P, Y); y = [Y, T/Tref];
 * wdot = net production rates (getReactionRatesLimiter, mechanism.h:143);
 * jac = SetupJacobianSparse values (reactor_nvector_serial.cpp:610-771)
 * in compressed-column order, [nnz][ld]; ydot = GetTimeDerivative
 * (reactor_constant_volume_cpu.cpp:64-128), [nsp+1][ld].  jac and ydot may
 * be NULL.  stream is a cudaStream_t (NULL = legacy default stream).  The
 * call is asynchronous; scratch needed by the global-workspace mapping is
 * allocated by the library on first use and shared by all calls on the
 * handle, so with that mapping calls on one handle must not overlap on the
 * GPU (use one stream or one handle per stream). */
int zrk_rates_jac_dev(zrk_mech_t m, int n, int ld, const double *T, const double *P,
                      const double *Y, double *wdot, double *jac, double *ydot, void *stream);

/* No counterpart in the reference.  zrk_rates_jac_dev for callers that
 * cannot have the library allocate device memory during a call: codes whose
 * own pool allocator owns the GPU's memory after start-up, code running
 * where a cudaMalloc would synchronize the device, or hosts whose device
 * footprint must stay fixed after set-up.  Same arguments, kernel and
 * results as zrk_rates_jac_dev, with the kernel's global-workspace mapping
 * (the handle's tile size, states per thread and warps) always used and its
 * workspace taken from a fixed array of ZRK_NOALLOC_SCRATCH_BYTES inside the
 * library, which every device that loads the library holds until the
 * process exits; the grid is cut to the tiles that fit in it.  Returns
 * ZRK_ERR_INVALID_ARGUMENT, with the sizes in zrk_last_error(), when one
 * tile's workspace alone is larger than the array.  The first call on a
 * device looks the array's device address up (cudaGetSymbolAddress) and
 * caches it for the life of the process: make that first call before
 * capturing any stream, and do not call this entry point on a device after
 * a cudaDeviceReset of it (the cached address would be stale).  The kernel
 * writes every workspace word before reading it, so the array needs no
 * clearing, but all calls in the process share it: calls that overlap on
 * the GPU (different streams or handles without ordering between them)
 * race and give wrong results. */
#define ZRK_NOALLOC_SCRATCH_BYTES (8u << 20)
int zrk_rates_jac_dev_noalloc(zrk_mech_t m, int n, int ld, const double *T, const double *P,
                              const double *Y, double *wdot, double *jac, double *ydot,
                              void *stream);

/* Rates from temperature and concentrations for n independent states:
 * mechanism_cuda::getReactionRates_CUDA_mr_dev and
 * getReactionRatesLimiter_CUDA_mr_dev (src/zerork/mechanism_cuda.h:19-26,
 * perf_net.cpp:126-274 per state).  Device arrays, species-major with
 * leading dimension ld: T[ld], C[nsp][ld] (kmol/m^3); outputs net, create,
 * destroy [nsp][ld] and rop [nstep][ld] (rates of progress per step); any
 * output may be NULL.  step_limiter: one limit per step [nstep] (a step is
 * limited as K L / (L + K) when 0 < L < 1e300), or NULL for the unlimited
 * rates of getReactionRates.  T is used as given; PLOG reactions see the
 * pressure Csum Ru T.  Asynchronous on stream. */
int zrk_rates_tc_dev(zrk_mech_t m, int n, int ld, const double *T, const double *C,
                     const double *step_limiter, double *net, double *create, double *destroy,
                     double *rop, void *stream);

/* The same with host arrays (species-major, ld = n; for one state simply
 * C[nsp], net[nsp], rop[nstep]): the host-side mechanism::getReactionRates /
 * getNetReactionRates / getReactionRatesLimiter (src/zerork/mechanism.h:
 * 114-143).  Copies in, computes on the GPU, copies out, synchronizes. */
int zrk_rates_tc_host(zrk_mech_t m, int n, const double *T, const double *C,
                      const double *step_limiter, double *net, double *create, double *destroy,
                      double *rop);

/* Same with host buffers (species-major, ld = n): copies in, computes,
 * copies out, synchronizes.  Host buffers may be pageable or pinned. */
int zrk_rates_jac_host(zrk_mech_t m, int n, const double *T, const double *P, const double *Y,
                       double *wdot, double *jac);

/* Totals of the last zerork_reactor_solve call on a plugin handle
 * (struct zerork_handle_impl *, include/zerork_cfd_plugin.h): totals7 =
 * {steps, rejected steps, Newton iterations, Jacobians, factorizations,
 * right-hand sides, failed reactors}; kernel_ms = integration kernel time.
 * No counterpart in the reference beyond its per-solve performance log
 * (zerork_reactor_manager.cpp:1285-1330). */
struct zerork_handle_impl;
int zrk_plugin_last_stats(struct zerork_handle_impl *h, long *totals7, float *kernel_ms);

/* Krylov iterations of the last zerork_reactor_solve call (the FP32 path's
 * preconditioned FP64 GMRES; 0 on the FP64 path).  No counterpart in the
 * reference beyond CVODE's linear-iteration counter. */
int zrk_plugin_krylov_iterations(struct zerork_handle_impl *h, long *iterations);

/* Counters of the last solve on the plain FP64 group path (option
 * gpu_method = 3, one BDF integration per group of n_reactors_max reactors
 * with a shared step size, as the reference GPU path integrates a batch with
 * one CVODE instance, zerork_reactor_manager.cpp:909-1054): out6 = {groups,
 * steps summed over the groups, Newton iterations summed over the groups,
 * kernel launches, host synchronizations, the status of the first group that
 * failed (0: none; the batched integrators' negative codes)}; zeros after a
 * solve on another method.  No counterpart in the reference. */
int zrk_plugin_group_stats(struct zerork_handle_impl *h, long *out6);

/* Species count of the handle's loaded mechanism (the step callback's y and
 * dy hold nsp + 1 entries: mass fractions, then T / Tref), or -1 before
 * zerork_reactor_load_mechanism.  No counterpart in the reference. */
int zrk_plugin_num_species(struct zerork_handle_impl *h);

/* Every zerork_reactor_solve call runs as one CUDA graph (copies in, work
 * queue reset, the persistent integration kernel, copies out), captured when
 * the call's configuration (reactor count, launch mapping, options, dt)
 * changes and replayed otherwise.  Counts of captures and launches so far.
 * No counterpart in the reference. */
int zrk_plugin_graph_stats(struct zerork_handle_impl *h, long *captures, long *launches);

/* Integrator launch-mapping autotuner: times the dense path's CTA sizes
 * (128/256/512 threads) or the sparse path's warps per CTA (4/8/12) on a
 * sample of the given reactors (at most 2 per SM) over dt / 20, keeps the
 * fastest as the handle's gpu_threads / gpu_warps_per_cta option and
 * returns it with its kernel time.  The inputs are not modified.  No
 * counterpart in the reference (its GPU path has fixed launch sizes). */
int zrk_plugin_autotune(struct zerork_handle_impl *h, int n, double dt, const double *T,
                        const double *P, const double *mass_fractions, int *best, float *best_ms);

#ifdef __cplusplus
}
#endif
#endif
