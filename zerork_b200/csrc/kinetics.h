// kinetics.h -- launchers for the fused FP64 rates + Jacobian kernel.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "devmech.h"

namespace zrk {

struct KinParams {
  double Tref;     // reference_temperature option (state y[S] = T / Tref)
  double mmf;      // min_mass_fraction option (Jacobian clamp)
  double lim;      // step_limiter option (same value for every step)
  double sqrt_ur;  // sqrt(DBL_EPSILON), the forward-difference scale
};

// Tile / CTA mapping: ts states per tile (8, 16 or 32), v states per thread,
// warps per CTA, and
// whether the per-tile workspace lives in global scratch (grid CTAs, each
// with its own slice) instead of shared memory.
struct LaunchCfg {
  int ts = 16;
  int v = 1;  // states per thread (1, 2 or 4); ts / v threads share one work item
  int warps = 8;
  bool global_ws = false;
  int grid = 0;
  bool stage = false;  // mechanism tables staged in each CTA's shared memory
  int minb = 1;        // resident CTAs per SM the kernel is compiled for (1 or 2)
};

// Species-major arrays x[item * ld + state]; ld >= n.
struct RatesJacArgs {
  int n = 0, ld = 0;
  const double *T = nullptr, *P = nullptr, *Y = nullptr;  // Y: [nsp][ld]
  double *wdot = nullptr;                                 // [nsp][ld]  (required)
  double *jac = nullptr;                                  // [nnz][ld]  (optional)
  double *ydot = nullptr;                                 // [nsp+1][ld] (optional)
  double *scratch = nullptr;                              // global workspace
  size_t scratch_bytes = 0;
};

// Rates from temperature and concentrations (rates_tc.cu): species-major
// C[nsp][ld], outputs net / create / destroy [nsp][ld] and rates of progress
// rop [nstep][ld] (any output may be null); lim_step: one limit per step
// (null: no limiter).
struct RatesTCArgs {
  int n = 0, ld = 0;
  const double *T = nullptr, *C = nullptr, *lim_step = nullptr;
  double *net = nullptr, *create = nullptr, *destroy = nullptr, *rop = nullptr;
};
size_t rates_tc_smem_bytes(const DevMech &m, int ts, int threads);
cudaError_t launch_rates_tc(const DevMech &m, const RatesTCArgs &a, cudaStream_t stream);

size_t rates_jac_ws_bytes(const DevMech &m, const LaunchCfg &cfg);
// Dynamic shared memory of a launch: the workspace (unless global) plus the
// staged tables (cfg.stage).
size_t rates_jac_smem_bytes(const DevMech &m, const LaunchCfg &cfg);
bool rates_jac_mapping_ok(const LaunchCfg &cfg);
cudaError_t launch_rates_jac(const DevMech &m, const RatesJacArgs &a, const KinParams &kp,
                             const LaunchCfg &cfg, cudaStream_t stream);

}  // namespace zrk
