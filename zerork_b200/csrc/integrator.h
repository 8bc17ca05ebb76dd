// integrator.h -- batched stiff reactor integration on sm_100a.
//
// One warp integrates one reactor (constant volume, or constant pressure
// with IntegOpts.cp) at a time with a
// variable-order BDF (orders 1-5, quasi-constant step size, Shampine &
// Reichelt 1997) and a modified Newton iteration with CVODE's convergence
// test (Hindmarsh et al., ACM TOMS 2005), the Newton matrix I - cJ built from
// the reactor Jacobian of reactor_nvector_serial.cpp:610-771 and factored by
// the warp over the fixed symbolic pattern (sparse_lu.h).  Warps take
// reactors from a work queue until it is empty: one persistent launch per
// solve call, each reactor with its own step size, order and Jacobian age.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "devmech.h"
#include "mlp.h"
#include "kinetics.h"

namespace zrk {

constexpr int kMaxOrder = 5;
// Per-step failure limits, CVODE's defaults (the plugin sets neither
// CVodeSetMaxErrTestFails nor CVodeSetMaxConvFails, solver_cvode.cpp:51-212):
// the 7th error-test failure or the 10th convergence failure (after a fresh
// Jacobian) within one step fails the attempt, which then goes to the
// plugin's retry loop.
constexpr int kMaxErrTestFails = 7;
constexpr int kMaxConvFails = 10;
// From the 4th error-test failure within a step on, CVODE's rule (user
// guide, sec. 2.1): the order drops by one and the step to a tenth; at
// order 1 the first difference is reloaded from f at the last accepted state.
constexpr int kErrFailsBeforeCut = 3;
constexpr double kEtaMinErrFail = 0.1;

struct LUDev {
  int n, nnz;
  const int *col_ptr, *row_idx, *diag;  // permuted CSC of L+U
  const int *iperm;                     // original variable -> permuted
  const int *jac_to_lu;                 // Jacobian nonzero -> LU storage index
  const int *diag_of_orig;              // original variable -> LU diagonal index
};

// Learned BDF predictor attached to the dense integrator: the network
// (mlp.h) and the standardisation of its inputs and targets.
struct PredDev {
  MlpDev net;
  const float *x_mu = nullptr, *x_sd = nullptr, *t_mu = nullptr, *t_sd = nullptr;
  int enabled = 0;
  int reserved = 0;  // no implicit padding: the struct's bytes key captured graphs
};

struct IntegOpts {
  double rtol, atol, max_dt, nlscoef;
  int max_steps, max_retries;
  double retry_atol_factor, retry_rtol_factor;
  double Tref, mmf, lim, sqrt_ur;
  int lu_fp32;  // factor and apply the Newton matrix in FP32
  int cp;       // 1: constant-pressure reactor (plugin option constant_volume = 0)
  int always_T; // always_solve_temperature: 0 = integrate at fixed temperature the
                // reactors whose input temperature delta is <= 0
  double eps_lin;  // Krylov tolerance: eps_lin * nlscoef / error constant (WRMS)
  PredDev pred;    // learned predictor (dense integrator only; enabled = 0: off)
  double dT_ign;   // delta_temperature_ignition: > 0 records when T reaches T0 + dT_ign
  int stop_ign;    // stop_after_ignition: the call ends at the crossing
                   // (solver_cvode.cpp:259-263); its state is interpolated
                   // linearly between the two accepted steps around it
  int abstol_dens; // absolute tolerance of species k scaled by 1 / molar density
                   // (reactor_nvector_serial.cpp:107-119)
};

// Per-reactor statistics written by the kernel.
struct ReactorStats {
  int nsteps, nrej, nnewt, njac, nlu, nrhs, status, retries;
  int nkry;  // Krylov iterations (FP32 path)
  int pad;
};

// Per-step records for the plugin's step callback
// (zerork_reactor_set_callback_fn; solver_cvode.cpp:247-257 calls it after
// every successful CVode call with the state and the interpolant's
// derivative).  With rec set, each accepted step of the reactor appends one
// record of 3 + 2n doubles {t from the call's start, t - previous record's t,
// the reference's call counter, y[n], dy/dt[n]}, up to cap records; cnt
// counts every record, also past the cap.  The first crossing of the
// ignition temperature adds a record at the crossing before the step's own,
// as CVode's root return does.  stop > 0 ends the reactor's call at its
// stop-th record, with that record's state.
struct CbCtx {
  double *rec;
  int cap, stop;
  int cnt, ncalls;
  double tprev;
};

#ifdef __CUDACC__
// Appends one callback record at x = (t_rec - t) / h in [-1, 0] of the step
// just accepted (x = 0: the step itself): y and y' of the backward-difference
// interpolant sum_k D_k prod_{j<k} (x + j) / (j + 1) through the last q + 1
// steps, or, with prev set, y = prev + wprev (D_0 - prev) (the state
// stop_after_ignition gives the crossing).  Threads i0, i0 + di, ... share the
// entries.  Returns true when this record ends the call; then ystop (all n
// entries) holds the record's y.
__device__ inline bool cb_record(CbCtx &cb, const double *D, const double *prev, int n, int q,
                                 double h, double x, double wprev, double tabs, double *ystop,
                                 int i0, int di) {
  cb.ncalls++;
  const bool stop = cb.stop > 0 && cb.cnt + 1 >= cb.stop;
  double *e = cb.cnt < cb.cap ? cb.rec + (size_t)cb.cnt * (3 + 2 * n) : nullptr;
  if (e && i0 == 0) {
    e[0] = tabs;
    e[1] = tabs - cb.tprev;
    e[2] = (double)cb.ncalls;
  }
  if (e || stop) {
    for (int i = i0; i < n; i += di) {
      double c = 1.0, dc = 0.0, y = D[i], yd = 0.0;
      for (int k = 1; k <= q; ++k) {
        dc = (dc * (x + k - 1) + c) / k;
        c = c * (x + k - 1) / k;
        y += D[k * n + i] * c;
        yd += D[k * n + i] * dc;
      }
      if (prev) y = prev[i] + wprev * (D[i] - prev[i]);
      if (e) {
        e[3 + i] = y;
        e[3 + n + i] = yd / h;
      }
      if (stop) ystop[i] = y;
    }
  }
  cb.cnt++;
  cb.tprev = tabs;
  return stop;
}
#endif

struct IntegArgs {
  int n_reactors;
  const int *order;         // queue order (reactor indices), may be null
  int *queue_head;          // device counter, zero before launch
  double dt;
  double *T, *P, *Y;        // in/out, Y reactor-major [n_reactors][nsp]
  double *v;                // inverse densities (filled by the kernel)
  double *state;            // per-reactor workspace, state_stride doubles each
  long state_stride;
  void *lu;                 // per-reactor LU values (double or float), lu_stride elements
  long lu_stride;
  ReactorStats *stats;
  double *rop_scratch;      // optional global ROP rows (one per warp slot)
  const double *ysrc;       // optional mass-fraction sources [n_reactors][nsp] (1/s)
  double *t_ign;            // optional ignition times [n_reactors] (-1: not reached)
  const double *dpdt;       // optional pressure rates [n_reactors] (Pa/s)
  const double *esrc;       // optional energy sources [n_reactors] (J/kg/s)
  const double *tdel_in;    // previous temperature deltas [n_reactors] (read when !always_T)
  // step-callback records (CbCtx): cb_cap records of 3 + 2 (nsp + 1) doubles
  // per work-queue position (the reactor order[i] writes slot i), cb_cnt
  // [reactor] step counts, cb_stop [reactor] (may be null) steps after which
  // a reactor's call ends (0: none); all null when no callback is set
  double *cb_rec;
  int cb_cap;
  int *cb_cnt;
  const int *cb_stop;
};

size_t integ_smem_per_warp(const DevMech &m, const LUDev &lu, bool rop_in_smem);
// CTA-per-reactor dense-block integrator (integrator_dense.cu); IntegArgs.state
// holds the per-reactor Jacobian (state_stride = Jacobian nonzeros).
// spill: bit 1 puts rates of progress, bit 2 the BDF differences, in a global
// slice of IntegArgs.rop_scratch per CTA (dense_spill_doubles each); bit 4
// keeps the reactor Jacobian in shared memory instead of IntegArgs.state.
constexpr int kDenseMaxN = 256;  // dense-block integrator: n = nsp + 1 <= 256
size_t dense_smem_bytes(const DevMech &m, bool fp32, int *lda_out, int spill);
size_t dense_spill_doubles(const DevMech &m);
cudaError_t launch_integrate_dense(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                   int threads, int ctas, int spill, cudaStream_t stream);
long integ_state_doubles(const DevMech &m, const LUDev &lu);
cudaError_t launch_integrate(const DevMech &m, const LUDev &lu, const IntegOpts &o,
                             const IntegArgs &a, int warps_per_cta, int ctas, bool rop_in_smem,
                             cudaStream_t stream);

}  // namespace zrk
