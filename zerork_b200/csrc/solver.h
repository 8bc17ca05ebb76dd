// solver.h -- host driver of the batched reactor integration.
//
// Mirrors what ZeroRKReactorManager::SolveReactors does per call
// (applications/cfd_plugin/zerork_reactor_manager.cpp:835-1155): order the
// reactors by the previous call's cost (sort_reactors), integrate every
// reactor (constant volume or constant pressure, with optional DPDT, E_SRC
// and Y_SRC sources) for dt, write back T, P, mass fractions, cost (steps),
// time and temperature delta.  All reactors run on the GPU (no CPU
// fallback).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "devmech.h"
#include "integrator.h"
#include "mech.h"
#include "sparse_lu.h"

namespace zrk {

struct SolveOptions {
  double rtol = 1.0e-8, atol = 1.0e-20, max_dt = 0.05, nlscoef = 0.05;
  double eps_lin = 1.0e-3;  // Krylov tolerance factor (FP32 path)
  int max_steps = 5000, max_retries = 5;
  double retry_atol = 0.1, retry_rtol = 1.0;
  double Tref = 1.0, mmf = 1.0e-30, lim = 1.0e22;
  bool lu_fp32 = false;
  bool sort_reactors = true;
  int warps_per_cta = 0;  // 0 = automatic
  int method = 0;         // 0 automatic, 1 CTA dense block, 2 warp sparse LU, 3 the plain
                          // FP64 group path (integrator_group.h)
  int group_max = 1024;   // method 3: reactors per group (plugin option n_reactors_max)
  int threads = 0;        // CTA size of the dense method (0 = automatic)
  PredDev pred{};         // learned predictor (dense method only)
  double dT_ign = 0.0;    // delta_temperature_ignition (> 0: record ignition times)
  bool constant_pressure = false;  // plugin option constant_volume = 0
  bool always_solve_T = true;      // always_solve_temperature; false: reactors whose
                                   // input temperature delta is <= 0 keep T fixed
  bool stop_after_ignition = false;  // end each reactor's call at its ignition time
  bool abstol_dens = false;          // species absolute tolerances / molar density
};

// The plugin's per-step callback (zerork_callback_fn of zerork_cfd_plugin.h):
// called after every accepted step of every reactor, and once more at the
// first crossing of the ignition temperature, with the reactor's id
// (reactor_ids[k], or the reactor's index k where the reference passes its
// position in the cost-sorted order, zerork_reactor_manager.cpp:1105-1108),
// the reference's call counter, the time from the call's start, the time
// since the previous call, the state y = [Y, T/Tref] and its derivative; a
// nonzero return ends that reactor's call there (solver_cvode.cpp:247-262).
// Calls come reactor by reactor in index order after the batch integrated.
struct StepCallback {
  int (*fn)(int reactor_id, int steps, double time, double dt, const double *y, const double *dy,
            void *data) = nullptr;
  void *data = nullptr;
  const int *reactor_ids = nullptr;
};

struct SolveStatsTotals {
  long nsteps = 0, nrej = 0, nnewt = 0, njac = 0, nlu = 0, nrhs = 0, nkry = 0;
  int nfailed = 0;
  float kernel_ms = 0.f;
  int method = 0;
  // method 3: groups, steps and Newton iterations of all groups, kernel
  // launches and host synchronizations
  long groups = 0, group_steps = 0, group_newton = 0, launches = 0, syncs = 0;
  long group_status = 0;  // status of the first failed group (0: none)
};

class ReactorSolver {
 public:
  ReactorSolver(const std::string &mech, const std::string &therm);
  ~ReactorSolver();
  int nsp() const { return tables_.nsp; }
  const MechTables &tables() const { return tables_; }
  const LUSymbolic &lu() const { return lus_; }
  // Integrate n reactors (host arrays; mf reactor-major with stride >= nsp).
  // cost/gpu_time/temp_delta may be null.  Returns the number of failed
  // reactors (state left unchanged for those), or -1 on a CUDA error.
  // ysrc: optional mass-fraction sources [n][nsp] (1/s); t_ign: optional
  // ignition times [n] (when o.dT_ign > 0, written for the reactors that
  // integrated and reached T0 + dT_ign in this call; left as they were
  // otherwise);
  // dpdt, esrc: optional pressure rates (Pa/s) and energy sources (J/kg/s) [n].
  int solve(const SolveOptions &o, int n, double dt, double *T, double *P, double *mf,
            int stride, double *cost, double *gpu_time, double *temp_delta,
            double temp_threshold, std::vector<ReactorStats> *stats, SolveStatsTotals *tot,
            const double *ysrc = nullptr, double *t_ign = nullptr, const double *dpdt = nullptr,
            const double *esrc = nullptr, const StepCallback *cb = nullptr);
  std::string last_error;

 private:
  cudaError_t reserve(int n, bool fp32);
  cudaError_t solve_with_callback(int method, const IntegOpts &io, IntegArgs a, int dthreads,
                                  int dctas, int spill, int W, int ctas, bool rop_smem, int n,
                                  double dt, const StepCallback &cb);
  MechTables tables_;
  JacPattern pat_;
  LUSymbolic lus_;
  std::unique_ptr<DeviceMechanism> dm_;
  void *lu_blob_ = nullptr;
  LUDev lud_{};
  // device buffers
  int cap_ = 0;
  bool cap_fp32_ = false;
  double *dT_ = nullptr, *dP_ = nullptr, *dY_ = nullptr, *dv_ = nullptr, *dstate_ = nullptr;
  void *dlu_ = nullptr;
  ReactorStats *dstats_ = nullptr;
  int *dorder_ = nullptr, *dhead_ = nullptr;
  double *drop_ = nullptr;
  size_t drop_bytes_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  // pinned host staging (fixed addresses for the captured copies)
  double *hT_ = nullptr, *hP_ = nullptr, *hY_ = nullptr, *hsrc_ = nullptr, *hign_ = nullptr;
  double *dsrc_ = nullptr, *dign_ = nullptr;
  double *hde_ = nullptr, *dde_ = nullptr;  // [dpdt | esrc | temp_delta in], cap_ each
  int *horder_ = nullptr;
  ReactorStats *hstats_ = nullptr;
  // one CUDA graph per call configuration: H2D copies, queue reset, the
  // persistent integration kernel between two timing events, D2H copies
  cudaGraphExec_t graph_ = nullptr;
  // step-callback records (solve with a StepCallback)
  double *dcb_rec_ = nullptr;
  int *dcb_cnt_ = nullptr, *dcb_stop_ = nullptr, *dcb_order_ = nullptr;
  size_t dcb_bytes_ = 0;
  int dcb_n_ = 0;
  std::vector<unsigned char> graph_key_;
  // plain FP64 group path (method 3): per-reactor slots and partial sums
  double *dgrp_ = nullptr, *dpart_ = nullptr, *hpart_ = nullptr;
  size_t dgrp_bytes_ = 0;
  int part_cap_ = 0;
 public:
  long graph_launches = 0, graph_captures = 0;
};

}  // namespace zrk
