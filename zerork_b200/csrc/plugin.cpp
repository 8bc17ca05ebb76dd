// plugin.cpp -- zerork_reactor_* C ABI (include/zerork_cfd_plugin.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/zerork_b200.h"
#include "../../include/zerork_b200_predictor.h"
#include "../../include/zerork_cfd_plugin.h"
#include "mlp.h"
#include "solver.h"

struct zerork_handle_impl {
  std::map<std::string, int> iopt;
  std::map<std::string, double> dopt;
  std::map<std::string, std::string> sopt;
  std::unique_ptr<zrk::ReactorSolver> solver;
  std::string loaded_mech, loaded_therm;
  double *aux[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  std::vector<double> own_cost, own_gpu, own_ign, own_tdelta;
  zerork_callback_fn cb = nullptr;
  void *cb_data = nullptr;
  int *reactor_ids = nullptr;
  zrk::SolveStatsTotals last;
  std::string last_error;
  zrk::PredDev pred{};       // learned predictor (network owned by the caller)
  float *pred_norm = nullptr;  // device copy of the standardisation vectors
  ~zerork_handle_impl() { cudaFree(pred_norm); }
};

namespace {

// ZeroRKReactorManager constructor defaults (zerork_reactor_manager.cpp:49-101),
// plus the GPU integrator's own options ("lu_fp32", "gpu_warps_per_cta").
void set_defaults(zerork_handle_impl *h) {
  auto &I = h->iopt;
  auto &D = h->dopt;
  auto &S = h->sopt;
  S["mech_filename"] = "mech.dat";
  S["therm_filename"] = "therm.dat";
  S["reactor_timing_log_filename"] = "/dev/null";
  S["mechanism_parsing_log_filename"] = "/dev/null";
  I["verbosity"] = 4;
  I["sort_reactors"] = 1;
  I["load_balance"] = 0;
  I["load_balance_noise"] = 0;
  I["load_balance_mem"] = 1;
  I["reactor_weight_mult"] = 1;
  I["dump_reactors"] = 0;
  I["dump_failed_reactors"] = 0;
  I["output_performance_log"] = 1;
  I["max_steps"] = 5000;
  I["dense"] = 0;
  I["analytic"] = 1;
  I["iterative"] = 1;
  I["integrator"] = 0;
  I["abstol_dens"] = 0;
  I["cvode_num_retries"] = 5;
  D["rel_tol"] = 1.0e-8;
  D["abs_tol"] = 1.0e-20;
  D["eps_lin"] = 1.0e-3;
  D["nonlinear_convergence_coeff"] = 0.05;
  D["preconditioner_threshold"] = 1.0e-3;
  D["max_dt"] = 0.05;
  D["cvode_retry_absolute_tolerance_adjustment"] = 0.1;
  D["cvode_retry_relative_tolerance_adjustment"] = 1.0;
  I["constant_volume"] = 1;
  D["reference_temperature"] = 1.0;
  D["delta_temperature_ignition"] = 0.0;
  D["min_mass_fraction"] = 1.0e-30;
  I["always_solve_temperature"] = 1;
  D["solve_temperature_threshold"] = 2.0;
  D["step_limiter"] = 1.0e22;
  I["gpu"] = 1;
  I["initial_gpu_multiplier"] = 8;
  I["n_reactors_min"] = 128;
  I["n_reactors_max"] = 1024;
  I["lu_fp32"] = 0;
  I["gpu_warps_per_cta"] = 0;
  I["gpu_method"] = 0;
  I["gpu_threads"] = 0;
}

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n\"'");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n\"'");
  return s.substr(a, b - a + 1);
}

zerork_status_t ensure_mechanism(zerork_handle_impl *h) {
  const std::string &m = h->sopt["mech_filename"], &t = h->sopt["therm_filename"];
  if (h->solver && m == h->loaded_mech && t == h->loaded_therm) return ZERORK_STATUS_SUCCESS;
  h->solver.reset();
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    h->last_error = "no CUDA device";
    return ZERORK_STATUS_UNKNOWN_ERROR;
  }
  try {
    h->solver = std::make_unique<zrk::ReactorSolver>(m, t);
  } catch (const zrk::ParseError &e) {
    h->last_error = e.what();
    std::fprintf(stderr, "zerork_b200: mechanism parse failed: %s\n", e.what());
    return ZERORK_STATUS_FAILED_MECHANISM_PARSE;
  } catch (const std::exception &e) {
    h->last_error = e.what();
    return ZERORK_STATUS_UNKNOWN_ERROR;
  }
  h->loaded_mech = m;
  h->loaded_therm = t;
  return ZERORK_STATUS_SUCCESS;
}

}  // namespace

extern "C" {

zerork_handle zerork_reactor_init(void) {
  zerork_handle h = new (std::nothrow) zerork_handle_impl();
  if (h) set_defaults(h);
  return h;
}

zerork_status_t zerork_reactor_read_options_file(const char *options_filename, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!options_filename) return ZERORK_STATUS_INVALID_FILENAME;
  std::ifstream in(options_filename);
  if (!in) return ZERORK_STATUS_FAILED_OPTIONS_PARSE;
  // option file keys that differ from the option names
  const std::map<std::string, std::string> alias = {
      {"relative_tolerance", "rel_tol"},
      {"absolute_tolerance", "abs_tol"},
      {"reactor_timing_log", "reactor_timing_log_filename"},
      {"mechanism_parsing_log", "mechanism_parsing_log_filename"},
      {"mechanism_file", "mech_filename"},
      {"therm_file", "therm_filename"}};
  std::string line;
  while (std::getline(in, line)) {
    size_t c = line.find('#');
    if (c != std::string::npos) line = line.substr(0, c);
    size_t colon = line.find(':');
    if (colon == std::string::npos) {
      if (!trim(line).empty()) return ZERORK_STATUS_FAILED_OPTIONS_PARSE;
      continue;
    }
    std::string key = trim(line.substr(0, colon)), val = trim(line.substr(colon + 1));
    if (key.empty()) continue;
    auto al = alias.find(key);
    if (al != alias.end()) key = al->second;
    char *end = nullptr;
    if (h->iopt.count(key)) {
      long v = std::strtol(val.c_str(), &end, 10);
      if (!end || *end) {
        double dv = std::strtod(val.c_str(), &end);
        if (!end || *end) return ZERORK_STATUS_FAILED_OPTIONS_PARSE;
        v = (long)dv;
      }
      h->iopt[key] = (int)v;
    } else if (h->dopt.count(key)) {
      double v = std::strtod(val.c_str(), &end);
      if (!end || *end) return ZERORK_STATUS_FAILED_OPTIONS_PARSE;
      h->dopt[key] = v;
    } else {
      h->sopt[key] = val;
    }
  }
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_set_mechanism_files(const char *mech_file, const char *therm_file,
                                                   zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!mech_file) return ZERORK_STATUS_INVALID_FILENAME;
  h->sopt["mech_filename"] = mech_file;
  if (therm_file) h->sopt["therm_filename"] = therm_file;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_load_mechanism(zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  return ensure_mechanism(h);
}

// Solver options from the handle's option maps (names as the reference's).
static zrk::SolveOptions options_of(zerork_handle_impl *h) {
  auto &I = h->iopt;
  auto &D = h->dopt;
  zrk::SolveOptions o;
  o.rtol = D["rel_tol"];
  o.atol = D["abs_tol"];
  o.max_dt = D["max_dt"];
  o.nlscoef = D["nonlinear_convergence_coeff"];
  o.eps_lin = D["eps_lin"];
  o.max_steps = I["max_steps"];
  o.max_retries = I["cvode_num_retries"];
  o.retry_atol = D["cvode_retry_absolute_tolerance_adjustment"];
  o.retry_rtol = D["cvode_retry_relative_tolerance_adjustment"];
  o.Tref = D["reference_temperature"];
  o.mmf = D["min_mass_fraction"];
  o.lim = D["step_limiter"];
  o.lu_fp32 = I["lu_fp32"] != 0;
  o.sort_reactors = I["sort_reactors"] != 0;
  o.warps_per_cta = I["gpu_warps_per_cta"];
  o.method = I["gpu_method"];
  o.group_max = std::max(1, I["n_reactors_max"]);
  o.threads = I["gpu_threads"];
  o.pred = h->pred;
  o.dT_ign = D["delta_temperature_ignition"];
  o.constant_pressure = I["constant_volume"] == 0;  // zerork_reactor_manager.cpp:913-917
  o.always_solve_T = I["always_solve_temperature"] != 0;  // :1107-1113
  // solver_cvode.cpp:262 and reactor_nvector_serial.cpp:107-119; the
  // reference's defaults table has no stop_after_ignition entry (unset = 0)
  auto si = I.find("stop_after_ignition");
  o.stop_after_ignition = si != I.end() && si->second != 0;
  o.abstol_dens = I["abstol_dens"] != 0;
  return o;
}

zerork_status_t zerork_reactor_solve(const int n_cycle, const double time, const double dt,
                                     const int n_reactors, double *T, double *P, double *mf,
                                     zerork_handle h) {
  (void)n_cycle;
  (void)time;
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  zerork_status_t f = ensure_mechanism(h);
  if (f != ZERORK_STATUS_SUCCESS) return f;
  if (n_reactors <= 0) return ZERORK_STATUS_SUCCESS;
  if (!T || !P || !mf) return ZERORK_STATUS_INVALID_POINTER;
  auto &D = h->dopt;
  zrk::SolveOptions o = options_of(h);
  // aux fields owned by the handle when the caller gave none
  // (zerork_reactor_manager.cpp:502-519)
  const int n = n_reactors;
  double *cost = h->aux[ZERORK_FIELD_COST], *gpu = h->aux[ZERORK_FIELD_GPU];
  double *tdel = h->aux[ZERORK_FIELD_TEMPERATURE_DELTA], *ign = h->aux[ZERORK_FIELD_IGNITION_TIME];
  if (!cost) {
    h->own_cost.resize(n, 1.0);
    cost = h->own_cost.data();
  }
  if (!gpu) {
    h->own_gpu.resize(n, 0.0);
    gpu = h->own_gpu.data();
  }
  if (!tdel) {
    h->own_tdelta.resize(n, 0.0);
    tdel = h->own_tdelta.data();
  }
  if (!ign) {
    h->own_ign.assign(n, -1.0);
    ign = h->own_ign.data();
  }
  const int ns = h->solver->nsp();
  // aux sources (zerork_reactor_manager.cpp:1092-1104): DPDT, E_SRC and
  // Y_SRC per reactor where the caller set them
  // the per-step callback and reactor ids (solver_cvode.cpp:247-257,
  // zerork_reactor_manager.cpp:1105-1108)
  zrk::StepCallback cbs;
  cbs.fn = h->cb;
  cbs.data = h->cb_data;
  cbs.reactor_ids = h->reactor_ids;
  int nfail = h->solver->solve(o, n, dt, T, P, mf, ns, cost, gpu, tdel,
                               D["solve_temperature_threshold"], nullptr, &h->last,
                               h->aux[ZERORK_FIELD_Y_SRC], ign, h->aux[ZERORK_FIELD_DPDT],
                               h->aux[ZERORK_FIELD_E_SRC], h->cb ? &cbs : nullptr);
  if (nfail < 0) {
    h->last_error = h->solver->last_error;
    std::fprintf(stderr, "zerork_b200: %s\n", h->last_error.c_str());
    return ZERORK_STATUS_UNKNOWN_ERROR;
  }
  return nfail > 0 ? ZERORK_STATUS_FAILED_SOLVE : ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_set_aux_field_pointer(zerork_field_t ft, double *field_pointer,
                                                     zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!field_pointer) return ZERORK_STATUS_INVALID_POINTER;
  if ((int)ft < 0 || (int)ft > ZERORK_FIELD_TEMPERATURE_DELTA) return ZERORK_STATUS_INVALID_FIELD_NAME;
  h->aux[ft] = field_pointer;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_set_int_option(const char *name, int v, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!name) return ZERORK_STATUS_INVALID_POINTER;
  h->iopt[name] = v;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_set_double_option(const char *name, double v, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!name) return ZERORK_STATUS_INVALID_POINTER;
  h->dopt[name] = v;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_set_string_option(const char *name, const char *v, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!name || !v) return ZERORK_STATUS_INVALID_POINTER;
  h->sopt[name] = v;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_get_int_option(const char *name, int *v, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!name || !v) return ZERORK_STATUS_INVALID_POINTER;
  auto it = h->iopt.find(name);
  if (it == h->iopt.end()) return ZERORK_STATUS_OPTION_NOT_DEFINED;
  *v = it->second;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_get_double_option(const char *name, double *v, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!name || !v) return ZERORK_STATUS_INVALID_POINTER;
  auto it = h->dopt.find(name);
  if (it == h->dopt.end()) return ZERORK_STATUS_OPTION_NOT_DEFINED;
  *v = it->second;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_get_string_option(const char *name, char **v, int len,
                                                 zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!name || !v || !*v) return ZERORK_STATUS_INVALID_POINTER;
  auto it = h->sopt.find(name);
  if (it == h->sopt.end()) return ZERORK_STATUS_OPTION_NOT_DEFINED;
  std::strncpy(*v, it->second.c_str(), len);
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_set_callback_fn(zerork_callback_fn fn, void *data, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!fn) return ZERORK_STATUS_INVALID_POINTER;
  h->cb = fn;
  h->cb_data = data;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_set_reactor_ids(int *ids, zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  if (!ids) return ZERORK_STATUS_INVALID_POINTER;
  h->reactor_ids = ids;
  return ZERORK_STATUS_SUCCESS;
}

zerork_status_t zerork_reactor_free(zerork_handle h) {
  if (!h) return ZERORK_STATUS_INVALID_HANDLE;
  delete h;
  return ZERORK_STATUS_SUCCESS;
}

// Totals of the last solve call: steps, rejected steps, Newton iterations,
// Jacobians, factorizations, right-hand sides, failed reactors; kernel ms.
int zrk_plugin_krylov_iterations(zerork_handle h, long *iterations) {
  if (!h) return ZRK_ERR_INVALID_HANDLE;
  if (iterations) *iterations = h->last.nkry;
  return ZRK_OK;
}

int zrk_plugin_num_species(zerork_handle h) {
  return (h && h->solver) ? h->solver->nsp() : -1;
}

int zrk_plugin_group_stats(zerork_handle h, long *out6) {
  if (!h) return ZRK_ERR_INVALID_HANDLE;
  if (!out6) return ZRK_ERR_INVALID_POINTER;
  out6[0] = h->last.groups;
  out6[1] = h->last.group_steps;
  out6[2] = h->last.group_newton;
  out6[3] = h->last.launches;
  out6[4] = h->last.syncs;
  out6[5] = h->last.group_status;
  return ZRK_OK;
}

int zrk_plugin_graph_stats(zerork_handle h, long *captures, long *launches) {
  if (!h) return ZRK_ERR_INVALID_HANDLE;
  if (captures) *captures = h->solver ? h->solver->graph_captures : 0;
  if (launches) *launches = h->solver ? h->solver->graph_launches : 0;
  return ZRK_OK;
}

// Integrator launch-mapping autotuner: the CTA size of the dense-block path
// (128, 256, 512 threads) or the warps per CTA of the sparse path (4, 8, 12),
// each timed on the same sample of the caller's reactors over a short
// interval; the fastest becomes the handle's gpu_threads / gpu_warps_per_cta.
int zrk_plugin_autotune(zerork_handle h, int n, double dt, const double *T, const double *P,
                        const double *mf, int *best, float *best_ms) {
  if (!h) return ZRK_ERR_INVALID_HANDLE;
  if (!T || !P || !mf) return ZRK_ERR_INVALID_POINTER;
  if (n <= 0 || !(dt > 0.0)) return ZRK_ERR_INVALID_ARGUMENT;
  if (ensure_mechanism(h) != ZERORK_STATUS_SUCCESS) return ZRK_ERR_PARSE;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ns = h->solver->nsp();
  const int m = std::min(n, 2 * sms);
  const double dtt = dt / 20.0;
  zrk::SolveOptions o = options_of(h);
  int method = o.method;
  // probe which path runs: the dense path sets gpu_threads, the sparse path warps
  std::vector<double> T1(T, T + m), P1(P, P + m), Y1(mf, mf + (size_t)m * ns);
  zrk::SolveStatsTotals tot;
  if (h->solver->solve(o, m, dtt, T1.data(), P1.data(), Y1.data(), ns, nullptr, nullptr, nullptr, 2.0,
                       nullptr, &tot) < 0)
    return ZRK_ERR_CUDA;
  method = tot.method;
  const std::vector<int> cand = method == 1 ? std::vector<int>{128, 256, 512} : std::vector<int>{4, 8, 12};
  float bms = 1e30f;
  int bc = cand.back();
  for (int c : cand) {
    zrk::SolveOptions oc = o;
    if (method == 1) oc.threads = c;
    else oc.warps_per_cta = c;
    std::copy(T, T + m, T1.begin());
    std::copy(P, P + m, P1.begin());
    std::copy(mf, mf + (size_t)m * ns, Y1.begin());
    if (h->solver->solve(oc, m, dtt, T1.data(), P1.data(), Y1.data(), ns, nullptr, nullptr, nullptr, 2.0,
                         nullptr, &tot) < 0)
      continue;
    if (tot.kernel_ms < bms) {
      bms = tot.kernel_ms;
      bc = c;
    }
  }
  h->iopt[method == 1 ? "gpu_threads" : "gpu_warps_per_cta"] = bc;
  if (best) *best = bc;
  if (best_ms) *best_ms = bms;
  return ZRK_OK;
}

int zrk_plugin_set_predictor(zerork_handle h, zrk_mlp_t net, const float *x_mu, const float *x_sd,
                             const float *t_mu, const float *t_sd) {
  if (!h) return ZRK_ERR_INVALID_HANDLE;
  if (!net) {
    h->pred.enabled = 0;
    return ZRK_OK;
  }
  if (!x_mu || !x_sd || !t_mu || !t_sd) return ZRK_ERR_INVALID_POINTER;
  if (ensure_mechanism(h) != ZERORK_STATUS_SUCCESS) return ZRK_ERR_PARSE;
  const zrk::MlpDev d = reinterpret_cast<zrk::Mlp *>(net)->device_view();
  const int nsp = h->solver->nsp();
  if (d.n_in != nsp + 3 || d.n_out != nsp + 1) {
    h->last_error = "predictor sizes must be nsp + 3 inputs and nsp + 1 outputs";
    return ZRK_ERR_INVALID_ARGUMENT;
  }
  for (int l = 0; l <= d.layers; ++l)
    if (d.dims[l] > 256) {
      h->last_error = "predictor layers wider than 256 are not supported by the integrator";
      return ZRK_ERR_INVALID_ARGUMENT;
    }
  const size_t ni = d.n_in, no = d.n_out;
  std::vector<float> buf;
  buf.insert(buf.end(), x_mu, x_mu + ni);
  buf.insert(buf.end(), x_sd, x_sd + ni);
  buf.insert(buf.end(), t_mu, t_mu + no);
  buf.insert(buf.end(), t_sd, t_sd + no);
  cudaFree(h->pred_norm);
  h->pred_norm = nullptr;
  if (cudaMalloc(&h->pred_norm, buf.size() * sizeof(float)) != cudaSuccess ||
      cudaMemcpy(h->pred_norm, buf.data(), buf.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    return ZRK_ERR_CUDA;
  h->pred.net = d;
  h->pred.x_mu = h->pred_norm;
  h->pred.x_sd = h->pred_norm + ni;
  h->pred.t_mu = h->pred_norm + 2 * ni;
  h->pred.t_sd = h->pred_norm + 2 * ni + no;
  h->pred.enabled = 1;
  return ZRK_OK;
}

int zrk_plugin_last_stats(zerork_handle h, long *totals7, float *kernel_ms) {
  if (!h) return ZRK_ERR_INVALID_HANDLE;
  if (totals7) {
    totals7[0] = h->last.nsteps;
    totals7[1] = h->last.nrej;
    totals7[2] = h->last.nnewt;
    totals7[3] = h->last.njac;
    totals7[4] = h->last.nlu;
    totals7[5] = h->last.nrhs;
    totals7[6] = h->last.nfailed;
  }
  if (kernel_ms) *kernel_ms = h->last.kernel_ms;
  return ZRK_OK;
}

}  // extern "C"
