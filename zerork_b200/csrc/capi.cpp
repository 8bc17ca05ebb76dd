// capi.cpp -- extern "C" entry points of include/zerork_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/zerork_b200.h"
#include "capi_internal.h"
#include "devmech.h"
#include "kinetics.h"
#include "mech.h"

namespace zrk {

thread_local std::string g_last_error;

int set_error(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char *what) {
  return set_error(ZRK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

LaunchCfg default_launch(const DevMech &m) {
  // Largest tile whose workspace fits in shared memory at 8 warps per CTA,
  // two states per thread; the autotuner (zrk_mech_autotune) refines this.
  const size_t kMaxSmem = 227 * 1024;
  for (int ts : {16, 8}) {
    LaunchCfg c;
    c.ts = ts;
    c.v = 2;
    c.warps = 8;
    if (rates_jac_ws_bytes(m, c) <= kMaxSmem) return c;
  }
  LaunchCfg c;
  c.ts = 16;
  c.v = 2;
  c.warps = 8;
  c.global_ws = true;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  c.grid = 4 * sms;
  return c;
}

MechHandle::~MechHandle() {
  if (scratch) cudaFree(scratch);
  if (pipe) cudaFree(pipe);
  for (auto &s : pipe_stream)
    if (s) cudaStreamDestroy(s);
  for (void *p : host_bufs) cudaFree(p);
}

cudaError_t MechHandle::ensure_pipe(size_t bytes) {
  cudaError_t e;
  for (auto &s : pipe_stream)
    if (!s && (e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) return e;
  if (pipe_bytes >= bytes) return cudaSuccess;
  if (pipe) cudaFree(pipe);
  pipe = nullptr;
  pipe_bytes = 0;
  e = cudaMalloc(&pipe, bytes);
  if (e == cudaSuccess) pipe_bytes = bytes;
  return e;
}

cudaError_t MechHandle::ensure_scratch(size_t bytes) {
  if (scratch_bytes >= bytes) return cudaSuccess;
  if (scratch) cudaFree(scratch);
  scratch = nullptr;
  scratch_bytes = 0;
  cudaError_t e = cudaMalloc(&scratch, bytes);
  if (e == cudaSuccess) scratch_bytes = bytes;
  return e;
}

}  // namespace zrk

using namespace zrk;

extern "C" {

const char *zrk_last_error(void) { return g_last_error.c_str(); }

static int parse_into(const char *mech_file, const char *therm_file, MechHandle *h) {
  try {
    h->tables = load_chemkin(mech_file, therm_file);
    h->pattern = build_jac_pattern(h->tables);
  } catch (const std::exception &e) {
    return set_error(ZRK_ERR_PARSE, e.what());
  }
  return ZRK_OK;
}

int zrk_mech_parse(const char *mech_file, const char *therm_file, zrk_mech_t *out) {
  if (!mech_file || !therm_file || !out) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  *out = nullptr;
  auto h = std::make_unique<MechHandle>();
  int rc = parse_into(mech_file, therm_file, h.get());
  if (rc != ZRK_OK) return rc;
  *out = reinterpret_cast<zrk_mech_t>(h.release());
  return ZRK_OK;
}

int zrk_mech_create(const char *mech_file, const char *therm_file, zrk_mech_t *out) {
  if (!mech_file || !therm_file || !out) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_error(ZRK_ERR_NO_DEVICE, "no CUDA device is visible");
  auto h = std::make_unique<MechHandle>();
  int rc = parse_into(mech_file, therm_file, h.get());
  if (rc != ZRK_OK) return rc;
  try {
    h->dev = std::make_unique<DeviceMechanism>(h->tables, h->pattern);
  } catch (const std::exception &e) {
    return set_error(ZRK_ERR_CUDA, e.what());
  }
  h->cfg = default_launch(h->dev->view());
  *out = reinterpret_cast<zrk_mech_t>(h.release());
  return ZRK_OK;
}

int zrk_mech_free(zrk_mech_t m) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  delete reinterpret_cast<MechHandle *>(m);
  return ZRK_OK;
}

int zrk_mech_sizes(zrk_mech_t m, int *nsp, int *nrxn, int *nstep, int *nnz) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (nsp) *nsp = h->tables.nsp;
  if (nrxn) *nrxn = h->tables.nrxn;
  if (nstep) *nstep = h->tables.nstep;
  if (nnz) *nnz = h->pattern.nnz;
  return ZRK_OK;
}

int zrk_mech_table(zrk_mech_t m, const char *name, void *out, long capacity, long *count,
                   int *is_double) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (!name || !count || !is_double) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  const MechTables &t = reinterpret_cast<MechHandle *>(m)->tables;
  const std::vector<int> *vi = nullptr;
  const std::vector<double> *vd = nullptr;
  std::string n(name);
#define TI(x) if (n == #x) vi = &t.x;
#define TD(x) if (n == #x) vd = &t.x;
  TD(mw) TD(thermo) TI(step_rxn) TI(step_dir) TI(reac_ptr) TI(reac_spc) TI(prod_ptr) TI(prod_spc)
  TI(arr_step) TD(arr_lnA) TD(arr_n) TD(arr_Ta) TI(keq_step) TI(keq_fwd) TD(keq_dn)
  TI(tb_fwd) TI(tb_rev) TI(tb_ptr) TI(tb_spc) TD(tb_alpha)
  TI(fo_fwd) TI(fo_rev) TI(fo_type) TI(fo_spc) TI(fo_ptr) TI(fo_eff_spc) TD(fo_alpha) TD(fo_par)
  TI(plog_step) TI(plog_pt_ptr) TI(plog_ln_ptr) TD(plog_p) TD(plog_lnp) TD(plog_lnA) TD(plog_sgn)
  TD(plog_n) TD(plog_Ta)
#undef TI
#undef TD
  if (!vi && !vd) return set_error(ZRK_ERR_INVALID_ARGUMENT, "unknown table " + n);
  *is_double = vd ? 1 : 0;
  *count = vd ? (long)vd->size() : (long)vi->size();
  if (out && capacity >= *count) {
    if (vd) std::memcpy(out, vd->data(), vd->size() * sizeof(double));
    else std::memcpy(out, vi->data(), vi->size() * sizeof(int));
  }
  return ZRK_OK;
}

const char *zrk_mech_species_name(zrk_mech_t m, int idx) {
  if (!m) return nullptr;
  const MechTables &t = reinterpret_cast<MechHandle *>(m)->tables;
  if (idx < 0 || idx >= t.nsp) return nullptr;
  return t.species[idx].c_str();
}

int zrk_mech_jac_pattern(zrk_mech_t m, int *col_ptr, int *row_idx) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  const JacPattern &p = reinterpret_cast<MechHandle *>(m)->pattern;
  if (col_ptr) std::memcpy(col_ptr, p.col_ptr.data(), p.col_ptr.size() * sizeof(int));
  if (row_idx) std::memcpy(row_idx, p.row_idx.data(), p.row_idx.size() * sizeof(int));
  return ZRK_OK;
}

int zrk_mech_set_double_option(zrk_mech_t m, const char *name, double value) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (!name) return set_error(ZRK_ERR_INVALID_POINTER, "null name");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  std::string n(name);
  if (n == "reference_temperature") h->Tref = value;
  else if (n == "min_mass_fraction") h->mmf = value;
  else if (n == "step_limiter") h->lim = value;
  else return set_error(ZRK_ERR_INVALID_ARGUMENT, "unknown option " + n);
  return ZRK_OK;
}

int zrk_mech_get_double_option(zrk_mech_t m, const char *name, double *value) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (!name || !value) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  std::string n(name);
  if (n == "reference_temperature") *value = h->Tref;
  else if (n == "min_mass_fraction") *value = h->mmf;
  else if (n == "step_limiter") *value = h->lim;
  else return set_error(ZRK_ERR_INVALID_ARGUMENT, "unknown option " + n);
  return ZRK_OK;
}

int zrk_mech_set_launch(zrk_mech_t m, int ts, int v, int warps, int flags, int grid) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (!h->dev) return set_error(ZRK_ERR_NO_DEVICE, "handle has no device tables (zrk_mech_parse)");
  if (ts == 0) {
    h->cfg = default_launch(h->dev->view());
    return ZRK_OK;
  }
  LaunchCfg c;
  c.ts = ts;
  c.v = v;
  c.warps = warps;
  c.global_ws = (flags & ZRK_LAUNCH_GLOBAL_WS) != 0;
  c.stage = (flags & ZRK_LAUNCH_STAGE_TABLES) != 0;
  c.minb = (flags & ZRK_LAUNCH_TWO_CTAS) ? 2 : 1;
  c.grid = grid;
  if (!rates_jac_mapping_ok(c) || grid < 0 || (flags & ~7))
    return set_error(ZRK_ERR_INVALID_ARGUMENT, "bad launch mapping");
  if (rates_jac_smem_bytes(h->dev->view(), c) > 227 * 1024)
    return set_error(ZRK_ERR_INVALID_ARGUMENT, "workspace and staged tables do not fit in shared memory");
  h->cfg = c;
  return ZRK_OK;
}

int zrk_mech_get_launch(zrk_mech_t m, int *ts, int *v, int *warps, int *flags, int *grid) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (ts) *ts = h->cfg.ts;
  if (v) *v = h->cfg.v;
  if (warps) *warps = h->cfg.warps;
  if (flags)
    *flags = (h->cfg.global_ws ? ZRK_LAUNCH_GLOBAL_WS : 0) | (h->cfg.stage ? ZRK_LAUNCH_STAGE_TABLES : 0) |
             (h->cfg.minb == 2 ? ZRK_LAUNCH_TWO_CTAS : 0);
  if (grid) *grid = h->cfg.grid;
  return ZRK_OK;
}

int zrk_mech_autotune(zrk_mech_t m, int n, int ld, const double *T, const double *P,
                      const double *Y, double *wdot, double *jac, void *stream, float *best_ms) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (!h->dev) return set_error(ZRK_ERR_NO_DEVICE, "handle has no device tables (zrk_mech_parse)");
  if (n <= 0 || ld < n || !T || !P || !Y || !wdot) return set_error(ZRK_ERR_INVALID_ARGUMENT, "bad sample");
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  LaunchCfg best = h->cfg;
  float best_t = 1e30f;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  for (int ts : {8, 16, 32})
    for (int v : {1, 2, 4})
      for (int warps : {4, 8, 16, 32}) {
        LaunchCfg c;
        c.ts = ts;
        c.v = v;
        c.warps = warps;
        if (!rates_jac_mapping_ok(c)) continue;
        if (rates_jac_ws_bytes(h->dev->view(), c) > 227 * 1024) {
          c.global_ws = true;
          c.grid = 2 * sms;
        }
        for (int variant = 0; variant < 3; ++variant) {
          c.stage = variant == 1;
          c.minb = variant == 2 ? 2 : 1;
          if (c.stage && rates_jac_smem_bytes(h->dev->view(), c) > 227 * 1024) continue;
          if (!rates_jac_mapping_ok(c)) continue;
          h->cfg = c;
          float t = 0.f;
          bool ok = true;
          for (int rep = 0; rep < 3 && ok; ++rep) {
            cudaEventRecord(e0, st);
            ok = zrk_rates_jac_dev(m, n, ld, T, P, Y, wdot, jac, nullptr, stream) == ZRK_OK;
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) t += ms;  // first launch warms up
          }
          if (ok && cudaGetLastError() == cudaSuccess && t < best_t) {
            best_t = t;
            best = c;
          }
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->cfg = best;
  if (best_ms) *best_ms = best_t / 2;
  return ZRK_OK;
}

int zrk_rates_jac_dev(zrk_mech_t m, int n, int ld, const double *T, const double *P,
                      const double *Y, double *wdot, double *jac, double *ydot, void *stream) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (n < 0 || ld < n) return set_error(ZRK_ERR_INVALID_ARGUMENT, "need 0 <= n <= ld");
  if (n == 0) return ZRK_OK;
  if (!T || !P || !Y || !wdot) return set_error(ZRK_ERR_INVALID_POINTER, "null array");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (!h->dev) return set_error(ZRK_ERR_NO_DEVICE, "handle has no device tables (zrk_mech_parse)");
  RatesJacArgs a;
  a.n = n;
  a.ld = ld;
  a.T = T;
  a.P = P;
  a.Y = Y;
  a.wdot = wdot;
  a.jac = jac;
  a.ydot = ydot;
  KinParams kp{h->Tref, h->mmf, h->lim, std::sqrt(2.2204460492503131e-16)};
  if (h->cfg.global_ws) {
    const int ntiles = (n + h->cfg.ts - 1) / h->cfg.ts;
    int grid = h->cfg.grid > 0 ? h->cfg.grid : ntiles;
    if (grid > ntiles) grid = ntiles;
    size_t need = (size_t)grid * rates_jac_ws_bytes(h->dev->view(), h->cfg);
    cudaError_t e = h->ensure_scratch(need);
    if (e != cudaSuccess) return cuda_error(e, "scratch allocation");
    a.scratch = (double *)h->scratch;
    a.scratch_bytes = h->scratch_bytes;
  }
  cudaError_t e = launch_rates_jac(h->dev->view(), a, kp, h->cfg, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "rates_jac launch");
  return ZRK_OK;
}

int zrk_rates_tc_dev(zrk_mech_t m, int n, int ld, const double *T, const double *C,
                     const double *step_limiter, double *net, double *create, double *destroy,
                     double *rop, void *stream) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (n < 0 || ld < n) return set_error(ZRK_ERR_INVALID_ARGUMENT, "need 0 <= n <= ld");
  if (n == 0) return ZRK_OK;
  if (!T || !C) return set_error(ZRK_ERR_INVALID_POINTER, "null array");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (!h->dev) return set_error(ZRK_ERR_NO_DEVICE, "handle has no device tables (zrk_mech_parse)");
  RatesTCArgs a;
  a.n = n;
  a.ld = ld;
  a.T = T;
  a.C = C;
  a.lim_step = step_limiter;
  a.net = net;
  a.create = create;
  a.destroy = destroy;
  a.rop = rop;
  cudaError_t e = launch_rates_tc(h->dev->view(), a, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "rates_tc launch");
  return ZRK_OK;
}

int zrk_rates_tc_host(zrk_mech_t m, int n, const double *T, const double *C,
                      const double *step_limiter, double *net, double *create, double *destroy,
                      double *rop) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (n < 0) return set_error(ZRK_ERR_INVALID_ARGUMENT, "n < 0");
  if (n == 0) return ZRK_OK;
  if (!T || !C) return set_error(ZRK_ERR_INVALID_POINTER, "null array");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (!h->dev) return set_error(ZRK_ERR_NO_DEVICE, "handle has no device tables (zrk_mech_parse)");
  const size_t S = h->tables.nsp, N = h->tables.nstep, dp = sizeof(double);
  // device slot: T | C | limiter | net | create | destroy | rop
  const size_t doubles = n + S * n + N + 3 * S * n + N * n;
  cudaError_t e = h->ensure_pipe(doubles * dp);
  if (e != cudaSuccess) return cuda_error(e, "device buffers");
  double *dT = (double *)h->pipe, *dC = dT + n, *dL = dC + S * n, *dN = dL + N, *dCr = dN + S * n,
         *dDe = dCr + S * n, *dR = dDe + S * n;
  cudaStream_t st = h->pipe_stream[0];
  if ((e = cudaMemcpyAsync(dT, T, n * dp, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dC, C, S * n * dp, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (step_limiter &&
       (e = cudaMemcpyAsync(dL, step_limiter, N * dp, cudaMemcpyHostToDevice, st)) != cudaSuccess))
    return cuda_error(e, "copy in");
  RatesTCArgs a;
  a.n = n;
  a.ld = n;
  a.T = dT;
  a.C = dC;
  a.lim_step = step_limiter ? dL : nullptr;
  a.net = net ? dN : nullptr;
  a.create = create ? dCr : nullptr;
  a.destroy = destroy ? dDe : nullptr;
  a.rop = rop ? dR : nullptr;
  if ((e = launch_rates_tc(h->dev->view(), a, st)) != cudaSuccess) return cuda_error(e, "rates_tc launch");
  if ((net && (e = cudaMemcpyAsync(net, dN, S * n * dp, cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
      (create && (e = cudaMemcpyAsync(create, dCr, S * n * dp, cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
      (destroy && (e = cudaMemcpyAsync(destroy, dDe, S * n * dp, cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
      (rop && (e = cudaMemcpyAsync(rop, dR, N * n * dp, cudaMemcpyDeviceToHost, st)) != cudaSuccess))
    return cuda_error(e, "copy out");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(e, "rates_tc");
  return ZRK_OK;
}

int zrk_rates_jac_host(zrk_mech_t m, int n, const double *T, const double *P, const double *Y,
                       double *wdot, double *jac) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (n < 0) return set_error(ZRK_ERR_INVALID_ARGUMENT, "n < 0");
  if (n == 0) return ZRK_OK;
  if (!T || !P || !Y || !wdot) return set_error(ZRK_ERR_INVALID_POINTER, "null array");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (!h->dev) return set_error(ZRK_ERR_NO_DEVICE, "handle has no device tables (zrk_mech_parse)");
  const int S = h->tables.nsp, nnz = h->pattern.nnz;
  // Two-slot pipeline: chunk i uses stream/slot i%2, so with pinned host
  // buffers the copies of one chunk overlap the kernel of the other
  // (pageable buffers are staged by the driver and overlap little; the
  // global-workspace mapping shares one scratch area and uses one stream).
  // Device slots are cached.
  const size_t per_state = sizeof(double) * (2 + 2 * (size_t)S + (jac ? nnz : 0));
  long chunk = (long)((512ull << 20) / per_state);
  chunk = std::max(1024L, std::min<long>(chunk, n));
  chunk = (chunk + 31) / 32 * 32;
  cudaError_t e = h->ensure_pipe(2 * chunk * per_state);
  if (e != cudaSuccess) return cuda_error(e, "pipeline buffers");
  const size_t dp = sizeof(double);
  for (long c0 = 0, i = 0; c0 < n; c0 += chunk, ++i) {
    const int cn = (int)std::min<long>(chunk, n - c0);
    // the global-workspace mapping shares one scratch area: keep one stream
    cudaStream_t st = h->pipe_stream[h->cfg.global_ws ? 0 : i % 2];
    double *base = (double *)h->pipe + (i % 2) * chunk * (per_state / dp);
    double *dT = base, *dP = dT + chunk, *dY = dP + chunk, *dW = dY + (size_t)S * chunk;
    double *dJ = jac ? dW + (size_t)S * chunk : nullptr;
    if ((e = cudaMemcpyAsync(dT, T + c0, cn * dp, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dP, P + c0, cn * dp, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpy2DAsync(dY, chunk * dp, Y + c0, (size_t)n * dp, cn * dp, S,
                               cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return cuda_error(e, "H2D");
    int rc = zrk_rates_jac_dev(m, cn, (int)chunk, dT, dP, dY, dW, dJ, nullptr, st);
    if (rc != ZRK_OK) return rc;
    if ((e = cudaMemcpy2DAsync(wdot + c0, (size_t)n * dp, dW, chunk * dp, cn * dp, S,
                               cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return cuda_error(e, "D2H");
    if (jac && (e = cudaMemcpy2DAsync(jac + c0, (size_t)n * dp, dJ, chunk * dp, cn * dp, nnz,
                                      cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return cuda_error(e, "D2H");
  }
  for (int k = 0; k < 2; ++k)
    if ((e = cudaStreamSynchronize(h->pipe_stream[k])) != cudaSuccess) return cuda_error(e, "synchronize");
  return ZRK_OK;
}

}  // extern "C"
