// solver.cpp -- see solver.h.
#include "solver.h"

#include "integrator_group.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>

namespace zrk {
namespace {

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
size_t put(std::vector<unsigned char> &b, const std::vector<T> &v) {
  size_t off = (b.size() + 255) & ~size_t(255);
  b.resize(off + std::max<size_t>(v.size() * sizeof(T), 16), 0);
  if (!v.empty()) std::memcpy(b.data() + off, v.data(), v.size() * sizeof(T));
  return off;
}

}  // namespace

ReactorSolver::ReactorSolver(const std::string &mech, const std::string &therm) {
  tables_ = load_chemkin(mech, therm);
  pat_ = build_jac_pattern(tables_);
  lus_ = analyze_lu(pat_);
  dm_ = std::make_unique<DeviceMechanism>(tables_, pat_);
  std::vector<unsigned char> b;
  size_t o_cp = put(b, lus_.col_ptr), o_ri = put(b, lus_.row_idx), o_dg = put(b, lus_.diag_pos),
         o_ip = put(b, lus_.iperm), o_jl = put(b, lus_.jac_to_lu), o_do = put(b, lus_.diag_of_orig);
  ck(cudaMalloc(&lu_blob_, b.size()), "cudaMalloc(LU tables)");
  ck(cudaMemcpy(lu_blob_, b.data(), b.size(), cudaMemcpyHostToDevice), "cudaMemcpy(LU tables)");
  auto P = [&](size_t off) { return (const int *)((const unsigned char *)lu_blob_ + off); };
  lud_.n = lus_.n;
  lud_.nnz = lus_.nnz;
  lud_.col_ptr = P(o_cp);
  lud_.row_idx = P(o_ri);
  lud_.diag = P(o_dg);
  lud_.iperm = P(o_ip);
  lud_.jac_to_lu = P(o_jl);
  lud_.diag_of_orig = P(o_do);
  ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  ck(cudaEventCreate(&ev0_), "event");
  ck(cudaEventCreate(&ev1_), "event");
}

ReactorSolver::~ReactorSolver() {
  if (graph_) cudaGraphExecDestroy(graph_);
  cudaFreeHost(hT_); cudaFreeHost(hP_); cudaFreeHost(hY_); cudaFreeHost(horder_); cudaFreeHost(hstats_);
  cudaFreeHost(hsrc_); cudaFreeHost(hign_); cudaFree(dsrc_); cudaFree(dign_);
  cudaFreeHost(hde_); cudaFree(dde_);
  cudaFree(lu_blob_);
  cudaFree(dcb_rec_); cudaFree(dcb_cnt_); cudaFree(dcb_stop_); cudaFree(dcb_order_);
  cudaFree(dT_); cudaFree(dP_); cudaFree(dY_); cudaFree(dv_); cudaFree(dstate_); cudaFree(dlu_);
  cudaFree(dstats_); cudaFree(dorder_); cudaFree(dhead_); cudaFree(drop_);
  cudaFree(dgrp_); cudaFree(dpart_); cudaFreeHost(hpart_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
}

cudaError_t ReactorSolver::reserve(int n, bool fp32) {
  if (n <= cap_ && fp32 == cap_fp32_) return cudaSuccess;
  cudaFree(dT_); cudaFree(dP_); cudaFree(dY_); cudaFree(dv_); cudaFree(dstate_); cudaFree(dlu_);
  cudaFree(dstats_); cudaFree(dorder_); cudaFree(dhead_);
  cudaFreeHost(hT_); cudaFreeHost(hP_); cudaFreeHost(hY_); cudaFreeHost(horder_); cudaFreeHost(hstats_);
  cudaFreeHost(hsrc_); cudaFreeHost(hign_); cudaFree(dsrc_); cudaFree(dign_);
  cudaFreeHost(hde_); cudaFree(dde_);
  hsrc_ = hign_ = dsrc_ = dign_ = hde_ = dde_ = nullptr;
  hT_ = hP_ = hY_ = nullptr;
  horder_ = nullptr;
  hstats_ = nullptr;
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  graph_key_.clear();
  dT_ = dP_ = dY_ = dv_ = dstate_ = nullptr;
  dlu_ = nullptr;
  dstats_ = nullptr;
  dorder_ = dhead_ = nullptr;
  cap_ = 0;
  const int cap = std::max(n, 32);
  const size_t S = tables_.nsp;
  const long st = integ_state_doubles(dm_->view(), lud_);
  cudaError_t e;
  if ((e = cudaMalloc(&dT_, cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dP_, cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dv_, cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dY_, cap * S * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dstate_, (size_t)cap * st * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dlu_, (size_t)cap * lud_.nnz * (fp32 ? sizeof(float) : sizeof(double)))) !=
      cudaSuccess)
    return e;
  if ((e = cudaMalloc(&dstats_, cap * sizeof(ReactorStats))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dorder_, cap * sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dhead_, sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&hT_, cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&hP_, cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&hY_, cap * S * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&horder_, cap * sizeof(int))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&hstats_, cap * sizeof(ReactorStats))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&hsrc_, cap * S * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&hign_, cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dsrc_, cap * S * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dign_, cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMallocHost(&hde_, 3 * (size_t)cap * sizeof(double))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&dde_, 3 * (size_t)cap * sizeof(double))) != cudaSuccess) return e;
  cap_ = cap;
  cap_fp32_ = fp32;
  return cudaSuccess;
}

// Solve with the plugin's step callback: every accepted step is recorded on
// the device (integrator.h CbCtx) and the callback runs on the host, reactor
// by reactor and step by step, after the integration (a host function cannot
// run inside the kernel).  Reactors with more steps than the record capacity
// are integrated again with room for all of their steps (the integration is
// deterministic, so the steps are the same), and reactors whose callback
// returned nonzero are integrated again up to that step, which ends their
// call with that step's state, as the reference's break out of its step loop
// does (solver_cvode.cpp:247-257).  Staging: hT_/hP_/hY_ hold the inputs on
// entry and the results on return; hstats_ and hign_ the results.
cudaError_t ReactorSolver::solve_with_callback(int method, const IntegOpts &io, IntegArgs a,
                                               int dthreads, int dctas, int spill, int W, int ctas,
                                               bool rop_smem, int n, double dt,
                                               const StepCallback &cb) {
  const int S = tables_.nsp, nv = S + 1;
  const size_t rec = 3 + 2 * (size_t)nv;
  const size_t kBudget = (size_t)1 << 30;  // record memory per launch
  const long steps_max = (long)io.max_steps * io.max_retries;
  cudaStream_t s = stream_;
  cudaError_t e;
  auto ensure = [&](size_t rec_bytes) -> cudaError_t {
    if (dcb_n_ < n) {
      cudaFree(dcb_cnt_);
      cudaFree(dcb_stop_);
      cudaFree(dcb_order_);
      dcb_cnt_ = dcb_stop_ = dcb_order_ = nullptr;
      dcb_n_ = 0;
      cudaError_t r;
      if ((r = cudaMalloc(&dcb_cnt_, n * sizeof(int))) != cudaSuccess) return r;
      if ((r = cudaMalloc(&dcb_stop_, n * sizeof(int))) != cudaSuccess) return r;
      if ((r = cudaMalloc(&dcb_order_, n * sizeof(int))) != cudaSuccess) return r;
      dcb_n_ = n;
    }
    if (dcb_bytes_ < rec_bytes) {
      cudaFree(dcb_rec_);
      dcb_rec_ = nullptr;
      dcb_bytes_ = 0;
      cudaError_t r = cudaMalloc(&dcb_rec_, rec_bytes);
      if (r != cudaSuccess) return r;
      dcb_bytes_ = rec_bytes;
    }
    return cudaSuccess;
  };
  // inputs as staged by solve(), kept for the repeated integrations
  const std::vector<double> T0(hT_, hT_ + n), P0(hP_, hP_ + n), Y0(hY_, hY_ + (size_t)n * S);
  std::vector<double> Tr(n), Pr(n), Yr((size_t)n * S), ign(n, -1.0);
  std::vector<ReactorStats> str(n);
  std::vector<int> cnt(n, 0);
  // one integration of the reactors in `sel` from their initial states, with
  // `cap` records each and per-reactor stops (empty: none); results merged
  auto run = [&](const std::vector<int> &sel, int cap, const std::vector<int> &stop,
                 std::vector<double> *recs) -> cudaError_t {
    const int m = (int)sel.size();
    cudaError_t r;
    if ((r = ensure((size_t)m * cap * rec * sizeof(double))) != cudaSuccess) return r;
    std::memcpy(hT_, T0.data(), n * sizeof(double));
    std::memcpy(hP_, P0.data(), n * sizeof(double));
    std::memcpy(hY_, Y0.data(), (size_t)n * S * sizeof(double));
    std::memcpy(horder_, sel.data(), m * sizeof(int));
    if ((r = cudaMemcpyAsync(dT_, hT_, n * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (r = cudaMemcpyAsync(dP_, hP_, n * sizeof(double), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (r = cudaMemcpyAsync(dY_, hY_, (size_t)n * S * sizeof(double), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (r = cudaMemcpyAsync(dcb_order_, horder_, m * sizeof(int), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess ||
        (a.ysrc && (r = cudaMemcpyAsync(dsrc_, hsrc_, (size_t)n * S * sizeof(double),
                                        cudaMemcpyHostToDevice, s)) != cudaSuccess) ||
        (a.dpdt && (r = cudaMemcpyAsync(dde_, hde_, n * sizeof(double), cudaMemcpyHostToDevice, s)) !=
                       cudaSuccess) ||
        (a.esrc && (r = cudaMemcpyAsync(dde_ + cap_, hde_ + cap_, n * sizeof(double),
                                        cudaMemcpyHostToDevice, s)) != cudaSuccess) ||
        (a.tdel_in && (r = cudaMemcpyAsync(dde_ + 2 * cap_, hde_ + 2 * cap_, n * sizeof(double),
                                           cudaMemcpyHostToDevice, s)) != cudaSuccess) ||
        (r = cudaMemsetAsync(dhead_, 0, sizeof(int), s)) != cudaSuccess ||
        (r = cudaMemsetAsync(dcb_cnt_, 0, n * sizeof(int), s)) != cudaSuccess)
      return r;
    if (!stop.empty() &&
        (r = cudaMemcpyAsync(dcb_stop_, stop.data(), n * sizeof(int), cudaMemcpyHostToDevice, s)) !=
            cudaSuccess)
      return r;
    IntegArgs b = a;
    b.n_reactors = m;
    b.order = dcb_order_;
    b.cb_rec = dcb_rec_;
    b.cb_cap = cap;
    b.cb_cnt = dcb_cnt_;
    b.cb_stop = stop.empty() ? nullptr : dcb_stop_;
    if ((r = cudaEventRecord(ev0_, s)) != cudaSuccess) return r;
    r = method == 1 ? launch_integrate_dense(dm_->view(), io, b, dthreads, std::min(dctas, m), spill, s)
                    : launch_integrate(dm_->view(), lud_, io, b, W, ctas, rop_smem, s);
    if (r != cudaSuccess) return r;
    if ((r = cudaEventRecord(ev1_, s)) != cudaSuccess) return r;
    std::vector<int> c(n);
    if ((r = cudaMemcpyAsync(hT_, dT_, n * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (r = cudaMemcpyAsync(hP_, dP_, n * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (r = cudaMemcpyAsync(hY_, dY_, (size_t)n * S * sizeof(double), cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (r = cudaMemcpyAsync(hstats_, dstats_, n * sizeof(ReactorStats), cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (a.t_ign && (r = cudaMemcpyAsync(hign_, dign_, n * sizeof(double), cudaMemcpyDeviceToHost, s)) !=
                        cudaSuccess) ||
        (r = cudaMemcpyAsync(c.data(), dcb_cnt_, n * sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return r;
    if (recs) {  // slot i holds the records of sel[i]
      recs->resize((size_t)m * cap * rec);
      if ((r = cudaMemcpyAsync(recs->data(), dcb_rec_, recs->size() * sizeof(double),
                               cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return r;
    }
    if ((r = cudaStreamSynchronize(s)) != cudaSuccess) return r;
    for (int k : sel) {
      Tr[k] = hT_[k];
      Pr[k] = hP_[k];
      std::memcpy(&Yr[(size_t)k * S], &hY_[(size_t)k * S], S * sizeof(double));
      str[k] = hstats_[k];
      if (a.t_ign) ign[k] = hign_[k];
      cnt[k] = c[k];
    }
    return cudaSuccess;
  };
  std::vector<int> all(n), slot(n);
  for (int k = 0; k < n; ++k) all[k] = horder_[k];  // the cost order solve() chose
  for (int i = 0; i < n; ++i) slot[all[i]] = i;
  int cap = (int)std::max<long>(
      8, std::min<long>(steps_max, (long)(kBudget / ((size_t)n * rec * sizeof(double)))));
  cap = std::min(cap, 4096);
  std::vector<double> recs;
  if ((e = run(all, cap, {}, &recs)) != cudaSuccess) return e;
  // callbacks in reactor order; reactors past the capacity are integrated
  // again alone with room for all of their steps
  std::vector<int> stop(n, 0);
  bool any_stop = false;
  std::vector<double> more;
  for (int k = 0; k < n; ++k) {
    const double *base = recs.data() + (size_t)slot[k] * cap * rec;
    if (cnt[k] > cap) {
      const int keep = cnt[k];
      if ((e = run({k}, keep, {}, &more)) != cudaSuccess) return e;
      if (cnt[k] != keep) return cudaErrorUnknown;  // a replay must take the same steps
      base = more.data();
    }
    const int id = cb.reactor_ids ? cb.reactor_ids[k] : k;
    for (int i = 0; i < cnt[k]; ++i) {
      const double *r0 = base + (size_t)i * rec;
      if (cb.fn(id, (int)r0[2], r0[0], r0[1], r0 + 3, r0 + 3 + nv, cb.data) != 0) {
        if (i + 1 < cnt[k]) {
          stop[k] = i + 1;
          any_stop = true;
        }
        break;
      }
    }
  }
  if (any_stop) {  // the reactors whose callback ended their call early
    std::vector<int> sel;
    for (int k = 0; k < n; ++k)
      if (stop[k] > 0) sel.push_back(k);
    if ((e = run(sel, 1, stop, nullptr)) != cudaSuccess) return e;
  }
  std::memcpy(hT_, Tr.data(), n * sizeof(double));
  std::memcpy(hP_, Pr.data(), n * sizeof(double));
  std::memcpy(hY_, Yr.data(), (size_t)n * S * sizeof(double));
  std::memcpy(hstats_, str.data(), n * sizeof(ReactorStats));
  if (a.t_ign) std::memcpy(hign_, ign.data(), n * sizeof(double));
  return cudaSuccess;
}

int ReactorSolver::solve(const SolveOptions &o, int n, double dt, double *T, double *P, double *mf,
                         int stride, double *cost, double *gpu_time, double *temp_delta,
                         double temp_threshold, std::vector<ReactorStats> *stats,
                         SolveStatsTotals *tot, const double *ysrc, double *t_ign,
                         const double *dpdt, const double *esrc, const StepCallback *cb) {
  if (n <= 0) return 0;
  const int S = tables_.nsp;
  cudaError_t e = reserve(n, o.lu_fp32);
  if (e != cudaSuccess) {
    last_error = std::string("device allocation: ") + cudaGetErrorString(e);
    return -1;
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  if (o.sort_reactors && cost)  // longest previous cost first (work queue)
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return std::fabs(cost[a]) > std::fabs(cost[b]); });
  std::vector<double> T0(T, T + n);
  double *Y = hY_;  // packed reactor-major mass fractions in pinned staging
  for (int r = 0; r < n; ++r) std::memcpy(&Y[(size_t)r * S], mf + (size_t)r * stride, S * sizeof(double));
  std::memcpy(hT_, T, n * sizeof(double));
  std::memcpy(hP_, P, n * sizeof(double));
  const DevMech &m = dm_->view();
  const size_t kSmemMax = 227 * 1024;
  // dense block in shared memory, spilling the rates of progress and then the
  // BDF differences to an L2-resident global slice if needed
  int spill = -1;
  // preference: the Jacobian beside the factor in shared memory (the FP32
  // path reads it in every Krylov iteration), then rates of progress and
  // BDF history spilled to an L2-resident slice
  for (int sp : {4, 0, 5, 1, 3})
    if (m.nsp + 1 <= kDenseMaxN && dense_smem_bytes(m, o.lu_fp32, nullptr, sp) <= kSmemMax) {
      spill = sp;
      break;
    }
  int method = o.method;
  if (method == 0) method = spill >= 0 ? 1 : 2;
  if (method == 3) {  // the plain FP64 group path supports the reference's basic reactor
    const char *why = nullptr;
    if (m.nsp + 1 > kDenseMaxN) why = "more than 255 species";
    else if (o.lu_fp32) why = "lu_fp32";
    else if (o.pred.enabled) why = "a learned predictor";
    else if (esrc) why = "E_SRC";
    else if (cb && cb->fn) why = "a step callback";
    else if (o.stop_after_ignition && o.dT_ign > 0.0) why = "stop_after_ignition";
    if (why) {
      last_error = std::string("gpu_method 3 (plain FP64 group path) does not support ") + why;
      return -1;
    }
  } else if (method < 0 || method > 3) {
    last_error = "gpu_method must be 0, 1, 2 or 3";
    return -1;
  }
  if (method == 1 && spill < 0) {
    last_error = "dense block does not fit in shared memory";
    return -1;
  }
  // launch mapping: up to 12 warps per CTA (register bound), rates of
  // progress in shared memory when they fit, else in an L2-resident scratch
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t kSmem = 227 * 1024;
  bool rop_smem = integ_smem_per_warp(m, lud_, true) * 12 <= kSmem;
  int W = o.warps_per_cta > 0 ? o.warps_per_cta : 12;
  while (W > 1 && integ_smem_per_warp(m, lud_, rop_smem) * W > kSmem) --W;
  if (!rop_smem && integ_smem_per_warp(m, lud_, false) * W > kSmem) {
    last_error = "mechanism too large for the integrator's shared memory";
    return -1;
  }
  const int ctas = sms;
  int dthreads = o.threads;
  int dctas = ctas;
  if (method == 1) {
    if (dthreads <= 0) {
      const int work = std::max(m.nsp + 1, m.nrxn / 2);
      dthreads = 32;
      while (dthreads < work && dthreads < 512) dthreads *= 2;
    }
    const size_t sm = dense_smem_bytes(m, o.lu_fp32, nullptr, spill);
    int per_sm = (int)std::min<size_t>(kSmemMax / sm, (size_t)(2048 / dthreads));
    per_sm = std::max(1, std::min(per_sm, 65536 / (dthreads * 128)));
    dctas = std::min(n, sms * per_sm);
  }
  // the dense integrator's slice also holds the energy-source coupling vectors
  if (!rop_smem || method == 1) {
    size_t need = method == 1 ? (size_t)dctas * dense_spill_doubles(m) * sizeof(double)
                              : (size_t)ctas * W * m.nstep * sizeof(double);
    if (need > drop_bytes_) {
      cudaFree(drop_);
      drop_ = nullptr;
      drop_bytes_ = 0;
      if ((e = cudaMalloc(&drop_, need)) != cudaSuccess) {
        last_error = "ROP scratch allocation";
        return -1;
      }
      drop_bytes_ = need;
    }
  }
  IntegOpts io;
  std::memset(&io, 0, sizeof(io));  // padding too: the bytes key the captured graph
  io.rtol = o.rtol;
  io.atol = o.atol;
  io.max_dt = o.max_dt;
  io.nlscoef = o.nlscoef;
  io.eps_lin = o.eps_lin;
  io.pred = o.pred;
  io.dT_ign = o.dT_ign;
  if (io.pred.enabled && method != 1) io.pred.enabled = 0;  // dense integrator only
  io.max_steps = o.max_steps;
  io.max_retries = std::max(1, o.max_retries);
  io.retry_atol_factor = o.retry_atol;
  io.retry_rtol_factor = o.retry_rtol;
  io.Tref = o.Tref;
  io.mmf = o.mmf;
  io.lim = o.lim;
  io.sqrt_ur = std::sqrt(2.2204460492503131e-16);
  io.lu_fp32 = o.lu_fp32 ? 1 : 0;
  io.cp = o.constant_pressure ? 1 : 0;
  io.always_T = o.always_solve_T ? 1 : 0;
  io.stop_ign = (o.stop_after_ignition && o.dT_ign > 0.0) ? 1 : 0;
  io.abstol_dens = o.abstol_dens ? 1 : 0;
  IntegArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n_reactors = n;
  a.order = dorder_;
  a.queue_head = dhead_;
  a.dt = dt;
  a.T = dT_;
  a.P = dP_;
  a.Y = dY_;
  a.v = dv_;
  a.state = dstate_;
  a.state_stride = integ_state_doubles(m, lud_);
  a.lu = dlu_;
  a.lu_stride = lud_.nnz;
  a.stats = dstats_;
  a.rop_scratch = drop_;
  a.ysrc = ysrc ? dsrc_ : nullptr;
  // ignition times are tracked whenever delta_temperature_ignition > 0 (the
  // stop_after_ignition option needs them even without a caller field)
  a.t_ign = (o.dT_ign > 0.0) ? dign_ : nullptr;
  a.dpdt = dpdt ? dde_ : nullptr;
  a.esrc = esrc ? dde_ + cap_ : nullptr;
  a.tdel_in = (!o.always_solve_T && temp_delta) ? dde_ + 2 * cap_ : nullptr;
  cudaStream_t s = stream_;
  std::memcpy(horder_, order.data(), n * sizeof(int));
  if (ysrc) std::memcpy(hsrc_, ysrc, (size_t)n * S * sizeof(double));
  if (dpdt) std::memcpy(hde_, dpdt, n * sizeof(double));
  if (esrc) std::memcpy(hde_ + cap_, esrc, n * sizeof(double));
  if (a.tdel_in) std::memcpy(hde_ + 2 * cap_, temp_delta, n * sizeof(double));
  if (method == 1) {
    a.state = dstate_;
    a.state_stride = m.nnz;
  }
  const bool with_cb = cb && cb->fn;
  GroupCounters gcnt;
  if (method == 3) {
    // host-driven, kernel by kernel (the reference GPU path's structure):
    // not captured in a graph
    const int gmax = std::min(std::max(1, o.group_max), n);
    const size_t slot_bytes = group_slot_doubles(m) * sizeof(double);
    const size_t need = (size_t)gmax * slot_bytes;
    if (need > dgrp_bytes_) {
      cudaFree(dgrp_);
      dgrp_ = nullptr;
      dgrp_bytes_ = 0;
      if ((e = cudaMalloc(&dgrp_, need)) != cudaSuccess) {
        last_error = "group workspace allocation";
        return -1;
      }
      dgrp_bytes_ = need;
    }
    if (gmax > part_cap_) {
      cudaFree(dpart_);
      cudaFreeHost(hpart_);
      dpart_ = hpart_ = nullptr;
      part_cap_ = 0;
      if ((e = cudaMalloc(&dpart_, (size_t)gmax * 6 * sizeof(double))) != cudaSuccess ||
          (e = cudaMallocHost(&hpart_, (size_t)gmax * 6 * sizeof(double))) != cudaSuccess) {
        last_error = "group partial-sum allocation";
        return -1;
      }
      part_cap_ = gmax;
    }
    int threads = o.threads;
    if (threads <= 0) {
      const int work = std::max(m.nsp + 1, m.nrxn / 2);
      threads = 32;
      while (threads < work && threads < 512) threads *= 2;
    }
    cudaError_t ce = cudaSuccess;
    auto q = [&](cudaError_t r) {
      if (ce == cudaSuccess) ce = r;
    };
    q(cudaMemcpyAsync(dT_, hT_, n * sizeof(double), cudaMemcpyHostToDevice, s));
    q(cudaMemcpyAsync(dP_, hP_, n * sizeof(double), cudaMemcpyHostToDevice, s));
    q(cudaMemcpyAsync(dY_, hY_, (size_t)n * S * sizeof(double), cudaMemcpyHostToDevice, s));
    q(cudaMemcpyAsync(dorder_, horder_, n * sizeof(int), cudaMemcpyHostToDevice, s));
    if (a.ysrc) q(cudaMemcpyAsync(dsrc_, hsrc_, (size_t)n * S * sizeof(double), cudaMemcpyHostToDevice, s));
    if (a.dpdt) q(cudaMemcpyAsync(dde_, hde_, n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (a.tdel_in)
      q(cudaMemcpyAsync(dde_ + 2 * cap_, hde_ + 2 * cap_, n * sizeof(double), cudaMemcpyHostToDevice, s));
    q(cudaEventRecord(ev0_, s));
    if (ce == cudaSuccess)
      q(integrate_group(m, io, a, dorder_, gmax, threads, dgrp_, dpart_, hpart_, s, &gcnt));
    q(cudaEventRecord(ev1_, s));
    q(cudaMemcpyAsync(hT_, dT_, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    q(cudaMemcpyAsync(hP_, dP_, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    q(cudaMemcpyAsync(hY_, dY_, (size_t)n * S * sizeof(double), cudaMemcpyDeviceToHost, s));
    q(cudaMemcpyAsync(hstats_, dstats_, n * sizeof(ReactorStats), cudaMemcpyDeviceToHost, s));
    if (a.t_ign) q(cudaMemcpyAsync(hign_, dign_, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    q(cudaStreamSynchronize(s));
    if (ce != cudaSuccess) {
      last_error = std::string("group integration: ") + cudaGetErrorString(ce);
      return -1;
    }
  } else if (with_cb) {
    if ((e = solve_with_callback(method, io, a, dthreads, dctas, spill, W, ctas, rop_smem, n, dt, *cb)) !=
        cudaSuccess) {
      last_error = std::string("integration with step callback: ") + cudaGetErrorString(e);
      return -1;
    }
  } else {
    // The whole call (copies in, queue reset, the persistent kernel between
    // two timing events, copies out) is one CUDA graph, captured once per
    // configuration and replayed while nothing it depends on changes.
    std::vector<unsigned char> key;
    auto put_key = [&](const void *p, size_t b) {
      key.insert(key.end(), (const unsigned char *)p, (const unsigned char *)p + b);
    };
    const int kv[9] = {n, method, dthreads, dctas, spill, W, ctas, rop_smem ? 1 : 0, S};
    put_key(kv, sizeof(kv));
    put_key(&io, sizeof(io));
    put_key(&a, sizeof(a));
    if (!graph_ || key != graph_key_) {
      if (graph_) cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
      graph_key_.clear();
      if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed)) != cudaSuccess) {
        last_error = std::string("graph capture: ") + cudaGetErrorString(e);
        return -1;
      }
      cudaError_t ce = cudaSuccess;
      auto q = [&](cudaError_t r) {
        if (ce == cudaSuccess) ce = r;
      };
      q(cudaMemcpyAsync(dT_, hT_, n * sizeof(double), cudaMemcpyHostToDevice, s));
      q(cudaMemcpyAsync(dP_, hP_, n * sizeof(double), cudaMemcpyHostToDevice, s));
      q(cudaMemcpyAsync(dY_, hY_, (size_t)n * S * sizeof(double), cudaMemcpyHostToDevice, s));
      q(cudaMemcpyAsync(dorder_, horder_, n * sizeof(int), cudaMemcpyHostToDevice, s));
      if (a.ysrc) q(cudaMemcpyAsync(dsrc_, hsrc_, (size_t)n * S * sizeof(double), cudaMemcpyHostToDevice, s));
      if (a.dpdt) q(cudaMemcpyAsync(dde_, hde_, n * sizeof(double), cudaMemcpyHostToDevice, s));
      if (a.esrc)
        q(cudaMemcpyAsync(dde_ + cap_, hde_ + cap_, n * sizeof(double), cudaMemcpyHostToDevice, s));
      if (a.tdel_in)
        q(cudaMemcpyAsync(dde_ + 2 * cap_, hde_ + 2 * cap_, n * sizeof(double),
                          cudaMemcpyHostToDevice, s));
      q(cudaMemsetAsync(dhead_, 0, sizeof(int), s));
      q(cudaEventRecordWithFlags(ev0_, s, cudaEventRecordExternal));  // a timing node in the graph
      q(method == 1 ? launch_integrate_dense(m, io, a, dthreads, dctas, spill, s)
                    : launch_integrate(m, lud_, io, a, W, ctas, rop_smem, s));
      q(cudaEventRecordWithFlags(ev1_, s, cudaEventRecordExternal));
      q(cudaMemcpyAsync(hT_, dT_, n * sizeof(double), cudaMemcpyDeviceToHost, s));
      q(cudaMemcpyAsync(hP_, dP_, n * sizeof(double), cudaMemcpyDeviceToHost, s));
      q(cudaMemcpyAsync(hY_, dY_, (size_t)n * S * sizeof(double), cudaMemcpyDeviceToHost, s));
      q(cudaMemcpyAsync(hstats_, dstats_, n * sizeof(ReactorStats), cudaMemcpyDeviceToHost, s));
      if (a.t_ign) q(cudaMemcpyAsync(hign_, dign_, n * sizeof(double), cudaMemcpyDeviceToHost, s));
      cudaGraph_t g = nullptr;
      const cudaError_t ee = cudaStreamEndCapture(s, &g);
      if (ce == cudaSuccess) ce = ee;
      if (ce == cudaSuccess) ce = cudaGraphInstantiate(&graph_, g, 0);
      if (g) cudaGraphDestroy(g);
      if (ce != cudaSuccess) {
        graph_ = nullptr;
        last_error = std::string("graph capture: ") + cudaGetErrorString(ce);
        return -1;
      }
      graph_key_ = key;
      ++graph_captures;
    }
    if ((e = cudaGraphLaunch(graph_, s)) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess) {
      last_error = std::string("integration: ") + cudaGetErrorString(e);
      return -1;
    }
    ++graph_launches;
  }
  std::memcpy(T, hT_, n * sizeof(double));
  std::memcpy(P, hP_, n * sizeof(double));
  const ReactorStats *st = hstats_;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ev0_, ev1_) != cudaSuccess) {  // (the callback path records them too)
    ms = 0.f;
    (void)cudaGetLastError();  // timing only: leave no error for the next launch check
  }
  int nfail = 0;
  for (int r = 0; r < n; ++r) {
    const ReactorStats &q = st[r];
    if (q.status == 0) {
      std::memcpy(mf + (size_t)r * stride, &Y[(size_t)r * S], S * sizeof(double));
      // the root time of a reactor that integrated and crossed T0 + dT in
      // this call (zerork_reactor_manager.cpp:1128-1131 sets it only for
      // reactors that integrated); otherwise the caller's value stays
      if (t_ign && a.t_ign && hign_[r] >= 0.0) t_ign[r] = hign_[r];
      if (temp_delta) {
        double d = T[r] - T0[r];
        temp_delta[r] = (d < temp_threshold) ? 0.0 : d;
      }
    } else {
      ++nfail;
    }
    if (cost) cost[r] = q.status == 0 ? q.nsteps : -(double)std::max(1, q.nsteps);
    if (gpu_time) gpu_time[r] = ms * 1e-3 / n;
  }
  if (stats) stats->assign(st, st + n);
  if (tot) {
    *tot = SolveStatsTotals();
    for (int r = 0; r < n; ++r) {
      const ReactorStats &q = st[r];
      tot->nsteps += q.nsteps;
      tot->nrej += q.nrej;
      tot->nnewt += q.nnewt;
      tot->njac += q.njac;
      tot->nlu += q.nlu;
      tot->nrhs += q.nrhs;
      tot->nkry += q.nkry;
    }
    tot->nfailed = nfail;
    tot->kernel_ms = ms;
    tot->method = method;
    tot->groups = gcnt.groups;
    tot->group_steps = gcnt.group_steps;
    tot->group_newton = gcnt.group_newton;
    tot->launches = gcnt.launches;
    tot->syncs = gcnt.syncs;
    tot->group_status = gcnt.first_fail;
  }
  return nfail;
}

}  // namespace zrk
