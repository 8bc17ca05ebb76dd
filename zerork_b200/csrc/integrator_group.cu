// integrator_group.cu -- the plain FP64 GPU path: the reference GPU
// algorithm of the cfd_plugin, one BDF integration per group of reactors.
//
// The reference's GPU branch of SolveReactors
// (applications/cfd_plugin/zerork_reactor_manager.cpp:909-1054) cuts the
// cost-sorted reactors into groups of n_reactors_max (the last two split
// evenly, :933-940) and integrates each group with ONE CVODE instance over
// the stacked state vector of all its reactors (solver_cvode.cpp:52,
// reactor_nvector_serial_cuda.cu:56-59): one time step, one order and one
// WRMS norm for the whole group, the host running the step and Newton logic
// and every vector operation, right-hand side, Jacobian, factorization and
// solve being a kernel launch over the group with a host synchronization for
// every norm.  This file restates that architecture with this library's
// kernels and the same BDF as the batched integrators (Shampine-Reichelt
// quasi-constant-step BDF with CVODE's Newton test, step hysteresis, per-step
// failure limits and the plugin's retry loop), so that the batched
// integrators' gain over it measures per-reactor step control in one
// persistent launch, not a different method:
//   * the norms of the step-size selection, the Newton test and the error
//     test are RMS norms over all reactors' components;
//   * each reactor keeps its own Jacobian and Newton-matrix inverse (the
//     reference's batched cusolverRf factors, cusolver_rf_manager.cu:109-303),
//     formed and applied by one CTA per reactor;
//   * a failed attempt fails the group, which restarts from its last
//     accepted state under the retry loop; if every attempt fails, every
//     reactor of the group reports FAILED_SOLVE (zerork_reactor_manager.cpp:
//     1123-1125 marks a failed batch the same way).
// Supported: constant volume and constant pressure, DPDT and Y_SRC sources,
// fixed-temperature reactors and ignition times.  Not supported (the solver
// rejects them for this method): E_SRC, the step callback,
// stop_after_ignition, the FP32 factor and the learned predictor, which
// belong to the batched integrators.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "integrator_dense.cuh"
#include "integrator_group.h"

namespace zrk {
namespace {

constexpr int kHdr = 16;   // per-reactor header: v, T_prev, t_ign, pad, ReactorSrc at [8, 16)
constexpr int kPart = 6;   // partial sums per reactor: 4 sums, a failure flag, pad
static_assert(sizeof(ReactorSrc) <= 8 * sizeof(double), "ReactorSrc must fit the slot header");

struct GroupKArgs {
  DevMech m;
  IntegOpts o;
  const int *order;  // reactor indices in group order (device)
  int g0, n_group;   // this group: order[g0 .. g0 + n_group)
  double *slots;     // one slot of slot_stride doubles per group position
  long slot_stride;
  int lda;
  double *part;      // [n_group][kPart]
  const double *T, *P, *Y, *ysrc, *dpdt, *tdel_in;
};

// Per-reactor views into the reactor's global slot; rates workspace (C, G,
// U, rates of progress, reduction slots) in dynamic shared memory.
struct Bound {
  Smem s;
  double *hdr, *J, *A;
  int r;
};

__device__ Bound bind(const GroupKArgs &k, double *smem) {
  const DevMech &m = k.m;
  const int S = m.nsp, n = S + 1;
  Bound b;
  b.r = k.order[k.g0 + blockIdx.x];
  double *p = smem;
  Smem &s = b.s;
  s.red = p; p += 128;
  s.C = p; p += S;
  s.G = p; p += S;
  s.U = p; p += S;
  s.ROP = p; p += m.nstep;
  s.mlp = nullptr;
  s.Jsm = nullptr;
  s.V = nullptr;
  double *g = k.slots + (size_t)blockIdx.x * k.slot_stride;
  b.hdr = g; g += kHdr;
  s.y = g; g += n;
  s.f = g; g += n;
  s.f0 = g; g += n;
  s.ypred = g; g += n;
  s.psi = g; g += n;
  s.d = g; g += n;
  s.scale = g; g += n;
  s.tmp = g; g += n;
  s.yp = g; g += n;
  s.colk = g; g += n;
  s.wlu = g; g += n;
  s.bs = g; g += n;
  s.r1g = g; g += n;
  s.r1d = g; g += n;
  s.r1w = g; g += n;
  s.D = g; g += (kMaxOrder + 3) * n;
  b.J = g; g += (m.nnz + 1) & ~1;
  b.A = g; g += (size_t)n * k.lda;
  s.perm = (int *)g;
  s.A = b.A;
  s.src = *reinterpret_cast<const ReactorSrc *>(b.hdr + 8);
  s.ysrc = k.ysrc ? k.ysrc + (size_t)b.r * S : nullptr;
  return b;
}

__device__ __forceinline__ void put_part(const GroupKArgs &k, int i, double v) {
  if (threadIdx.x == 0) k.part[(size_t)blockIdx.x * kPart + i] = v;
}

__device__ __forceinline__ double atol_of(const DevMech &m, const IntegOpts &o, double v, double atol, int i) {
  return (o.abstol_dens && i < m.nsp) ? atol * (1.0 / ((1.0 / v) * m.inv_mw[i] * 1.0e-3)) : atol;
}

// x = (I - c J)^-1 b with the reactor's stored inverse in global memory:
// a warp per row, lanes over the columns (coalesced row reads).
__device__ void apply_inverse_g(const Smem &s, int n, int lda, const double *A, const double *b, double *x) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  for (int i = tid; i < n; i += nt) {
    const int pi = s.perm[i];
    s.bs[i] = b[pi] / s.wlu[pi];
  }
  __syncthreads();
  for (int i = w; i < n; i += nw) {
    const double *row = A + (size_t)i * lda;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += row[j] * s.bs[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane == 0) x[i] = acc * s.wlu[i];
  }
  __syncthreads();
}

// Newton-matrix inverse of the reactor at c into its slot: inverted in
// shared memory when the block fits (smem_A), else in place in global.
__device__ int factor_g(const GroupKArgs &k, Bound &b, double c, double *smem_A) {
  const int n = k.m.nsp + 1, nc = (n + 31) / 32;
  Smem s = b.s;
  if (smem_A) s.A = smem_A;
  const int bad = invert_any<double>(nc, k.m, s, b.J, c, n, k.lda);
  if (smem_A && !bad) {
    for (int i = threadIdx.x; i < n * k.lda; i += blockDim.x) b.A[i] = smem_A[i];
    __syncthreads();
  }
  return bad;
}

// ---- kernels: one CTA per reactor of the group

// Reactor set-up on the group's first attempt (the batched integrators'
// InitializeState): inverse density, sources, initial energy, y = [Y, T/Tref].
__global__ void __launch_bounds__(512) grp_init(GroupKArgs k) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const DevMech &m = k.m;
  const int S = m.nsp, tid = threadIdx.x, nt = blockDim.x, r = b.r;
  Smem &s = b.s;
  const double T0 = k.T[r], P0 = k.P[r];
  const double *Y0 = k.Y + (size_t)r * S;
  double pa = 0.0;
  for (int i = tid; i < S; i += nt) pa += Y0[i] * m.inv_mw[i];
  const double mwmix = 1.0 / block_sum(pa, s.red);
  const double v = 1.0 / (P0 * mwmix / (kRuD * T0));
  ReactorSrc src;
  src.dpdt = k.dpdt ? k.dpdt[r] : 0.0;
  src.esrc = 0.0;
  src.P0 = P0;
  src.ysrc = k.ysrc != nullptr;
  src.fixT = !k.o.always_T && k.tdel_in && !(k.tdel_in[r] > 0.0);
  src.T0 = T0;
  src.E0 = 0.0;
  if (src.fixT) {
    double cx;
    mix_energy(m, k.o.cp != 0, false, T0, Y0, false, 0.0, tid, nt,
               [&](double x) { return block_sum(x, s.red); }, src.E0, cx);
  }
  for (int i = tid; i < S; i += nt) s.y[i] = Y0[i];
  if (tid == 0) {
    s.y[S] = T0 / k.o.Tref;
    b.hdr[0] = v;
    b.hdr[2] = -1.0;  // ignition time: not reached
    *reinterpret_cast<ReactorSrc *>(b.hdr + 8) = src;
  }
}

// Start of an attempt from y at t_off: f0 = ydot(y), the error weights, and
// the partial sums of the initial step-size estimate (|y|_w^2, |f0|_w^2).
__global__ void __launch_bounds__(512) grp_begin(GroupKArgs k, double t_off, double rtol, double atol) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const DevMech &m = k.m;
  const int n = m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  Smem &s = b.s;
  const double v = b.hdr[0];
  const int bad = rhs_cta(m, k.o, s, v, t_off, s.y, s.f0, false, nullptr);
  double a0 = 0.0, a1 = 0.0;
  for (int i = tid; i < n; i += nt) {
    const double sc = atol_of(m, k.o, v, atol, i) + fabs(s.y[i]) * rtol;
    s.scale[i] = sc;
    a0 += (s.y[i] / sc) * (s.y[i] / sc);
    a1 += (s.f0[i] / sc) * (s.f0[i] / sc);
  }
  a0 = block_sum(a0, s.red);
  a1 = block_sum(a1, s.red);
  if (tid == 0) b.hdr[1] = s.y[m.nsp] * k.o.Tref;  // temperature at the last accepted step
  put_part(k, 0, a0);
  put_part(k, 1, a1);
  put_part(k, 4, bad ? 1.0 : 0.0);
}

// Second-derivative probe of the initial step: f(y + h0 f0) - f0.
__global__ void __launch_bounds__(512) grp_probe(GroupKArgs k, double t_abs, double h0) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const int n = k.m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  Smem &s = b.s;
  for (int i = tid; i < n; i += nt) s.tmp[i] = s.y[i] + h0 * s.f0[i];
  __syncthreads();
  const int bad = rhs_cta(k.m, k.o, s, b.hdr[0], t_abs, s.tmp, s.f, false, nullptr);
  double a = 0.0;
  if (!bad)
    for (int i = tid; i < n; i += nt) {
      const double t = (s.f[i] - s.f0[i]) / s.scale[i];
      a += t * t;
    }
  a = block_sum(a, s.red);
  put_part(k, 2, a);
  put_part(k, 4, bad ? 1.0 : 0.0);
}

// History D = [y, h f0, 0...], Jacobian at (t_off, y) and the inverse at c.
__global__ void __launch_bounds__(512) grp_start(GroupKArgs k, double t_off, double h, double c, int fac_smem) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const int n = k.m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  Smem &s = b.s;
  for (int i = tid; i < (kMaxOrder + 3) * n; i += nt) s.D[i] = 0.0;
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    s.D[i] = s.y[i];
    s.D[n + i] = s.f0[i] * h;
  }
  __syncthreads();
  int bad = jac_cta(k.m, k.o, s, b.hdr[0], t_off, s.y, s.f0, b.J);
  if (!bad) bad = factor_g(k, b, c, fac_smem ? smem + 128 + 3 * k.m.nsp + k.m.nstep : nullptr);
  put_part(k, 4, bad ? 1.0 : 0.0);
}

__global__ void __launch_bounds__(512) grp_change(GroupKArgs k, int q, double fac) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  change_D_cta(b.s.D, k.m.nsp + 1, q, fac);
}

// Predictor of a step of order q: ypred = sum D_k, psi, error weights.
__global__ void __launch_bounds__(512) grp_predict(GroupKArgs k, int q, double rtol, double atol, Consts bc) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const int n = k.m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  Smem &s = b.s;
  const double v = b.hdr[0];
  for (int i = tid; i < n; i += nt) {
    double a = 0.0, ps = 0.0;
    for (int j = 0; j <= q; ++j) a += s.D[j * n + i];
    for (int j = 1; j <= q; ++j) ps += bc.gam[j] * s.D[j * n + i];
    s.ypred[i] = a;
    s.psi[i] = ps / bc.alp[q];
    s.scale[i] = atol_of(k.m, k.o, v, atol, i) + rtol * fabs(a);
    s.y[i] = a;
    s.d[i] = 0.0;
  }
}

// New inverse at c; with jac, first a fresh Jacobian at (t_abs, ypred).
__global__ void __launch_bounds__(512) grp_factor(GroupKArgs k, double t_abs, double c, int jac, int fac_smem) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  Smem &s = b.s;
  int bad = 0;
  if (jac) {
    bad = rhs_cta(k.m, k.o, s, b.hdr[0], t_abs, s.ypred, s.f0, false, nullptr);
    if (!bad) bad = jac_cta(k.m, k.o, s, b.hdr[0], t_abs, s.ypred, s.f0, b.J);
  }
  if (!bad) bad = factor_g(k, b, c, fac_smem ? smem + 128 + 3 * k.m.nsp + k.m.nstep : nullptr);
  put_part(k, 4, bad ? 1.0 : 0.0);
}

// One Newton iteration at t_abs: partial sums of the correction's and of
// the accumulated correction's (error estimate's) weighted squares.
__global__ void __launch_bounds__(512) grp_newton(GroupKArgs k, double t_abs, double c, double gs, int first,
                                                  double econ) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const int n = k.m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  Smem &s = b.s;
  int bad = rhs_cta(k.m, k.o, s, b.hdr[0], t_abs, s.y, s.f, false, nullptr);
  if (!bad) {
    int nf = 0;
    for (int i = tid; i < n; i += nt) nf |= !isfinite(s.f[i]);
    bad = __syncthreads_or(nf);
  }
  double a0 = 0.0, a1 = 0.0;
  if (!bad) {
    for (int i = tid; i < n; i += nt) {
      if (first) s.f0[i] = s.f[i];
      s.tmp[i] = c * s.f[i] - s.psi[i] - s.d[i];
    }
    __syncthreads();
    apply_inverse_g(s, n, k.lda, b.A, s.tmp, s.yp);
    for (int i = tid; i < n; i += nt) {
      const double dy = s.yp[i] * gs;
      s.y[i] += dy;
      s.d[i] += dy;
      const double t = dy / s.scale[i], e = econ * s.d[i] / s.scale[i];
      a0 += t * t;
      a1 += e * e;
    }
  }
  a0 = block_sum(a0, s.red);
  a1 = block_sum(a1, s.red);
  put_part(k, 0, a0);
  put_part(k, 1, a1);
  put_part(k, 4, bad ? 1.0 : 0.0);
}

// Order 1 after repeated error-test failures: D1 = f(t_abs, D0) * heta.
__global__ void __launch_bounds__(512) grp_reload(GroupKArgs k, double t_abs, double heta) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const int n = k.m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  Smem &s = b.s;
  const int bad = rhs_cta(k.m, k.o, s, b.hdr[0], t_abs, s.D, s.tmp, false, nullptr);
  if (!bad)
    for (int i = tid; i < n; i += nt) s.D[n + i] = s.tmp[i] * heta;
  put_part(k, 4, bad ? 1.0 : 0.0);
}

// Accepted step of order q ending at t_abs: history update, ignition
// crossing, and the partial sums of the order-change estimates.
__global__ void __launch_bounds__(512) grp_accept(GroupKArgs k, int q, double t_abs, double h, Consts bc) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const int n = k.m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  Smem &s = b.s;
  for (int i = tid; i < n; i += nt) {
    const double di = s.d[i];
    s.D[(q + 2) * n + i] = di - s.D[(q + 1) * n + i];
    s.D[(q + 1) * n + i] = di;
    for (int j = q; j >= 0; --j) s.D[j * n + i] += s.D[(j + 1) * n + i];
  }
  __syncthreads();
  if (k.o.dT_ign > 0.0 && tid == 0) {  // first crossing of T0 + dT_ign, linear between accepted steps
    const double Tn = s.D[n - 1] * k.o.Tref, Tp = b.hdr[1];
    const double target = s.src.T0 + k.o.dT_ign;
    if (b.hdr[2] < 0.0 && Tn >= target) {
      const double frac = (Tn > Tp) ? (target - Tp) / (Tn - Tp) : 1.0;
      b.hdr[2] = (t_abs - h) + frac * h;
    }
    b.hdr[1] = Tn;
  }
  double am = 0.0, ap = 0.0;
  for (int i = tid; i < n; i += nt) {
    if (q > 1) {
      const double e = bc.econ[q - 1] * s.D[q * n + i] / s.scale[i];
      am += e * e;
    }
    if (q < kMaxOrder) {
      const double e = bc.econ[q + 1] * s.D[(q + 2) * n + i] / s.scale[i];
      ap += e * e;
    }
  }
  am = block_sum(am, s.red);
  ap = block_sum(ap, s.red);
  put_part(k, 2, am);
  put_part(k, 3, ap);
}

// End of an attempt: y = the last accepted state (D0).
__global__ void __launch_bounds__(512) grp_restore(GroupKArgs k) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const int n = k.m.nsp + 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) b.s.y[i] = b.s.D[i];
}

// Results of the group: state, temperature, pressure, statistics.
__global__ void __launch_bounds__(512) grp_finish(GroupKArgs k, double dt, ReactorStats st, double *T,
                                                  double *P, double *Y, double *v_out, ReactorStats *stats,
                                                  double *t_ign) {
  extern __shared__ double smem[];
  Bound b = bind(k, smem);
  const DevMech &m = k.m;
  const int S = m.nsp, tid = threadIdx.x, nt = blockDim.x, r = b.r;
  Smem &s = b.s;
  const double v = b.hdr[0];
  if (st.status == 0) {
    double pb = 0.0;
    for (int i = tid; i < S; i += nt) {
      Y[(size_t)r * S + i] = s.y[i];
      pb += s.y[i] * m.inv_mw[i];
    }
    const double mw2 = 1.0 / block_sum(pb, s.red);
    const double Tn = end_temperature(m, k.o.cp != 0, s.src, dt, s.y, s.y[S] * k.o.Tref, tid, nt,
                                      [&](double x) { return block_sum(x, s.red); });
    if (tid == 0) {
      T[r] = Tn;
      P[r] = end_pressure(k.o.cp != 0, s.src, dt, Tn, mw2, v);
    }
  }
  if (tid == 0) {
    v_out[r] = v;
    if (stats) stats[r] = st;
    if (t_ign) t_ign[r] = b.hdr[2];
  }
}

// ---- host driver of one group

struct GroupDriver {
  GroupKArgs k;
  int threads;
  size_t smem, smem_fac;
  int fac_smem;
  cudaStream_t st;
  double *part_h;
  Consts bc;
  long launches = 0, syncs = 0;
  bool started = false;  // this attempt has set up the BDF history
  ReactorStats cnt{};

  cudaError_t sync_parts() {
    ++syncs;
    cudaError_t e = cudaMemcpyAsync(part_h, k.part, (size_t)k.n_group * kPart * sizeof(double),
                                    cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
  }
  // group RMS of partial sum i over n_group * n components
  double norm(int i) const {
    double a = 0.0;
    for (int g = 0; g < k.n_group; ++g) a += part_h[(size_t)g * kPart + i];
    return std::sqrt(a / ((double)k.n_group * (k.m.nsp + 1)));
  }
  bool any_bad() const {
    for (int g = 0; g < k.n_group; ++g)
      if (part_h[(size_t)g * kPart + 4] != 0.0) return true;
    return false;
  }
  template <class... KA, class... Args>
  cudaError_t go(void (*kern)(GroupKArgs, KA...), bool fac, Args... args) {
    ++launches;
    kern<<<k.n_group, threads, fac ? smem_fac : smem, st>>>(k, args...);
    return cudaGetLastError();
  }

  // One attempt over [t_off, t_off + t_end): returns 0 or a negative status
  // (as the batched integrators); -100 with e set on a CUDA error.
  int attempt(double t_off, double t_end, double rtol, double atol, double &t_done, cudaError_t &e) {
    const IntegOpts &o = k.o;
    t_done = 0.0;
    started = false;
#define GO(...) \
  if ((e = go(__VA_ARGS__)) != cudaSuccess) return -100
#define SYNC() \
  if ((e = sync_parts()) != cudaSuccess) return -100
    cnt.nrhs++;
    GO(grp_begin, false, t_off, rtol, atol);
    SYNC();
    if (any_bad()) return -1;
    const double d0 = norm(0), d1 = norm(1);
    double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
    if (h0 > t_end) h0 = t_end;
    cnt.nrhs++;
    GO(grp_probe, false, t_off + h0, h0);
    SYNC();
    const double d2 = any_bad() ? 0.0 : norm(2) / h0;
    double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? std::fmax(1e-6, h0 * 1e-3) : std::sqrt(0.01 / std::fmax(d1, d2));
    double h = std::fmin(100.0 * h0, h1);
    h = std::fmin(h, o.max_dt);
    h = std::fmin(h, t_end);
    int q = 1, neq = 0, jac_current = 1, nsteps = 0;
    double c_lu = h / bc.alp[q], crate = 1.0, t = 0.0;
    cnt.njac++;
    cnt.nlu++;
    GO(grp_start, true, t_off, h, c_lu, fac_smem);
    started = true;
    SYNC();
    if (any_bad()) return -2;
    auto change = [&](int qq, double fac) -> cudaError_t {
      if (fac == 1.0) return cudaSuccess;
      return go(grp_change, false, qq, fac);
    };
    while (t < t_end) {
      if (nsteps >= o.max_steps) return -4;
      bool accepted = false;
      double safety = 0.9, err_norm = 0.0;
      int nef = 0, ncf = 0;
      while (!accepted) {
        if (h > o.max_dt) {
          if ((e = change(q, o.max_dt / h)) != cudaSuccess) return -100;
          h = o.max_dt;
        }
        if (t + h > t_end) {
          if ((e = change(q, (t_end - t) / h)) != cudaSuccess) return -100;
          h = t_end - t;
        }
        if (!(t + h > t)) return -5;
        const double t_new = t + h;
        GO(grp_predict, false, q, rtol, atol, bc);
        const double c = h / bc.alp[q];
        if (std::fabs(c / c_lu - 1.0) > 0.3) {
          cnt.nlu++;
          c_lu = c;
          crate = 1.0;
          GO(grp_factor, true, t_off + t_new, c, 0, fac_smem);
          SYNC();
          if (any_bad()) return -3;
        }
        const double gscale = (c == c_lu) ? 1.0 : 2.0 / (1.0 + c / c_lu);
        bool conv = false;
        int it;
        double dnorm_old = -1.0;
        for (it = 0; it < kNewtonMaxIter; ++it) {
          cnt.nrhs++;
          GO(grp_newton, false, t_off + t_new, c, gscale, it == 0 ? 1 : 0, bc.econ[q]);
          SYNC();
          if (any_bad()) break;
          cnt.nnewt++;
          const double dn = norm(0);
          err_norm = norm(1);
          if (dnorm_old > 0.0) crate = std::fmax(0.3 * crate, dn / dnorm_old);
          if (bc.econ[q] * dn * std::fmin(1.0, crate) <= o.nlscoef) {
            conv = true;
            ++it;
            break;
          }
          if (dnorm_old > 0.0 && dn > 2.0 * dnorm_old) break;
          dnorm_old = dn;
        }
        if (!conv) {
          if (!jac_current) {
            cnt.nrhs++;
            cnt.njac++;
            cnt.nlu++;
            jac_current = 1;
            c_lu = c;
            crate = 1.0;
            GO(grp_factor, true, t_off + t_new, c, 1, fac_smem);
            SYNC();
            if (any_bad()) return -2;
            continue;
          }
          if (++ncf >= kMaxConvFails) return -8;
          if ((e = change(q, 0.5)) != cudaSuccess) return -100;
          h *= 0.5;
          cnt.nrej++;
          continue;
        }
        safety = 0.9 * (2 * kNewtonMaxIter + 1) / (2.0 * kNewtonMaxIter + it);
        if (!std::isfinite(err_norm)) return -7;
        if (err_norm > 1.0) {
          if (++nef >= kMaxErrTestFails) return -9;
          cnt.nrej++;
          if (nef > kErrFailsBeforeCut) {
            if (q > 1) {
              --q;
              if ((e = change(q, kEtaMinErrFail)) != cudaSuccess) return -100;
            } else {
              cnt.nrhs++;
              GO(grp_reload, false, t_off + t, h * kEtaMinErrFail);
              SYNC();
              if (any_bad()) return -6;
            }
            h *= kEtaMinErrFail;
            neq = 0;
            continue;
          }
          const double fac = std::fmax(kMinFactor, safety * std::pow(err_norm, -1.0 / (q + 1)));
          if ((e = change(q, fac)) != cudaSuccess) return -100;
          h *= fac;
          continue;
        }
        accepted = true;
        t = t_new;
      }
      ++nsteps;
      cnt.nsteps++;
      ++neq;
      jac_current = 0;
      t_done = t;
      GO(grp_accept, false, q, t_off + t, h, bc);
      if (neq < q + 1) continue;
      SYNC();
      const double em = q > 1 ? norm(2) : INFINITY, ep = q < kMaxOrder ? norm(3) : INFINITY;
      const double fm = (q > 1) ? std::pow(em, -1.0 / q) : 0.0;
      const double f0 = std::pow(err_norm, -1.0 / (q + 1));
      const double fp = (q < kMaxOrder) ? std::pow(ep, -1.0 / (q + 2)) : 0.0;
      int dq = 0;
      double best = f0;
      if (fm > best) { best = fm; dq = -1; }
      if (fp > best) { best = fp; dq = 1; }
      q += dq;
      double fac = std::fmin(kMaxFactor, safety * best);
      if (fac < kEtaKeep) fac = 1.0;
      if ((e = change(q, fac)) != cudaSuccess) return -100;
      h *= fac;
      neq = 0;
    }
#undef GO
#undef SYNC
    return 0;
  }
};

}  // namespace

size_t group_slot_doubles(const DevMech &m) {
  const int n = m.nsp + 1, lda = (n % 2 == 1) ? n : n + 1;
  const size_t d = kHdr + 15 * (size_t)n + (kMaxOrder + 3) * (size_t)n + ((m.nnz + 1) & ~1) +
                   (size_t)n * lda + ((n + 1) / 2 + 1);
  return (d + 31) & ~size_t(31);  // 256-byte slots
}

int group_sizes(int n, int group_max, std::vector<int> &sizes) {
  sizes.clear();
  int left = n;
  while (left > 0) {
    int cur = std::min(left, group_max);
    // zerork_reactor_manager.cpp:935-939: the last two groups split evenly
    if (cur != left && left < 2 * group_max && cur == group_max) cur = left / 2;
    sizes.push_back(cur);
    left -= cur;
  }
  return (int)sizes.size();
}

cudaError_t integrate_group(const DevMech &m, const IntegOpts &o, const IntegArgs &a, const int *order_dev,
                            int group_max, int threads, double *slots, double *part_dev,
                            double *part_host, cudaStream_t stream, GroupCounters *gc) {
  const int S = m.nsp, n = S + 1;
  const int lda = (n % 2 == 1) ? n : n + 1;
  if (n > kDenseMaxN) return cudaErrorInvalidValue;
  GroupDriver drv;
  std::memset(&drv.k, 0, sizeof(drv.k));
  drv.k.m = m;
  drv.k.o = o;
  drv.k.order = order_dev;
  drv.k.slots = slots;
  drv.k.slot_stride = (long)group_slot_doubles(m);
  drv.k.lda = lda;
  drv.k.part = part_dev;
  drv.k.T = a.T;
  drv.k.P = a.P;
  drv.k.Y = a.Y;
  drv.k.ysrc = a.ysrc;
  drv.k.dpdt = a.dpdt;
  drv.k.tdel_in = a.tdel_in;
  drv.threads = threads;
  drv.st = stream;
  drv.part_h = part_host;
  make_consts(drv.bc);
  drv.smem = (128 + 3 * (size_t)S + m.nstep) * sizeof(double);
  const size_t kSmemMax = 227 * 1024;
  drv.smem_fac = drv.smem + (size_t)n * lda * sizeof(double);
  drv.fac_smem = drv.smem_fac <= kSmemMax ? 1 : 0;
  if (!drv.fac_smem) drv.smem_fac = drv.smem;
  if (drv.smem > kSmemMax) return cudaErrorInvalidValue;
  cudaError_t e;
  // every kernel may use up to smem_fac of dynamic shared memory
  const void *all[] = {(const void *)grp_init, (const void *)grp_begin, (const void *)grp_probe,
                       (const void *)grp_start, (const void *)grp_change, (const void *)grp_predict,
                       (const void *)grp_factor, (const void *)grp_newton, (const void *)grp_reload,
                       (const void *)grp_accept, (const void *)grp_restore, (const void *)grp_finish};
  for (const void *f : all)
    if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)std::max(drv.smem, drv.smem_fac))) != cudaSuccess)
      return e;
  std::vector<int> sizes;
  group_sizes(a.n_reactors, group_max, sizes);
  int g0 = 0;
  for (int gs : sizes) {
    drv.k.g0 = g0;
    drv.k.n_group = gs;
    drv.cnt = ReactorStats{0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if ((e = drv.go(grp_init, false)) != cudaSuccess) return e;
    double rtol = o.rtol, atol = o.atol, t_left = a.dt;
    int rc = 0;
    for (int attempt = 0;; ++attempt) {
      double t_done = 0.0;
      e = cudaSuccess;
      rc = drv.attempt(a.dt - t_left, t_left, rtol, atol, t_done, e);
      if (rc == -100) return e;
      // y = the last accepted state (D0), unless the attempt failed before
      // it set up its history (y is then still the attempt's start)
      if (drv.started && (e = drv.go(grp_restore, false)) != cudaSuccess) return e;
      if (rc == 0) break;
      if (attempt + 1 >= o.max_retries) break;
      t_left -= t_done;
      drv.cnt.retries++;
      atol *= o.retry_atol_factor;
      rtol *= o.retry_rtol_factor;
    }
    drv.cnt.status = rc;
    if ((e = drv.go(grp_finish, false, a.dt, drv.cnt, a.T, a.P, a.Y, a.v, a.stats, a.t_ign)) != cudaSuccess)
      return e;
    if (gc) {
      gc->groups++;
      gc->group_steps += drv.cnt.nsteps;
      gc->group_newton += drv.cnt.nnewt;
      if (rc != 0 && gc->first_fail == 0) gc->first_fail = rc;
    }
    g0 += gs;
  }
  if (gc) {
    gc->launches += drv.launches;
    gc->syncs += drv.syncs;
  }
  return cudaStreamSynchronize(stream);
}

}  // namespace zrk
