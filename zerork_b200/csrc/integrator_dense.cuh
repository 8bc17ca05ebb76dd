// integrator_dense.cuh -- CTA-per-reactor BDF integration with the Newton
// matrix held as one dense block in shared memory.
//
// The symbolic factorization of the reactor Newton matrix P = I - cJ
// (sparse_lu.h) fills 64-100 % of the dense n x n block for the benchmark
// mechanisms, so the factor is handled as a single dense supernode: P is
// inverted in shared memory by Gauss-Jordan elimination with partial
// pivoting, and every Newton solve is a parallel matrix-vector product.  A
// persistent CTA takes reactors from the work queue; the reactor's BDF state
// (differences, iterate, right-hand sides, weights) and the rate workspace
// live in shared memory, the reactor Jacobian in global memory.  Step
// control is the same as integrator.cu (Shampine-Reichelt BDF with CVODE's
// Newton test and step hysteresis).
#pragma once
#include <cuda_runtime.h>

#include "integrator.h"
#include "kinetics_dev.cuh"
#include "reactor_src.cuh"

namespace zrk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kNewtonMaxIter = 3;
constexpr double kMinFactor = 0.2;
constexpr double kMaxFactor = 10.0;
constexpr double kEtaKeep = 1.5;
constexpr int kMaxl = 10;  // Krylov dimension (no restarts)
constexpr int kPredBuf = 256;  // widest predictor layer (padded)

struct Smem {
  double *red;  // 128 slots: block sums [0, 33), pivot candidates [64, 112)
  double *C, *G, *U, *ROP;
  double *D, *y, *f, *f0, *ypred, *psi, *d, *scale, *tmp, *yp;
  void *A;      // n x lda inverse (LT)
  int *perm;    // n: row i of the factored matrix is scaled row perm[i]
  double *colk; // n (LT-sized use)
  double *wlu;  // n: error-weight scale the stored inverse was formed with
  double *bs;   // n: scaled right-hand side
  double *V;    // FP32 path: (kMaxl + 1) Krylov vectors, then 2 work vectors
  float *mlp;   // learned predictor: two activation buffers of kPredBuf floats
  double *Jsm;  // reactor Jacobian when it is kept in shared memory (spill bit 4)
  const double *ysrc;  // this reactor's mass-fraction sources (global) or null
  ReactorSrc src;      // this reactor's pressure-rate / energy sources and initial state
  // energy-source temperature coupling (global, n each): g = df/dT*,
  // d = dT*/dY, w = (I - c J)^-1 g of the current factor
  double *r1g, *r1d, *r1w;
};

// What one right-hand-side evaluation used: mixture heat capacity (c_v, or
// c_p for constant pressure), temperature and inverse density.
struct RhsOut {
  double cx, T, v;
};

// Sum over the CTA; every thread gets thread 0's total (deterministic).
__device__ __forceinline__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < nw; ++i) s += red[i];
    red[32] = s;
  }
  __syncthreads();
  return red[32];
}

__device__ __forceinline__ double gather4(const double *v, const int *idx, int q0, int q1) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int q = q0;
  for (; q + 3 < q1; q += 4) {
    const int i0 = idx[q], i1 = idx[q + 1], i2 = idx[q + 2], i3 = idx[q + 3];
    a0 += v[i0];
    a1 += v[i1];
    a2 += v[i2];
    a3 += v[i3];
  }
  for (; q < q1; ++q) a0 += v[idx[q]];
  return (a0 + a1) + (a2 + a3);
}

// Source / constant-pressure adjustment of T and v (reactor_src.cuh).
__device__ __forceinline__ void source_cta(const DevMech &m, const IntegOpts &o, const Smem &s,
                                           double t, const double *y, bool clamp, double v0,
                                           double T_force, double &T, double &v) {
  source_T_v(m, o.cp != 0, s.src, t, y, clamp, o.mmf, v0, T_force, threadIdx.x, blockDim.x,
             [&](double x) { return block_sum(x, s.red); }, T, v);
}

// ydot at y (shared vector) and time t from the start of the call; v0 is the
// reactor's initial inverse density.  Returns 1 if T <= 0 (all threads agree).
// Constant volume: reactor_constant_volume_cpu.cpp:64-128; constant pressure
// (o.cp): reactor_constant_pressure_cpu.cpp:71-135, U then holds h/RT.
// T_force > 0 replaces the energy-source temperature.
__device__ __noinline__ int rhs_cta(const DevMech &m, const IntegOpts &o, const Smem &s,
                                       double v0, double t, const double *y, double *ydot,
                                       bool clamp, RhsOut *out, double T_force = 0.0) {
  const int S = m.nsp, tid = threadIdx.x, nt = blockDim.x;
  const double yS = y[S];
  double T = s.src.fixT ? s.src.T0 : yS * o.Tref;
  if (!(T > 0.0)) return 1;
  if (T > 1.0e4) T = 1.0e4;
  double v = v0;
  if (o.cp || s.src.dpdt != 0.0 || s.src.esrc != 0.0)
    source_cta(m, o, s, t, y, clamp, v0, T_force, T, v);
  const double logT = log(T), invT = 1.0 / T, lprt = log(kPatmD / (kRuD * T));
  const double dens = 1.0 / v;
  const double ush = o.cp ? 0.0 : 1.0;  // h/RT - 1 = u/RT; c_p/R - 1 = c_v/R
  double pc = 0.0, pcv = 0.0;
  for (int k = tid; k < S; k += nt) {
    double ys = y[k];
    if (clamp) ys = clamp_mass_fraction(ys, o.mmf);
    const double c = dens * m.inv_mw[k] * ys;
    s.C[k] = c;
    double cp, h, g;
    nasa_cp_h_g(m.thermo + 16 * k, T, logT, &cp, &h, &g);
    s.G[k] = g;
    s.U[k] = h - ush;
    pc += c;
    pcv += ((cp - ush) * m.ru_inv_mw[k]) * ys;
  }
  const double Csum = block_sum(pc, s.red);
  const double cv = block_sum(pcv, s.red);
  // reactions by decreasing cost in snake order over the threads
  for (int rr = 0; rr * nt < m.nrxn; ++rr) {
    const int pos = rr * nt + ((rr & 1) ? nt - 1 - tid : tid);
    if (pos < m.nrxn)
      reaction_item<1, 1>(m, load_rxn(m.rxn_by_cost + pos), 0, s.C, s.G, s.ROP, &T, &logT, &invT, &lprt, &Csum,
                          o.lim);
  }
  __syncthreads();
  double pe = 0.0;
  for (int k = tid; k < S; k += nt) {
    // four independent partial sums per list keep several rate loads in
    // flight (the rates of progress may sit in L2)
    const double des = gather4(s.ROP, m.sd_step, m.sd_ptr[k], m.sd_ptr[k + 1]);
    const double cre = gather4(s.ROP, m.sc_step, m.sc_ptr[k], m.sc_ptr[k + 1]);
    const double net = cre - des;
    if (s.ysrc) {  // reactor_constant_volume_cpu.cpp:108-113
      const double ys = s.ysrc[k];
      ydot[k] = net * m.mw[k] * v + ys;
      pe += s.U[k] * (net * v + ys * m.inv_mw[k]);
    } else {
      ydot[k] = net * m.mw[k] * v;
      pe += s.U[k] * net * v;
    }
  }
  const double es = block_sum(pe, s.red);
  if (tid == 0)
    ydot[S] = s.src.fixT ? 0.0 : -es * kRuD * yS / cv + (s.src.esrc + s.src.dpdt * v) / (cv * o.Tref);
  if (out) *out = RhsOut{cv, T, v};
  __syncthreads();
  return 0;
}

// Reactor Jacobian (SetupJacobianSparse semantics) into J (global, nnz) at
// y with fy = ydot(t, y).  The concentration derivatives use the reactor's
// inverse density: the initial one at constant volume, the current one at
// constant pressure; the temperature row uses the heat capacities at the
// temperature the right-hand side used.  Under an energy source the
// right-hand side takes T from the energy, T* = T(E0 + esrc t, Y), which
// this Jacobian does not see; the rank-one coupling g d^T (g = df/dT*,
// d_j = dT*/dY_j = -e_j / c_x) goes to s.r1g / s.r1d for the Newton solves.
__device__ __noinline__ int jac_cta(const DevMech &m, const IntegOpts &o, const Smem &s,
                                       double v0, double t, const double *y, const double *fy,
                                       double *J) {
  const int S = m.nsp, n = S + 1, tid = threadIdx.x, nt = blockDim.x;
  int need = 0;
  for (int k = tid; k < S; k += nt) need |= (fabs(y[k]) < o.mmf);
  need = __syncthreads_or(need);
  RhsOut ro;
  if (rhs_cta(m, o, s, v0, t, y, s.tmp, need != 0, &ro)) return 1;
  const double TdC = s.tmp[S];
  const double yS = y[S];
  const double RuTemp = kRuD * yS;
  const double multFact = -1.0 / ro.cx;
  const double T = ro.T, v = o.cp ? ro.v : v0;
  const double ush = o.cp ? 0.0 : 1.0;
  for (int jj = tid; jj < S; jj += nt) {  // one column per thread, costliest first
    const int j = m.col_order[jj];
    const double t2 = m.mw[j] / clamp_mass_fraction(y[j], o.mmf) * v;
    const int k0 = m.col_ptr[j], k1 = m.col_ptr[j + 1] - 1;
    const double wcol = m.inv_mw[j];
    double trow = 0.0;
    for (int kk = k0; kk < k1; ++kk) {
      const int row = m.row_idx[kk];
      const double des = gather4(s.ROP, m.nzd_step, m.nzd_ptr[kk], m.nzd_ptr[kk + 1]);
      const double cre = gather4(s.ROP, m.nzc_step, m.nzc_ptr[kk], m.nzc_ptr[kk + 1]);
      const double val = (0.0 - des * t2) + cre * t2;
      trow += val * s.U[row];
      J[kk] = val * (m.mw[row] * wcol);
    }
    const double cvj = (nasa_cp(m.thermo + 16 * j, T) - ush) * m.ru_inv_mw[j];
    double tr = trow * RuTemp;
    tr += TdC * cvj * m.mw[j];
    tr *= wcol * multFact;
    J[k1] = s.src.fixT ? 0.0 : tr;  // no temperature row when T is not solved
  }
  __syncthreads();
  const double ySp = yS + yS * o.sqrt_ur;
  const double mult = 1.0 / (ySp - yS);
  for (int k = tid; k < S; k += nt) s.yp[k] = y[k];
  if (tid == 0) s.yp[S] = ySp;
  __syncthreads();
  if (rhs_cta(m, o, s, v0, t, s.yp, s.tmp, false, nullptr)) return 1;
  for (int kk = m.col_ptr[S] + tid; kk < m.col_ptr[S + 1]; kk += nt) {
    const int row = m.row_idx[kk];
    J[kk] = (s.tmp[row] - fy[row]) * mult;
  }
  __syncthreads();
  if (s.src.esrc != 0.0) {
    RhsOut r1;
    if (rhs_cta(m, o, s, v0, t, y, s.yp, false, &r1)) return 1;
    for (int j = tid; j < S; j += nt) {
      double cpR, hRT;
      nasa_cp_h(m.thermo + 16 * j, r1.T, &cpR, &hRT);
      s.r1d[j] = -((hRT - ush) * (m.ru_inv_mw[j] * r1.T)) / r1.cx;
    }
    if (tid == 0) s.r1d[S] = 0.0;
    const double Tp = r1.T + r1.T * o.sqrt_ur;
    if (rhs_cta(m, o, s, v0, t, y, s.tmp, false, nullptr, Tp)) return 1;
    for (int i = tid; i < n; i += nt) s.r1g[i] = (s.tmp[i] - s.yp[i]) / (Tp - r1.T);
    __syncthreads();
  }
  return 0;
}

// Newton matrix inverse in shared memory, formed in error-weight-scaled
// coordinates: Pw = W^-1 (I - cJ) W with W = diag(scale), scale = atol +
// rtol |y| of the current step, so entry (i, j) is P_ij scale_j / scale_i,
// the Jacobian of relative changes.  It is far better balanced than P for
// species spanning 20 decades of mass fraction and keeps the inverse
// accurate in the weighted norm the Newton test uses.
//
// Gauss-Jordan with partial pivoting, in place, two pivots per sweep of the
// matrix.  Row interchanges are accumulated in perm (row i of the factored
// matrix is row perm[i] of Pw), so A ends as (Pi Pw)^-1 = Pw^-1 Pi^T and the
// right-hand side is permuted on application instead of unswapping columns.
// Per pair of pivots (k, k+1), four barriers:
//   S1  pick pivot k from the per-warp candidates (every thread makes the
//       same choice), swap rows, scaled pivot row r1 (kept in colk);
//   C   column k+1 as it will be after eliminating column k,
//       g_i = a_i[k+1] - a_i[k] r1[k+1], gives the candidates for pivot k+1
//       (each carries its a_i[k]);
//   S2  pick pivot k+1, swap the raw rows, r2 = scaled (a_{k+1} - a_{k+1}[k]
//       r1), row k becomes r1 - r1[k+1] r2;
//   U   every other row in one pass, a_i - a_i[k] r1 - g_i r2 (columns k and
//       k+1 get their Gauss-Jordan values from the lanes that own them), warp
//       w owning rows i = w (mod warps), two rows per pass with every load
//       issued before the stores, lane l the columns l (mod 32) with r1 and
//       r2 in registers; it leaves the candidates for column k+2.
// A lone last pivot is swept on its own.  Returns nonzero (all threads) for a
// singular or non-finite matrix.
__device__ __forceinline__ void track(double &ca, int &ci, double &cv, double &cf, double a, int i, double f) {
  const double d = fabs(a);
  if (d > ca) {
    ca = d;
    ci = i;
    cv = a;
    cf = f;
  }
}

// Largest |value| over the warp, ties to the lowest row; every lane ends
// with the same (a, i, v, f).
__device__ __forceinline__ void warp_argmax(double &a, int &i, double &v, double &f) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double oa = __shfl_xor_sync(kFull, a, o), ov = __shfl_xor_sync(kFull, v, o);
    const double of = __shfl_xor_sync(kFull, f, o);
    const int oi = __shfl_xor_sync(kFull, i, o);
    if (oa > a || (oa == a && oi < i)) {
      a = oa;
      i = oi;
      v = ov;
      f = of;
    }
  }
}

template <class LT, int NC>
__device__ __noinline__ int invert_cta(const DevMech &m, const Smem &s, const double *J, double c, int n,
                                       int lda) {
  LT *A = (LT *)s.A;
  LT *r1b = (LT *)s.colk;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, w = tid >> 5, nw = nt >> 5;
  double *cand = s.red + 64;  // [0,16) |pivot|, [16,32) row, [32,48) value, [48,64) a_row[k]
  for (int i = tid; i < n * lda; i += nt) A[i] = (LT)0;
  for (int i = tid; i < n; i += nt) {
    s.wlu[i] = s.scale[i];
    s.perm[i] = i;
  }
  __syncthreads();
  for (int i = tid; i < n; i += nt) {  // Jacobian row i from the row-wise view
    const double ci = -c / s.wlu[i];
    for (int q = m.jr_ptr[i]; q < m.jr_ptr[i + 1]; ++q) {
      const int j = m.jr_col[q];
      A[i * lda + j] = (LT)(ci * J[m.jr_kk[q]] * s.wlu[j]);
    }
  }
  __syncthreads();
  for (int i = tid; i < n; i += nt) A[i * lda + i] += (LT)1;
  __syncthreads();
  auto publish = [&](double ca, int ci, double cv, double cf) {
    warp_argmax(ca, ci, cv, cf);
    if (lane == 0) {
      cand[w] = ca;
      cand[16 + w] = (double)ci;
      cand[32 + w] = cv;
      cand[48 + w] = cf;
    }
  };
  // the pivot every thread picks from the candidates; -1 if singular
  auto pick = [&](double &pv, double &pf) -> int {
    double best = lane < nw ? cand[lane] : -1.0, v = lane < nw ? cand[32 + lane] : 0.0;
    double f = lane < nw ? cand[48 + lane] : 0.0;
    int p = lane < nw ? (int)cand[16 + lane] : n;
    warp_argmax(best, p, v, f);
    pv = v;
    pf = f;
    return (!(best > 0.0) || !isfinite(best) || p >= n) ? -1 : p;
  };
  {  // candidates for column 0
    double ca = -1.0, cv = 0.0, cf = 0.0;
    int ci = n;
    for (int i = tid; i < n; i += nt) track(ca, ci, cv, cf, (double)A[i * lda], i, 0.0);
    publish(ca, ci, cv, cf);
  }
  __syncthreads();
  int bad = 0;
  for (int k = 0; k < n;) {
    // ---- S1: first pivot of the pair
    double pv1, unused;
    const int p1 = pick(pv1, unused);
    if (p1 < 0) {
      bad = 1;
      break;  // uniform: every thread made the same choice
    }
    const LT pinv1 = (LT)1 / (LT)pv1;
    if (tid == 0) {
      const int t = s.perm[k];
      s.perm[k] = s.perm[p1];
      s.perm[p1] = t;
    }
    for (int j = tid; j < n; j += nt) {
      const LT a = A[k * lda + j], b = A[p1 * lda + j];
      A[p1 * lda + j] = a;
      const LT r = (j == k ? (LT)1 : b) * pinv1;
      A[k * lda + j] = r;
      r1b[j] = r;
    }
    __syncthreads();
    if (k + 1 == n) {  // lone last pivot
      for (int i = w; i < n; i += nw) {
        if (i == k) continue;
        const LT f = A[i * lda + k];
        __syncwarp();
        if (f != (LT)0)
          for (int j = lane; j < n; j += 32) A[i * lda + j] = (j == k ? (LT)0 : A[i * lda + j]) - f * r1b[j];
      }
      __syncthreads();
      break;
    }
    // ---- C: candidates for the second pivot
    const LT r1k1 = r1b[k + 1];
    {
      double ca = -1.0, cv = 0.0, cf = 0.0;
      int ci = n;
      for (int i = k + 1 + tid; i < n; i += nt) {
        const LT f = A[i * lda + k];
        track(ca, ci, cv, cf, (double)(A[i * lda + k + 1] - f * r1k1), i, (double)f);
      }
      publish(ca, ci, cv, cf);
    }
    __syncthreads();
    // ---- S2: second pivot, from the raw row
    double pv2, f2d;
    const int p2 = pick(pv2, f2d);
    if (p2 < 0) {
      bad = 1;
      break;
    }
    const LT pinv2 = (LT)1 / (LT)pv2, f2 = (LT)f2d;
    if (tid == 0) {
      const int t = s.perm[k + 1];
      s.perm[k + 1] = s.perm[p2];
      s.perm[p2] = t;
    }
    for (int j = tid; j < n; j += nt) {
      const LT a = A[(k + 1) * lda + j], b = A[p2 * lda + j];
      A[p2 * lda + j] = a;
      const LT ap = (j == k ? (LT)0 : b) - f2 * r1b[j];
      const LT r2 = (j == k + 1 ? (LT)1 : ap) * pinv2;
      A[(k + 1) * lda + j] = r2;
      A[k * lda + j] = (j == k + 1 ? (LT)0 : r1b[j]) - r1k1 * r2;
    }
    __syncthreads();
    // ---- U: every other row in one pass
    LT r1v[NC], r2v[NC];
#pragma unroll
    for (int t = 0; t < NC; ++t) {
      const int j = lane + 32 * t;
      const bool jv = t < NC - 1 || j < n;
      r1v[t] = (jv && j != k + 1) ? r1b[j] : (LT)0;
      r2v[t] = jv ? A[(k + 1) * lda + j] : (LT)0;
    }
    const LT r1kk = r1b[k], r2k = A[(k + 1) * lda + k], r2k1 = A[(k + 1) * lda + k + 1];
    const int ck = k & 31, ck1 = (k + 1) & 31, t2 = (k + 2) >> 5, c2 = (k + 2) & 31;
    double ca = -1.0, cv = 0.0, cf = 0.0;
    int ci = n;
    for (int i0 = w; i0 < n; i0 += 2 * nw) {
      const int i1 = i0 + nw;
      const bool in1 = i1 < n;
      const bool u0 = i0 != k && i0 != k + 1, u1 = in1 && i1 != k && i1 != k + 1;
      const LT f0 = u0 ? A[i0 * lda + k] : (LT)0, f1 = u1 ? A[i1 * lda + k] : (LT)0;
      const LT g0 = u0 ? A[i0 * lda + k + 1] - f0 * r1k1 : (LT)0;
      const LT g1 = u1 ? A[i1 * lda + k + 1] - f1 * r1k1 : (LT)0;
      LT a0[NC], a1[NC];
#pragma unroll
      for (int t = 0; t < NC; ++t) {
        const int j = lane + 32 * t;
        const bool jv = t < NC - 1 || j < n;
        a0[t] = jv ? A[i0 * lda + j] : (LT)0;
        a1[t] = (jv && in1) ? A[i1 * lda + j] : (LT)0;
      }
      __syncwarp();
      const bool s0 = f0 != (LT)0 || g0 != (LT)0, s1 = f1 != (LT)0 || g1 != (LT)0;
#pragma unroll
      for (int t = 0; t < NC; ++t) {
        const int j = lane + 32 * t;
        const bool jv = t < NC - 1 || j < n;
        a0[t] = a0[t] - f0 * r1v[t] - g0 * r2v[t];
        a1[t] = a1[t] - f1 * r1v[t] - g1 * r2v[t];
        if (jv && s0) A[i0 * lda + j] = a0[t];
        if (jv && s1) A[i1 * lda + j] = a1[t];
      }
      if (lane == ck) {  // Gauss-Jordan values of the eliminated columns
        if (s0) A[i0 * lda + k] = -f0 * r1kk - g0 * r2k;
        if (s1) A[i1 * lda + k] = -f1 * r1kk - g1 * r2k;
      }
      if (lane == ck1) {
        if (s0) A[i0 * lda + k + 1] = -g0 * r2k1;
        if (s1) A[i1 * lda + k + 1] = -g1 * r2k1;
      }
      if (lane == c2 && k + 2 < n) {  // candidates for column k + 2
        LT v0 = a0[0], v1 = a1[0];
#pragma unroll
        for (int t = 1; t < NC; ++t)
          if (t == t2) {
            v0 = a0[t];
            v1 = a1[t];
          }
        if (i0 >= k + 2) track(ca, ci, cv, cf, (double)v0, i0, 0.0);
        if (in1 && i1 >= k + 2) track(ca, ci, cv, cf, (double)v1, i1, 0.0);
      }
    }
    publish(ca, ci, cv, cf);
    __syncthreads();
    k += 2;
  }
  return __syncthreads_or(bad);
}

// invert_cta for the register-chunk count nc = ceil(n / 32) (1..8).
template <class LT>
__device__ __forceinline__ int invert_any(int nc, const DevMech &m, const Smem &s, const double *J,
                                          double c, int n, int lda) {
  switch (nc) {
    case 1: return invert_cta<LT, 1>(m, s, J, c, n, lda);
    case 2: return invert_cta<LT, 2>(m, s, J, c, n, lda);
    case 3: return invert_cta<LT, 3>(m, s, J, c, n, lda);
    case 4: return invert_cta<LT, 4>(m, s, J, c, n, lda);
    case 5: return invert_cta<LT, 5>(m, s, J, c, n, lda);
    case 6: return invert_cta<LT, 6>(m, s, J, c, n, lda);
    case 7: return invert_cta<LT, 7>(m, s, J, c, n, lda);
    default: return invert_cta<LT, 8>(m, s, J, c, n, lda);
  }
}

// x = (I - c_lu J)^{-1} b with the stored inverse: x = W A (perm of W^-1 b).
// Thread per row, four independent partial sums to hide the FMA latency.
template <class LT>
__device__ void apply_inverse(const Smem &s, int n, int lda, const double *b, double *x) {
  const LT *A = (const LT *)s.A;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int pi = s.perm[i];
    s.bs[i] = b[pi] / s.wlu[pi];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const LT *row = A + (size_t)i * lda;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int j = 0;
    for (; j + 3 < n; j += 4) {
      a0 += (double)row[j] * s.bs[j];
      a1 += (double)row[j + 1] * s.bs[j + 1];
      a2 += (double)row[j + 2] * s.bs[j + 2];
      a3 += (double)row[j + 3] * s.bs[j + 3];
    }
    for (; j < n; ++j) a0 += (double)row[j] * s.bs[j];
    x[i] = ((a0 + a1) + (a2 + a3)) * s.wlu[i];
  }
  __syncthreads();
}

// Energy-source coupling on a Newton solve x = A^-1 b (Sherman-Morrison):
// (A - c g d^T)^-1 b = x + w (r1k d.x) with w = A^-1 g, r1k = c / (1 - c d.w).
__device__ void rank1_fix(const Smem &s, int n, double r1k, double *x) {
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a += s.r1d[i] * x[i];
  const double dx = block_sum(a, s.red) * r1k;
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] += s.r1w[i] * dx;
  __syncthreads();
}

__device__ void change_D_cta(double *D, int n, int order, double fac) {
  double R[kMaxOrder + 1][kMaxOrder + 1], U[kMaxOrder + 1][kMaxOrder + 1];
  for (int pass = 0; pass < 2; ++pass) {
    const double f = pass == 0 ? fac : 1.0;
    double (*A)[kMaxOrder + 1] = pass == 0 ? R : U;
    for (int j = 0; j <= order; ++j) {
      A[0][j] = 1.0;
      for (int i = 1; i <= order; ++i) A[i][j] = A[i - 1][j] * (j == 0 ? 0.0 : (i - 1 - f * j) / i);
    }
  }
  double RU[kMaxOrder + 1][kMaxOrder + 1];
  for (int i = 0; i <= order; ++i)
    for (int j = 0; j <= order; ++j) {
      double t = 0.0;
      for (int k = 0; k <= order; ++k) t += R[i][k] * U[k][j];
      RU[i][j] = t;
    }
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    double old[kMaxOrder + 1];
    for (int k = 0; k <= order; ++k) old[k] = D[k * n + c];
    for (int i = 0; i <= order; ++i) {
      double t = 0.0;
      for (int k = 0; k <= order; ++k) t += RU[k][i] * old[k];
      D[i * n + c] = t;
    }
  }
  __syncthreads();
}

struct Consts {
  double gam[kMaxOrder + 2], alp[kMaxOrder + 2], econ[kMaxOrder + 2];
};

__host__ __device__ inline void make_consts(Consts &b) {
  const double kap[kMaxOrder + 1] = {0.0, -0.1850, -1.0 / 9.0, -0.0823, -0.0415, 0.0};
  for (int k = 0; k <= kMaxOrder + 1; ++k) {
    double g = 0.0;
    for (int i = 1; i <= k; ++i) g += 1.0 / i;
    b.gam[k] = g;
    const double kk = (k <= kMaxOrder) ? kap[k] : 0.0;
    b.alp[k] = (1.0 - kk) * g;
    b.econ[k] = kk * g + 1.0 / (k + 1);
  }
}


// Left-preconditioned GMRES for (I - cJ) x = b, the Newton system of the
// FP32 path, in the error-weighted coordinates (scale = atol + rtol |y|):
// the operator is applied in FP64 from the stored sparse Jacobian and the
// FP32 inverse is only the preconditioner, so the Newton corrections keep
// FP64 accuracy whatever the single-precision factor loses.  The method is
// SPGMR's (modified Gram-Schmidt, no restarts, x0 = 0, converged when the
// preconditioned residual's weighted 2-norm is <= delta), restated from Saad
// and Schultz, SIAM J. Sci. Stat. Comput. 7 (1986) 856-869; the reference
// plugin drives it through CVODE with PREC_LEFT / MODIFIED_GS
// (applications/cfd_plugin/solver_cvode.cpp:119-141, 201-212).  Every thread
// keeps the same Hessenberg matrix and rotations (the reductions broadcast
// one total), so no thread-0 phase is needed.  Returns 0 when converged, 1
// when the residual was reduced but not below delta, 2 otherwise.
template <class LT>
// Under an energy source the operator and the preconditioner carry the
// rank-one temperature coupling (r1k as in rank1_fix).
__device__ __noinline__ int gmres_cta(const DevMech &m, const Smem &s, const double *J, double c, int n, int lda,
                         double delta, const double *b, double *x, int &iters, double r1k) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool r1 = s.src.esrc != 0.0;
  double *V = s.V, *u = s.V + (kMaxl + 1) * n, *z = u + n;
  apply_inverse<LT>(s, n, lda, b, z);
  if (r1) rank1_fix(s, n, r1k, z);
  double a = 0.0;
  for (int i = tid; i < n; i += nt) {
    const double t = z[i] / s.scale[i];
    V[i] = t;
    a += t * t;
  }
  const double beta = sqrt(block_sum(a, s.red));
  if (!isfinite(beta)) return 2;
  if (beta <= delta) {  // the zero initial guess already satisfies the test
    for (int i = tid; i < n; i += nt) x[i] = 0.0;
    __syncthreads();
    return 0;
  }
  double H[kMaxl + 1][kMaxl], cs[kMaxl], sn[kMaxl], g[kMaxl + 1], yk[kMaxl];
  g[0] = beta;
  for (int i = tid; i < n; i += nt) V[i] /= beta;
  int nl = 0;
  double rho = beta;
  bool conv = false;
  for (int l = 0; l < kMaxl; ++l) {
    const double *vl = V + l * n;
    double *w = V + (l + 1) * n;
    double du = 0.0;
    for (int i = tid; i < n; i += nt) {
      u[i] = vl[i] * s.scale[i];
      if (r1) du += s.r1d[i] * u[i];
    }
    if (r1) du = block_sum(du, s.red);
    __syncthreads();
    for (int i = tid; i < n; i += nt) {  // (I - cJ) u, row i
      double jx = 0.0;
      for (int q = m.jr_ptr[i]; q < m.jr_ptr[i + 1]; ++q) jx += J[m.jr_kk[q]] * u[m.jr_col[q]];
      if (r1) jx += s.r1g[i] * du;
      s.colk[i] = u[i] - c * jx;
    }
    __syncthreads();
    apply_inverse<LT>(s, n, lda, s.colk, z);
    if (r1) rank1_fix(s, n, r1k, z);
    for (int i = tid; i < n; i += nt) w[i] = z[i] / s.scale[i];
    for (int k = 0; k <= l; ++k) {  // modified Gram-Schmidt
      const double *vk = V + k * n;
      double d = 0.0;
      for (int i = tid; i < n; i += nt) d += w[i] * vk[i];
      const double h = block_sum(d, s.red);
      H[k][l] = h;
      for (int i = tid; i < n; i += nt) w[i] -= h * vk[i];
    }
    double d2 = 0.0;
    for (int i = tid; i < n; i += nt) d2 += w[i] * w[i];
    const double hn = sqrt(block_sum(d2, s.red));
    for (int k = 0; k < l; ++k) {  // earlier rotations on the new column
      const double h0 = H[k][l], h1 = H[k + 1][l];
      H[k][l] = cs[k] * h0 + sn[k] * h1;
      H[k + 1][l] = -sn[k] * h0 + cs[k] * h1;
    }
    const double a0 = H[l][l];
    double cc, ss;
    if (hn == 0.0) {
      cc = 1.0;
      ss = 0.0;
    } else if (fabs(hn) > fabs(a0)) {
      const double t = a0 / hn;
      ss = 1.0 / sqrt(1.0 + t * t);
      cc = ss * t;
    } else {
      const double t = hn / a0;
      cc = 1.0 / sqrt(1.0 + t * t);
      ss = cc * t;
    }
    H[l][l] = cc * a0 + ss * hn;
    cs[l] = cc;
    sn[l] = ss;
    g[l + 1] = -ss * g[l];
    g[l] = cc * g[l];
    rho = fabs(g[l + 1]);
    nl = l + 1;
    ++iters;
    if (hn > 0.0)
      for (int i = tid; i < n; i += nt) w[i] /= hn;
    if (!isfinite(rho)) return 2;
    if (rho <= delta) {
      conv = true;
      break;
    }
    if (hn == 0.0) break;
  }
  for (int k = nl - 1; k >= 0; --k) {
    double t = g[k];
    for (int j = k + 1; j < nl; ++j) t -= H[k][j] * yk[j];
    yk[k] = t / H[k][k];
  }
  for (int i = tid; i < n; i += nt) {
    double acc = 0.0;
    for (int k = 0; k < nl; ++k) acc += yk[k] * V[k * n + i];
    x[i] = acc * s.scale[i];
  }
  __syncthreads();
  if (conv) return 0;
  return rho < beta ? 1 : 2;
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16(x)); }

// Batch-one forward pass of the predictor network (mlp.cu's layers, the
// same BF16 rounding of inputs and hidden activations, FP32 accumulation):
// thread per output, bf16 weights read from global memory (L2-resident).
// Returns the buffer holding the standardised outputs.
__device__ float *mlp_forward_cta(const MlpDev &net, float *a, float *b) {
  for (int l = 0; l < net.layers; ++l) {
    const int K = net.dims[l], N = net.dims[l + 1];
    const __nv_bfloat16 *W = net.w[l];
    const bool hidden = l + 1 < net.layers;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
      float acc = 0.0f;
#pragma unroll 8
      for (int k = 0; k < K; ++k) acc = fmaf(a[k], __bfloat162float(W[(size_t)k * N + j]), acc);
      const float z = acc + net.b[l][j];
      b[j] = hidden ? bf16_round(z / (1.0f + expf(-z))) : z;
    }
    __syncthreads();
    float *t = a;
    a = b;
    b = t;
  }
  return a;
}

// Learned predictor (N3 form): the network's estimate of y(t + h) from the
// last accepted state (row 0 of D) and h replaces the polynomial predictor
// as the Newton starting iterate; ypred, psi and the error estimate keep the
// polynomial predictor, so the error test judges the step exactly as
// without the network.  Inputs: log10 of the clamped mass fractions,
// (T - 1500 K) / 1000 K, log10(P / 1 bar), log10(h); targets: change of
// log10 mass fraction and (T' - T) / 100 K, standardised.
__device__ __noinline__ void predict_cta(const DevMech &m, const IntegOpts &o, const Smem &s, double v, double h) {
  const int S = m.nsp, n = S + 1, tid = threadIdx.x, nt = blockDim.x;
  const PredDev &p = o.pred;
  const double *y0 = s.D;
  double pw = 0.0;
  for (int k = tid; k < S; k += nt) pw += y0[k] * m.inv_mw[k];
  const double iw = block_sum(pw, s.red);
  const double T = y0[S] * o.Tref;
  const double P = kRuD * T * iw / v;
  float *xa = s.mlp, *xb = s.mlp + kPredBuf;
  for (int i = tid; i < p.net.dims[0]; i += nt) {
    double f = 0.0;
    if (i < S) f = log10(fmax(y0[i], 1e-30));
    else if (i == S) f = (T - 1500.0) / 1000.0;
    else if (i == S + 1) f = log10(fmax(P, 1e-300) / 1e5);
    else if (i == S + 2) f = log10(h);
    xa[i] = i < p.net.n_in ? bf16_round((float)((f - p.x_mu[i]) / p.x_sd[i])) : 0.0f;
  }
  __syncthreads();
  const float *r = mlp_forward_cta(p.net, xa, xb);
  for (int i = tid; i < n; i += nt) {
    const double t = (double)r[i] * p.t_sd[i] + p.t_mu[i];
    const double yi = i < S ? exp10(log10(fmax(y0[i], 1e-30)) + t) : (T + 100.0 * t) / o.Tref;
    s.y[i] = yi;
    s.d[i] = yi - s.ypred[i];
  }
  __syncthreads();
}

template <class LT>
__device__ __forceinline__ int attempt_cta(const DevMech &m, const IntegOpts &o, const Consts &bc, const Smem &s,
                           double *J, double v, double t_end, double rtol, double atol,
                           ReactorStats &st, int lda, double &t_done, double t_off, double T_target,
                           double &t_ign, CbCtx &cb) {
  const int n = m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
  const int nc = (n + 31) / 32;
  auto vrms = [&](const double *x, const double *sc) {
    double a = 0.0;
    for (int i = tid; i < n; i += nt) {
      const double t = x[i] / sc[i];
      a += t * t;
    }
    return sqrt(block_sum(a, s.red) / n);
  };
  double t = 0.0;
  int rc = 0;
  t_done = 0.0;
  double T_prev = s.y[m.nsp] * o.Tref;  // ignition: temperature at the last accepted step
  double r1k = 0.0;  // energy-source coupling of the current factor
  // absolute tolerance of component i: with abstol_dens the species' are
  // abs_tol / molar density (reactor_nvector_serial.cpp:107-119, the
  // correction formed as 1 / (rho / W_k * 1e-3)), at the initial density
  auto atol_of = [&](int i) {
    return (o.abstol_dens && i < m.nsp) ? atol * (1.0 / ((1.0 / v) * m.inv_mw[i] * 1.0e-3)) : atol;
  };
  auto rank1_setup = [&](double cc) {
    if (s.src.esrc == 0.0) return;
    apply_inverse<LT>(s, n, lda, s.r1g, s.r1w);
    double a = 0.0;
    for (int i = tid; i < n; i += nt) a += s.r1d[i] * s.r1w[i];
    const double dw = block_sum(a, s.red);
    r1k = cc / (1.0 - cc * dw);
  };
  st.nrhs++;
  if (rhs_cta(m, o, s, v, t_off, s.y, s.f0, false, nullptr)) return -1;
  for (int i = tid; i < n; i += nt) s.scale[i] = atol_of(i) + fabs(s.y[i]) * rtol;
  __syncthreads();
  const double d0 = vrms(s.y, s.scale), d1 = vrms(s.f0, s.scale);
  double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
  if (h0 > t_end) h0 = t_end;
  for (int i = tid; i < n; i += nt) s.tmp[i] = s.y[i] + h0 * s.f0[i];
  __syncthreads();
  double d2 = 0.0;
  st.nrhs++;
  if (rhs_cta(m, o, s, v, t_off + h0, s.tmp, s.f, false, nullptr) == 0) {
    for (int i = tid; i < n; i += nt) s.d[i] = s.f[i] - s.f0[i];
    __syncthreads();
    d2 = vrms(s.d, s.scale) / h0;
  }
  double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : sqrt(0.01 / fmax(d1, d2));
  double h = fmin(100.0 * h0, h1);
  h = fmin(h, o.max_dt);
  h = fmin(h, t_end);
  int q = 1, neq = 0, jac_current = 1, nsteps = 0, pred_fail = 0;
  double c_lu = h / bc.alp[q], crate = 1.0;
  for (int i = tid; i < (kMaxOrder + 3) * n; i += nt) s.D[i] = 0.0;
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    s.D[i] = s.y[i];
    s.D[n + i] = s.f0[i] * h;
  }
  __syncthreads();
  st.njac++;
  if (jac_cta(m, o, s, v, t_off, s.y, s.f0, J)) { rc = -2; goto failed; }
  st.nlu++;
  if (invert_any<LT>(nc, m, s, J, c_lu, n, lda)) { rc = -3; goto failed; }
  rank1_setup(c_lu);
  while (t < t_end) {
    if (nsteps >= o.max_steps) { rc = -4; goto failed; }
    bool accepted = false;
    // the learned predictor starts each step; any rejection falls back to
    // the polynomial predictor for the rest of the step, and after two
    // consecutive failed learned starts the reactor stops consulting the
    // network for the rest of the attempt
    bool use_pred = o.pred.enabled != 0 && pred_fail < 2;
    double safety = 0.9, err_norm = 0.0;
    int nef = 0, ncf = 0;  // this step's error-test and convergence failures
    while (!accepted) {
      if (h > o.max_dt) {
        change_D_cta(s.D, n, q, o.max_dt / h);
        h = o.max_dt;
      }
      if (t + h > t_end) {
        change_D_cta(s.D, n, q, (t_end - t) / h);
        h = t_end - t;
      }
      if (!(t + h > t)) { rc = -5; goto failed; }
      const double t_new = t + h;
      for (int i = tid; i < n; i += nt) {
        double a = 0.0, ps = 0.0;
        for (int k = 0; k <= q; ++k) a += s.D[k * n + i];
        for (int k = 1; k <= q; ++k) ps += bc.gam[k] * s.D[k * n + i];
        s.ypred[i] = a;
        s.psi[i] = ps / bc.alp[q];
        s.scale[i] = atol_of(i) + rtol * fabs(a);
        s.y[i] = a;
        s.d[i] = 0.0;
      }
      __syncthreads();
      if (use_pred) predict_cta(m, o, s, v, h);
      const double c = h / bc.alp[q];
      // new factor when c moved by more than 30 % (CVODE's dgmax); a looser
      // rule for the FP32 preconditioner costs more Krylov failures than the
      // factorizations it saves
      if (fabs(c / c_lu - 1.0) > 0.3) {
        st.nlu++;
        c_lu = c;
        crate = 1.0;
        if (invert_any<LT>(nc, m, s, J, c, n, lda)) { rc = -3; goto failed; }
        rank1_setup(c);
      }
      const double gscale = (c == c_lu) ? 1.0 : 2.0 / (1.0 + c / c_lu);
      bool conv = false;
      int it;
      double dnorm_old = -1.0;
      for (it = 0; it < kNewtonMaxIter; ++it) {
        st.nrhs++;
        if (rhs_cta(m, o, s, v, t_off + t_new, s.y, s.f, false, nullptr)) break;
        int bad = 0;
        for (int i = tid; i < n; i += nt) bad |= !isfinite(s.f[i]);
        if (__syncthreads_or(bad)) break;
        if (it == 0)
          for (int i = tid; i < n; i += nt) s.f0[i] = s.f[i];
        st.nnewt++;
        for (int i = tid; i < n; i += nt) s.tmp[i] = c * s.f[i] - s.psi[i] - s.d[i];
        __syncthreads();
        double gs = gscale;
        if constexpr (sizeof(LT) == sizeof(float)) {
          // Krylov tolerance eps_lin * nlscoef / error constant (WRMS), as a
          // weighted 2-norm.  Unlike CVODE, which accepts a reduced but
          // unconverged residual on the first Newton iteration, every solve
          // must converge: with a single-precision preconditioner a stalled
          // Krylov solve can pass the Newton test with a poor correction,
          // and a failure here costs only a Jacobian update or a step cut.
          const double delta = o.eps_lin * o.nlscoef / bc.econ[q] * sqrt((double)n);
          if (gmres_cta<LT>(m, s, J, c, n, lda, delta, s.tmp, s.yp, st.nkry, r1k) != 0) break;
          gs = 1.0;  // the Krylov solve uses the current c exactly
        } else {
          apply_inverse<LT>(s, n, lda, s.tmp, s.yp);
          if (s.src.esrc != 0.0) rank1_fix(s, n, r1k, s.yp);
        }
        double a = 0.0;
        for (int i = tid; i < n; i += nt) {
          const double dy = s.yp[i] * gs;
          s.y[i] += dy;
          s.d[i] += dy;
          const double tt = dy / s.scale[i];
          a += tt * tt;
        }
        const double dn = sqrt(block_sum(a, s.red) / n);
        if (dnorm_old > 0.0) crate = fmax(0.3 * crate, dn / dnorm_old);
        // from a learned starting iterate, convergence is only declared on
        // the last correction itself (two iterations at least): neither the
        // carried rate estimate (the polynomial predictor's start) nor one
        // measured from a large first correction bounds the remaining error
        const double dconv = use_pred ? dn : dn * fmin(1.0, crate);
        if (!(use_pred && it == 0) && bc.econ[q] * dconv <= o.nlscoef) {
          conv = true;
          ++it;
          break;
        }
        if (dnorm_old > 0.0 && dn > 2.0 * dnorm_old) break;
        dnorm_old = dn;
      }
      if (!conv) {
        if (use_pred) {  // the learned start failed: same step from the polynomial predictor
          use_pred = false;
          ++pred_fail;
          continue;
        }
        if (!jac_current) {
          st.nrhs++;
          if (rhs_cta(m, o, s, v, t_off + t_new, s.ypred, s.f0, false, nullptr)) { rc = -6; goto failed; }
          st.njac++;
          if (jac_cta(m, o, s, v, t_off + t_new, s.ypred, s.f0, J)) { rc = -2; goto failed; }
          jac_current = 1;
          st.nlu++;
          c_lu = c;
          crate = 1.0;
          if (invert_any<LT>(nc, m, s, J, c, n, lda)) { rc = -3; goto failed; }
          rank1_setup(c);
          continue;
        }
        if (++ncf >= kMaxConvFails) { rc = -8; goto failed; }
        change_D_cta(s.D, n, q, 0.5);
        h *= 0.5;
        st.nrej++;
        continue;
      }
      safety = 0.9 * (2 * kNewtonMaxIter + 1) / (2.0 * kNewtonMaxIter + it);
      double a = 0.0;
      for (int i = tid; i < n; i += nt) {
        const double e = bc.econ[q] * s.d[i] / s.scale[i];
        a += e * e;
      }
      err_norm = sqrt(block_sum(a, s.red) / n);
      if (!isfinite(err_norm)) { rc = -7; goto failed; }
      if (err_norm > 1.0) {
        if (++nef >= kMaxErrTestFails) { rc = -9; goto failed; }
        use_pred = false;
        st.nrej++;
        if (nef > kErrFailsBeforeCut) {  // order and step cut (integrator.h)
          if (q > 1) {
            --q;
            change_D_cta(s.D, n, q, kEtaMinErrFail);
          } else {
            st.nrhs++;
            if (rhs_cta(m, o, s, v, t_off + t, s.D, s.tmp, false, nullptr)) { rc = -6; goto failed; }
            for (int i = tid; i < n; i += nt) s.D[n + i] = s.tmp[i] * (h * kEtaMinErrFail);
            __syncthreads();
          }
          h *= kEtaMinErrFail;
          neq = 0;
          continue;
        }
        const double fac = fmax(kMinFactor, safety * pow(err_norm, -1.0 / (q + 1)));
        change_D_cta(s.D, n, q, fac);
        h *= fac;
        continue;
      }
      if (use_pred) pred_fail = 0;  // the learned start converged and passed
      accepted = true;
      t = t_new;
    }
    ++nsteps;
    st.nsteps++;
    ++neq;
    jac_current = 0;
    const bool keep_prev = T_target > 0.0 && o.stop_ign && t_ign < 0.0;
    for (int i = tid; i < n; i += nt) {
      if (keep_prev) s.tmp[i] = s.D[i];  // the previous accepted state
      const double di = s.d[i];
      s.D[(q + 2) * n + i] = di - s.D[(q + 1) * n + i];
      s.D[(q + 1) * n + i] = di;
      for (int k = q; k >= 0; --k) s.D[k * n + i] += s.D[(k + 1) * n + i];
    }
    __syncthreads();
    if (T_target > 0.0) {  // first crossing of T0 + dT_ign, linear between accepted steps
      const double Tn = s.D[n - 1] * o.Tref;
      if (t_ign < 0.0 && Tn >= T_target) {
        const double frac = (Tn > T_prev) ? (T_target - T_prev) / (Tn - T_prev) : 1.0;
        t_ign = t_off + (t - h) + frac * h;
        // the callback's record of CVode's root return (solver_cvode.cpp:249-262)
        const bool cb_end = cb.rec && cb_record(cb, s.D, o.stop_ign ? s.tmp : nullptr, n, q, h,
                                                frac - 1.0, frac, t_ign, s.y, tid, nt);
        if (o.stop_ign || cb_end) {  // stop_after_ignition: the call ends at the crossing
          if (!cb_end)
            for (int i = tid; i < n; i += nt) s.y[i] = s.tmp[i] + frac * (s.D[i] - s.tmp[i]);
          __syncthreads();
          t_done = (t - h) + frac * h;
          return 0;
        }
      }
      T_prev = Tn;
    }
    if (cb.rec && cb_record(cb, s.D, nullptr, n, q, h, 0.0, 0.0, t_off + t, s.y, tid, nt)) {
      __syncthreads();  // the callback asked to stop here
      t_done = t;
      return 0;
    }
    if (neq < q + 1) continue;
    double em = INFINITY, ep = INFINITY;
    {
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
      const double sm = block_sum(am, s.red), sp = block_sum(ap, s.red);
      if (q > 1) em = sqrt(sm / n);
      if (q < kMaxOrder) ep = sqrt(sp / n);
    }
    const double fm = (q > 1) ? pow(em, -1.0 / q) : 0.0;
    const double f0 = pow(err_norm, -1.0 / (q + 1));
    const double fp = (q < kMaxOrder) ? pow(ep, -1.0 / (q + 2)) : 0.0;
    int dq = 0;
    double best = f0;
    if (fm > best) { best = fm; dq = -1; }
    if (fp > best) { best = fp; dq = 1; }
    q += dq;
    double fac = fmin(kMaxFactor, safety * best);
    if (fac < kEtaKeep) fac = 1.0;
    change_D_cta(s.D, n, q, fac);
    h *= fac;
    neq = 0;
  }
  for (int i = tid; i < n; i += nt) s.y[i] = s.D[i];
  __syncthreads();
  t_done = t;
  return 0;
failed:  // D[0] holds the last accepted state (step-size changes keep it)
  for (int i = tid; i < n; i += nt) s.y[i] = s.D[i];
  __syncthreads();
  t_done = t;
  return rc;
}

// spill bits: 1 = rates of progress in a global slice, 2 = BDF differences
// in a global slice (both L2-resident: one slice per resident CTA).
template <class LT>
__global__ void __launch_bounds__(512, 1) integrate_dense_kernel(DevMech m, IntegOpts o, IntegArgs a,
                                                                 int lda, int spill) {
  extern __shared__ double smem_dyn[];
  const int S = m.nsp, n = S + 1, N = m.nstep, tid = threadIdx.x, nt = blockDim.x;
  Smem s;
  double *p = smem_dyn;
  double *g = a.rop_scratch + (size_t)blockIdx.x * ((size_t)N + (kMaxOrder + 6) * (size_t)n);
  s.red = p; p += 128;
  s.C = p; p += S;
  s.G = p; p += S;
  s.U = p; p += S;
  if (spill & 1) { s.ROP = g; } else { s.ROP = p; p += N; }
  if (spill & 2) { s.D = g + N; } else { s.D = p; p += (kMaxOrder + 3) * n; }
  s.Jsm = nullptr;
  if (spill & 4) { s.Jsm = p; p += m.nnz; }
  s.ysrc = nullptr;
  s.r1g = g + N + (kMaxOrder + 3) * n;
  s.r1d = s.r1g + n;
  s.r1w = s.r1d + n;
  s.y = p; p += n;
  s.f = p; p += n;
  s.f0 = p; p += n;
  s.ypred = p; p += n;
  s.psi = p; p += n;
  s.d = p; p += n;
  s.scale = p; p += n;
  s.tmp = p; p += n;
  s.yp = p; p += n;
  s.colk = p; p += n;
  s.wlu = p; p += n;
  s.bs = p; p += n;
  s.V = nullptr;
  if (sizeof(LT) == sizeof(float)) {
    s.V = p;
    p += (kMaxl + 3) * n;
  }
  s.mlp = (float *)p;
  p += kPredBuf;  // 2 * kPredBuf floats
  s.perm = (int *)p; p += (n + 1) / 2 + 1;
  s.A = p;
  Consts bc;
  make_consts(bc);
  __shared__ int next;
  for (;;) {
    if (tid == 0) next = atomicAdd(a.queue_head, 1);
    __syncthreads();
    const int idx = next;
    __syncthreads();
    if (idx >= a.n_reactors) break;
    const int r = a.order ? a.order[idx] : idx;
    double *J = (spill & 4) ? s.Jsm : a.state + (size_t)r * a.state_stride;
    const double T0 = a.T[r], P0 = a.P[r];
    const double *Y0 = a.Y + (size_t)r * S;
    double pa = 0.0;
    for (int k = tid; k < S; k += nt) pa += Y0[k] * m.inv_mw[k];
    const double mwmix = 1.0 / block_sum(pa, s.red);
    const double v = 1.0 / (P0 * mwmix / (kRuD * T0));
    s.src.dpdt = a.dpdt ? a.dpdt[r] : 0.0;
    s.src.esrc = a.esrc ? a.esrc[r] : 0.0;
    s.src.P0 = P0;
    s.src.ysrc = a.ysrc != nullptr;
    s.src.fixT = !o.always_T && a.tdel_in && !(a.tdel_in[r] > 0.0);
    s.src.T0 = T0;
    s.src.E0 = 0.0;
    if (s.src.esrc != 0.0 || s.src.fixT) {  // initial_energy_ (InitializeState)
      double cx;
      mix_energy(m, o.cp != 0, false, T0, Y0, false, 0.0, tid, nt,
                 [&](double x) { return block_sum(x, s.red); }, s.src.E0, cx);
    }
    for (int k = tid; k < S; k += nt) s.y[k] = Y0[k];
    if (tid == 0) s.y[S] = T0 / o.Tref;
    __syncthreads();
    ReactorStats rs = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    CbCtx cb{a.cb_rec ? a.cb_rec + (size_t)idx * a.cb_cap * (3 + 2 * (size_t)n) : nullptr, a.cb_cap,
             (a.cb_rec && a.cb_stop) ? a.cb_stop[r] : 0, 0, 0, 0.0};
    double rtol = o.rtol, atol = o.atol;
    int rc = 0;
    // retries (solver_cvode.cpp:227-246): restart the method from the last
    // accepted state for the remaining time with adjusted tolerances;
    // max_steps counts per attempt
    double t_left = a.dt, t_ign = -1.0;
    const double T_target = o.dT_ign > 0.0 ? T0 + o.dT_ign : -1.0;
    s.ysrc = a.ysrc ? a.ysrc + (size_t)r * S : nullptr;
    for (int attempt = 0;; ++attempt) {
      double t_done = 0.0;
      rc = attempt_cta<LT>(m, o, bc, s, J, v, t_left, rtol, atol, rs, lda, t_done, a.dt - t_left,
                               T_target, t_ign, cb);
      if (rc == 0 || attempt + 1 >= o.max_retries) break;
      cb.ncalls++;  // the failed CVode call counts as a step
      t_left -= t_done;
      rs.retries++;
      atol *= o.retry_atol_factor;
      rtol *= o.retry_rtol_factor;
    }
    rs.status = rc;
    if (rc == 0) {
      double pb = 0.0;
      for (int k = tid; k < S; k += nt) {
        const double ys = s.y[k];
        a.Y[(size_t)r * S + k] = ys;
        pb += ys * m.inv_mw[k];
      }
      const double mw2 = 1.0 / block_sum(pb, s.red);
      const double Tn = end_temperature(m, o.cp != 0, s.src, a.dt, s.y, s.y[S] * o.Tref, tid, nt,
                                        [&](double x) { return block_sum(x, s.red); });
      if (tid == 0) {
        a.T[r] = Tn;
        a.P[r] = end_pressure(o.cp != 0, s.src, a.dt, Tn, mw2, v);
      }
    }
    if (tid == 0) {
      a.v[r] = v;
      if (a.stats) a.stats[r] = rs;
      if (a.cb_cnt) a.cb_cnt[r] = cb.cnt;
      if (a.t_ign) a.t_ign[r] = t_ign;
    }
    __syncthreads();
  }
}


template <class LT>
cudaError_t launch_dense(const DevMech &m, const IntegOpts &o, const IntegArgs &a, int threads,
                         int ctas, int spill, size_t smem, int lda, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(integrate_dense_kernel<LT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  integrate_dense_kernel<LT><<<ctas, threads, smem, stream>>>(m, o, a, lda, spill);
  return cudaGetLastError();
}

}  // namespace

// One translation unit per factor type (integrator_dense_f64.cu,
// integrator_dense_f32.cu) so the two compile in parallel.
cudaError_t launch_integrate_dense_f64(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                       int threads, int ctas, int spill, size_t smem, int lda,
                                       cudaStream_t stream);
cudaError_t launch_integrate_dense_f32(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                       int threads, int ctas, int spill, size_t smem, int lda,
                                       cudaStream_t stream);

}  // namespace zrk
