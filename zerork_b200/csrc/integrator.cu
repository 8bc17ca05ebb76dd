// integrator.cu -- warp-per-reactor BDF integration of constant-volume and
// constant-pressure reactors (see integrator.h).
//
// Per warp: the reactor's right-hand side (reactor_constant_volume_cpu.cpp:
// 64-128) with lanes over species and reactions; its Jacobian
// (reactor_nvector_serial.cpp:610-771) with lanes over the nonzeros of each
// column; the Newton matrix P = I - cJ assembled into the fill pattern and
// factored left-looking with lanes over the entries of each update column;
// column-oriented triangular solves; WRMS norms by shuffle reductions.  All
// lanes hold identical copies of the step-control scalars (reduced values are
// broadcast from lane 0), so control flow is warp-uniform.
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

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0);
}

struct Warp {
  double *C, *G, *U, *ROP;  // species rows and rates of progress
  void *X;                  // LU work / solve vector (n elements of the LU type)
  const double *ysrc;       // this reactor's mass-fraction sources (global) or null
  ReactorSrc src;           // this reactor's pressure-rate / energy sources and initial state
};

// What one right-hand-side evaluation used: mixture heat capacity (c_v, or
// c_p for constant pressure), temperature and inverse density.
struct RhsOut {
  double cx, T, v;
};

struct BdfConst {
  double gam[kMaxOrder + 2], alp[kMaxOrder + 2], econ[kMaxOrder + 2];
};

__device__ void bdf_consts(BdfConst &b) {
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

// ydot at y (global or shared vector of nsp+1 entries) and time t from the
// start of the call; v0 is the reactor's initial inverse density.  Returns 1
// if T <= 0.  Constant pressure (o.cp): reactor_constant_pressure_cpu.cpp:
// 71-135, U then holds h/RT.  T_force > 0 replaces the energy-source
// temperature (reactor_src.cuh).
__device__ __forceinline__ int rhs_warp(const DevMech &m, const IntegOpts &o, const Warp &w,
                                        double v0, double t, const double *y, double *ydot,
                                        int lane, bool clamp, RhsOut *out,
                                        double T_force = 0.0) {
  const int S = m.nsp;
  const double yS = y[S];
  double T = w.src.fixT ? w.src.T0 : yS * o.Tref;
  if (!(T > 0.0)) return 1;
  if (T > 1.0e4) T = 1.0e4;
  double v = v0;
  if (o.cp || w.src.dpdt != 0.0 || w.src.esrc != 0.0)
    source_T_v(m, o.cp != 0, w.src, t, y, clamp, o.mmf, v0, T_force, lane, 32,
               [](double x) { return wsum(x); }, T, v);
  const double logT = log(T), invT = 1.0 / T, lprt = log(kPatmD / (kRuD * T));
  const double dens = 1.0 / v;
  const double ush = o.cp ? 0.0 : 1.0;  // h/RT - 1 = u/RT; c_p/R - 1 = c_v/R
  double pc = 0.0, pcv = 0.0;
  for (int s = lane; s < S; s += 32) {
    double ys = y[s];
    if (clamp) ys = clamp_mass_fraction(ys, o.mmf);
    const double c = dens * m.inv_mw[s] * ys;
    w.C[s] = c;
    double cp, h, g;
    nasa_cp_h_g(m.thermo + 16 * s, T, logT, &cp, &h, &g);
    w.G[s] = g;
    w.U[s] = h - ush;
    pc += c;
    pcv += ((cp - ush) * m.ru_inv_mw[s]) * ys;
  }
  const double Csum = wsum(pc), cv = wsum(pcv);
  __syncwarp();
  for (int r = lane; r < m.nrxn; r += 32)
    reaction_item<1, 1>(m, load_rxn(m.rxn + r), 0, w.C, w.G, w.ROP, &T, &logT, &invT, &lprt, &Csum, o.lim);
  __syncwarp();
  double pe = 0.0;
  for (int s = lane; s < S; s += 32) {
    double des = 0.0, cre = 0.0;
    for (int k = m.sd_ptr[s]; k < m.sd_ptr[s + 1]; ++k) des += w.ROP[m.sd_step[k]];
    for (int k = m.sc_ptr[s]; k < m.sc_ptr[s + 1]; ++k) cre += w.ROP[m.sc_step[k]];
    const double net = cre - des;
    if (w.ysrc) {  // reactor_constant_volume_cpu.cpp:108-113
      const double ys = w.ysrc[s];
      ydot[s] = net * m.mw[s] * v + ys;
      pe += w.U[s] * (net * v + ys * m.inv_mw[s]);
    } else {
      ydot[s] = net * m.mw[s] * v;
      pe += w.U[s] * net * v;
    }
  }
  const double es = wsum(pe);
  if (lane == 0)
    ydot[S] = w.src.fixT ? 0.0 : -es * kRuD * yS / cv + (w.src.esrc + w.src.dpdt * v) / (cv * o.Tref);
  if (out) *out = RhsOut{cv, T, v};
  __syncwarp();
  return 0;
}

// Jacobian values J[nnz] at y with fy = ydot(t, y); tmp: nsp+1 global
// doubles, yp: nsp+1 shared/global doubles of scratch.  Concentration
// derivatives use the initial inverse density at constant volume and the
// current one at constant pressure.  Under an energy source, the rank-one
// temperature coupling g = df/dT*, d = dT*/dY goes to r1g / r1d (see
// integrator_dense.cuh's jac_cta).
__device__ int jac_warp(const DevMech &m, const IntegOpts &o, const Warp &w, double v0, double t,
                        const double *y, const double *fy, double *J, double *tmp, double *yp,
                        double *r1g, double *r1d, int lane) {
  const int S = m.nsp;
  int need = 0;
  for (int s = lane; s < S; s += 32) need |= (fabs(y[s]) < o.mmf);
  need = __any_sync(kFull, need);
  RhsOut ro;
  if (rhs_warp(m, o, w, v0, t, y, tmp, lane, need != 0, &ro)) return 1;
  const double TdC = tmp[S];
  const double yS = y[S];
  const double RuTemp = kRuD * yS;
  const double multFact = -1.0 / ro.cx;
  const double T = ro.T, v = o.cp ? ro.v : v0;
  const double ush = o.cp ? 0.0 : 1.0;
  for (int j = 0; j < S; ++j) {
    const double t2 = m.mw[j] / clamp_mass_fraction(y[j], o.mmf) * v;
    const int k0 = m.col_ptr[j], k1 = m.col_ptr[j + 1] - 1;
    const double wcol = m.inv_mw[j];
    double trow = 0.0;
    for (int kk = k0 + lane; kk < k1; kk += 32) {
      const int row = m.row_idx[kk];
      double des = 0.0, cre = 0.0;
      for (int q = m.nzd_ptr[kk]; q < m.nzd_ptr[kk + 1]; ++q) des += w.ROP[m.nzd_step[q]];
      for (int q = m.nzc_ptr[kk]; q < m.nzc_ptr[kk + 1]; ++q) cre += w.ROP[m.nzc_step[q]];
      const double val = (0.0 - des * t2) + cre * t2;
      trow += val * w.U[row];
      J[kk] = val * (m.mw[row] * wcol);
    }
    trow = wsum(trow);
    if (lane == 0) {
      const double cvj = (nasa_cp(m.thermo + 16 * j, T) - ush) * m.ru_inv_mw[j];
      double tr = trow * RuTemp;
      tr += TdC * cvj * m.mw[j];
      tr *= wcol * multFact;
      J[k1] = w.src.fixT ? 0.0 : tr;  // no temperature row when T is not solved
    }
  }
  __syncwarp();
  // forward-difference temperature column
  const double ySp = yS + yS * o.sqrt_ur;
  const double mult = 1.0 / (ySp - yS);
  for (int s = lane; s < S; s += 32) yp[s] = y[s];
  if (lane == 0) yp[S] = ySp;
  __syncwarp();
  if (rhs_warp(m, o, w, v0, t, yp, tmp, lane, false, nullptr)) return 1;
  for (int kk = m.col_ptr[S] + lane; kk < m.col_ptr[S + 1]; kk += 32) {
    const int row = m.row_idx[kk];
    J[kk] = (tmp[row] - fy[row]) * mult;
  }
  __syncwarp();
  if (w.src.esrc != 0.0) {
    RhsOut r1;
    if (rhs_warp(m, o, w, v0, t, y, yp, lane, false, &r1)) return 1;
    for (int j = lane; j < S; j += 32) {
      double cpR, hRT;
      nasa_cp_h(m.thermo + 16 * j, r1.T, &cpR, &hRT);
      r1d[j] = -((hRT - ush) * (m.ru_inv_mw[j] * r1.T)) / r1.cx;
    }
    if (lane == 0) r1d[S] = 0.0;
    const double Tp = r1.T + r1.T * o.sqrt_ur;
    if (rhs_warp(m, o, w, v0, t, y, tmp, lane, false, nullptr, Tp)) return 1;
    for (int i = lane; i <= S; i += 32) r1g[i] = (tmp[i] - yp[i]) / (Tp - r1.T);
    __syncwarp();
  }
  return 0;
}

// Pw = W^-1 (I - cJ) W into the LU storage, W = diag(scale) the error
// weights of the current step (entry (i, j) is P_ij scale_j / scale_i, the
// Jacobian of relative changes: far better balanced than P for species
// spanning 20 decades of mass fraction), then left-looking factorization in
// place.  wsc receives the scale the factor was formed with.
template <class LT>
__device__ int lu_factor_warp(const DevMech &m, const LUDev &lu, const double *J, double c,
                              const double *scale, double *wsc, LT *LU, LT *x, int lane) {
  for (int p = lane; p < lu.nnz; p += 32) LU[p] = (LT)0;
  for (int i = lane; i < lu.n; i += 32) wsc[i] = scale[i];
  __syncwarp();
  for (int i = lane; i < lu.n; i += 32) {  // Jacobian row i from the row-wise view
    const double ci = -c / scale[i];
    for (int q = m.jr_ptr[i]; q < m.jr_ptr[i + 1]; ++q) {
      const int k = m.jr_kk[q];
      LU[lu.jac_to_lu[k]] = (LT)(ci * J[k] * scale[m.jr_col[q]]);
    }
  }
  __syncwarp();
  for (int i = lane; i < lu.n; i += 32) LU[lu.diag_of_orig[i]] += (LT)1;
  __syncwarp();
  int bad = 0;
  for (int j = 0; j < lu.n; ++j) {
    const int p0 = lu.col_ptr[j], p1 = lu.col_ptr[j + 1], dj = lu.diag[j];
    for (int p = p0 + lane; p < p1; p += 32) x[lu.row_idx[p]] = LU[p];
    __syncwarp();
    for (int p = p0; p < dj; ++p) {
      const int k = lu.row_idx[p];
      const LT xk = x[k];
      if (xk != (LT)0)
        for (int q = lu.diag[k] + 1 + lane; q < lu.col_ptr[k + 1]; q += 32)
          x[lu.row_idx[q]] -= LU[q] * xk;
      __syncwarp();
    }
    const LT piv = x[j];
    if (!(piv != (LT)0) || !isfinite((double)piv)) bad = 1;
    const LT inv = (LT)1 / piv;
    for (int p = p0 + lane; p < p1; p += 32) {
      const int r = lu.row_idx[p];
      const LT val = x[r];
      LU[p] = (r > j) ? val * inv : val;
    }
    __syncwarp();
  }
  return bad;
}

// x <- P^{-1} x in permuted ordering (x in shared memory).
template <class LT>
__device__ void lu_solve_warp(const LUDev &lu, const LT *LU, LT *x, int lane) {
  for (int k = 0; k < lu.n; ++k) {
    const LT xk = x[k];
    if (xk != (LT)0)
      for (int q = lu.diag[k] + 1 + lane; q < lu.col_ptr[k + 1]; q += 32)
        x[lu.row_idx[q]] -= LU[q] * xk;
    __syncwarp();
  }
  for (int k = lu.n - 1; k >= 0; --k) {
    const LT xk = x[k] / LU[lu.diag[k]];
    __syncwarp();
    if (lane == 0) x[k] = xk;
    if (xk != (LT)0)
      for (int q = lu.col_ptr[k] + lane; q < lu.diag[k]; q += 32) x[lu.row_idx[q]] -= LU[q] * xk;
    __syncwarp();
  }
}

// out = (I - c_lu J)^{-1} r from the scaled factor: W LU^-1 (W^-1 r), with
// the permuted solve vector x in shared memory.
template <class LT>
__device__ void precond_warp(const LUDev &lu, const LT *LU, LT *x, const double *wsc, const double *r,
                             double *out, int lane) {
  for (int i = lane; i < lu.n; i += 32) x[lu.iperm[i]] = (LT)(r[i] / wsc[i]);
  __syncwarp();
  lu_solve_warp<LT>(lu, LU, x, lane);
  for (int i = lane; i < lu.n; i += 32) out[i] = (double)x[lu.iperm[i]] * wsc[i];
  __syncwarp();
}

// D[0..order] <- (R(factor) U)^T D[0..order], lanes over the n columns.
__device__ void change_D(double *D, int n, int order, double fac, int lane) {
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
      double s = 0.0;
      for (int k = 0; k <= order; ++k) s += R[i][k] * U[k][j];
      RU[i][j] = s;
    }
  for (int mcol = lane; mcol < n; mcol += 32) {
    double old[kMaxOrder + 1];
    for (int k = 0; k <= order; ++k) old[k] = D[k * n + mcol];
    for (int i = 0; i <= order; ++i) {
      double s = 0.0;
      for (int k = 0; k <= order; ++k) s += RU[k][i] * old[k];
      D[i * n + mcol] = s;
    }
  }
  __syncwarp();
}

struct Vecs {
  double *D, *y, *f, *f0, *ypred, *psi, *d, *scale, *tmp, *J;
  double *wsc;  // scale the stored factor was formed with
  double *K;    // FP32 path: (kMaxl + 1) Krylov vectors, then 2 work vectors
  double *r1g, *r1d, *r1w;  // energy-source coupling: g, d, w = P^-1 g
};

// Energy-source coupling on a Newton solve x = P^-1 b (Sherman-Morrison):
// (P - c g d^T)^-1 b = x + w (r1k d.x), w = P^-1 g, r1k = c / (1 - c d.w).
__device__ void rank1_fix_warp(const Vecs &V, int n, double r1k, double *x, int lane) {
  double a = 0.0;
  for (int i = lane; i < n; i += 32) a += V.r1d[i] * x[i];
  const double dx = wsum(a) * r1k;
  for (int i = lane; i < n; i += 32) x[i] += V.r1w[i] * dx;
  __syncwarp();
}

constexpr int kMaxl = 10;  // Krylov dimension (no restarts)

// Left-preconditioned GMRES for (I - cJ) x = b on one warp, the Newton
// system of the FP32 path: the operator is applied in FP64 from the stored
// sparse Jacobian, the FP32 factor only preconditions, in the error-weighted
// coordinates; SPGMR's method (modified Gram-Schmidt, no restarts, x0 = 0,
// converged when the preconditioned residual's weighted 2-norm is <= delta),
// as the reference plugin drives it through CVODE (solver_cvode.cpp:119-141,
// 201-212), restated from Saad and Schultz, SIAM J. Sci. Stat. Comput. 7
// (1986) 856-869.  Every lane keeps the same Hessenberg matrix.  Under an
// energy source the operator and the preconditioner carry the rank-one
// temperature coupling (r1 set).  Returns 0 when converged, 1 otherwise.
template <class LT>
__device__ int gmres_warp(const DevMech &m, const LUDev &lu, const Vecs &V, const LT *LU, LT *x, double c,
                          double delta, const double *b, double *xo, int lane, int &iters,
                          bool r1, double r1k) {
  const int n = lu.n;
  double *Kv = V.K, *u = V.K + (kMaxl + 1) * n, *z = u + n;
  precond_warp<LT>(lu, LU, x, V.wsc, b, z, lane);
  if (r1) rank1_fix_warp(V, n, r1k, z, lane);
  double a = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double t = z[i] / V.scale[i];
    Kv[i] = t;
    a += t * t;
  }
  const double beta = sqrt(wsum(a));
  if (!isfinite(beta)) return 1;
  if (beta <= delta) {
    for (int i = lane; i < n; i += 32) xo[i] = 0.0;
    __syncwarp();
    return 0;
  }
  double H[kMaxl + 1][kMaxl], cs[kMaxl], sn[kMaxl], g[kMaxl + 1], yk[kMaxl];
  g[0] = beta;
  for (int i = lane; i < n; i += 32) Kv[i] /= beta;
  int nl = 0;
  bool conv = false;
  for (int l = 0; l < kMaxl; ++l) {
    const double *vl = Kv + l * n;
    double *w = Kv + (l + 1) * n;
    double du = 0.0;
    for (int i = lane; i < n; i += 32) {
      u[i] = vl[i] * V.scale[i];
      if (r1) du += V.r1d[i] * u[i];
    }
    if (r1) du = wsum(du);
    __syncwarp();
    for (int i = lane; i < n; i += 32) {  // (I - cJ) u, row i
      double jx = 0.0;
      for (int q = m.jr_ptr[i]; q < m.jr_ptr[i + 1]; ++q) jx += V.J[m.jr_kk[q]] * u[m.jr_col[q]];
      if (r1) jx += V.r1g[i] * du;
      z[i] = u[i] - c * jx;
    }
    __syncwarp();
    precond_warp<LT>(lu, LU, x, V.wsc, z, z, lane);
    if (r1) rank1_fix_warp(V, n, r1k, z, lane);
    for (int i = lane; i < n; i += 32) w[i] = z[i] / V.scale[i];
    __syncwarp();
    for (int k = 0; k <= l; ++k) {  // modified Gram-Schmidt
      const double *vk = Kv + k * n;
      double d = 0.0;
      for (int i = lane; i < n; i += 32) d += w[i] * vk[i];
      const double h = wsum(d);
      H[k][l] = h;
      for (int i = lane; i < n; i += 32) w[i] -= h * vk[i];
    }
    double d2 = 0.0;
    for (int i = lane; i < n; i += 32) d2 += w[i] * w[i];
    const double hn = sqrt(wsum(d2));
    for (int k = 0; k < l; ++k) {
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
    const double rho = fabs(g[l + 1]);
    nl = l + 1;
    ++iters;
    if (hn > 0.0)
      for (int i = lane; i < n; i += 32) w[i] /= hn;
    __syncwarp();
    if (!isfinite(rho)) return 1;
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
  for (int i = lane; i < n; i += 32) {
    double acc = 0.0;
    for (int k = 0; k < nl; ++k) acc += yk[k] * Kv[k * n + i];
    xo[i] = acc * V.scale[i];
  }
  __syncwarp();
  return conv ? 0 : 1;
}

__device__ __forceinline__ double wrms_scaled(const double *x, const double *s, int n, int lane) {
  double a = 0.0;
  for (int i = lane; i < n; i += 32) {
    const double t = x[i] / s[i];
    a += t * t;
  }
  return sqrt(wsum(a) / n);
}

// One integration attempt from t = 0 to t_end; y holds the start state and,
// on return, the last accepted state, reached at t_done.  Returns 0 or a
// negative failure code.
template <class LT>
__device__ int bdf_attempt(const DevMech &m, const LUDev &lu, const IntegOpts &o, const BdfConst &bc,
                           const Warp &w, const Vecs &V, LT *LU, double v, double t_end,
                           double rtol, double atol, ReactorStats &st, int lane, double &t_done,
                           double t_off, double T_target, double &t_ign, CbCtx &cb) {
  const int n = m.nsp + 1;
  LT *x = (LT *)w.X;
  double t = 0.0;
  int rc = 0;
  t_done = 0.0;
  double T_prev = V.y[m.nsp] * o.Tref;  // ignition: temperature at the last accepted step
  const bool r1 = w.src.esrc != 0.0;
  double r1k = 0.0;  // energy-source coupling of the current factor
  auto rank1_setup = [&](double cc) {
    if (!r1) return;
    precond_warp<LT>(lu, LU, x, V.wsc, V.r1g, V.r1w, lane);
    double a = 0.0;
    for (int i = lane; i < n; i += 32) a += V.r1d[i] * V.r1w[i];
    const double dw = wsum(a);
    r1k = cc / (1.0 - cc * dw);
  };
  // f0 = f(y0); initial step (Hairer-Norsett-Wanner)
  st.nrhs++;
  if (rhs_warp(m, o, w, v, t_off, V.y, V.f0, lane, false, nullptr)) return -1;
  // absolute tolerance of component i (abstol_dens: reactor_nvector_serial.cpp:107-119)
  auto atol_of = [&](int i) {
    return (o.abstol_dens && i < m.nsp) ? atol * (1.0 / ((1.0 / v) * m.inv_mw[i] * 1.0e-3)) : atol;
  };
  for (int i = lane; i < n; i += 32) V.scale[i] = atol_of(i) + fabs(V.y[i]) * rtol;
  __syncwarp();
  const double d0 = wrms_scaled(V.y, V.scale, n, lane), d1 = wrms_scaled(V.f0, V.scale, n, lane);
  double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
  if (h0 > t_end) h0 = t_end;
  for (int i = lane; i < n; i += 32) V.tmp[i] = V.y[i] + h0 * V.f0[i];
  __syncwarp();
  double d2 = 0.0;
  st.nrhs++;
  if (rhs_warp(m, o, w, v, t_off + h0, V.tmp, V.f, lane, false, nullptr) == 0) {
    for (int i = lane; i < n; i += 32) V.d[i] = V.f[i] - V.f0[i];
    __syncwarp();
    d2 = wrms_scaled(V.d, V.scale, n, lane) / h0;
  }
  double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : sqrt(0.01 / fmax(d1, d2));
  double h = fmin(100.0 * h0, h1);
  h = fmin(h, o.max_dt);
  h = fmin(h, t_end);
  int q = 1, neq = 0, jac_current = 1, nsteps = 0;
  double c_lu = h / bc.alp[q], crate = 1.0;
  for (int i = lane; i < (kMaxOrder + 3) * n; i += 32) V.D[i] = 0.0;
  __syncwarp();
  for (int i = lane; i < n; i += 32) {
    V.D[i] = V.y[i];
    V.D[n + i] = V.f0[i] * h;
  }
  __syncwarp();
  st.njac++;
  if (jac_warp(m, o, w, v, t_off, V.y, V.f0, V.J, V.tmp, V.d, V.r1g, V.r1d, lane)) { rc = -2; goto failed; }
  st.nlu++;
  if (lu_factor_warp<LT>(m, lu, V.J, c_lu, V.scale, V.wsc, LU, x, lane)) { rc = -3; goto failed; }
  rank1_setup(c_lu);
  while (t < t_end) {
    if (nsteps >= o.max_steps) { rc = -4; goto failed; }
    bool accepted = false;
    double safety = 0.9, err_norm = 0.0;
    int nef = 0, ncf = 0;  // this step's error-test and convergence failures
    while (!accepted) {
      if (h > o.max_dt) {
        change_D(V.D, n, q, o.max_dt / h, lane);
        h = o.max_dt;
      }
      if (t + h > t_end) {
        change_D(V.D, n, q, (t_end - t) / h, lane);
        h = t_end - t;
      }
      if (!(t + h > t)) { rc = -5; goto failed; }  // no progress (or h not finite)
      const double t_new = t + h;
      for (int i = lane; i < n; i += 32) {
        double s = 0.0, ps = 0.0;
        for (int k = 0; k <= q; ++k) s += V.D[k * n + i];
        for (int k = 1; k <= q; ++k) ps += bc.gam[k] * V.D[k * n + i];
        V.ypred[i] = s;
        V.psi[i] = ps / bc.alp[q];
        V.scale[i] = atol_of(i) + rtol * fabs(s);
        V.y[i] = s;
        V.d[i] = 0.0;
      }
      __syncwarp();
      const double c = h / bc.alp[q];
      if (fabs(c / c_lu - 1.0) > 0.3) {
        st.nlu++;
        c_lu = c;
        crate = 1.0;
        if (lu_factor_warp<LT>(m, lu, V.J, c, V.scale, V.wsc, LU, x, lane)) { rc = -3; goto failed; }
        rank1_setup(c);
      }
      const double gscale = (c == c_lu) ? 1.0 : 2.0 / (1.0 + c / c_lu);
      bool conv = false;
      int it;
      double dnorm_old = -1.0;
      for (it = 0; it < kNewtonMaxIter; ++it) {
        st.nrhs++;
        if (rhs_warp(m, o, w, v, t_off + t_new, V.y, V.f, lane, false, nullptr)) break;
        bool finite = true;
        for (int i = lane; i < n; i += 32) finite &= isfinite(V.f[i]);
        if (!__all_sync(kFull, finite)) break;
        if (it == 0)
          for (int i = lane; i < n; i += 32) V.f0[i] = V.f[i];
        st.nnewt++;
        for (int i = lane; i < n; i += 32) V.tmp[i] = c * V.f[i] - V.psi[i] - V.d[i];
        __syncwarp();
        double gs = gscale;
        if constexpr (sizeof(LT) == sizeof(float)) {
          // FP32 factor as the preconditioner of an FP64 Krylov solve with
          // tolerance eps_lin * nlscoef / error constant (WRMS); every solve
          // must converge (see integrator_dense.cuh)
          const double delta = o.eps_lin * o.nlscoef / bc.econ[q] * sqrt((double)n);
          if (gmres_warp<LT>(m, lu, V, LU, x, c, delta, V.tmp, V.tmp, lane, st.nkry, r1, r1k) != 0)
            break;
          gs = 1.0;
        } else {
          precond_warp<LT>(lu, LU, x, V.wsc, V.tmp, V.tmp, lane);
          if (r1) rank1_fix_warp(V, n, r1k, V.tmp, lane);
        }
        double a = 0.0;
        for (int i = lane; i < n; i += 32) {
          const double dy = V.tmp[i] * gs;
          V.y[i] += dy;
          V.d[i] += dy;
          const double tt = dy / V.scale[i];
          a += tt * tt;
        }
        const double dn = sqrt(wsum(a) / n);
        __syncwarp();
        if (dnorm_old > 0.0) crate = fmax(0.3 * crate, dn / dnorm_old);
        if (bc.econ[q] * dn * fmin(1.0, crate) <= o.nlscoef) {
          conv = true;
          ++it;
          break;
        }
        if (dnorm_old > 0.0 && dn > 2.0 * dnorm_old) break;
        dnorm_old = dn;
      }
      if (!conv) {
        if (!jac_current) {
          st.nrhs++;
          if (rhs_warp(m, o, w, v, t_off + t_new, V.ypred, V.f0, lane, false, nullptr)) { rc = -6; goto failed; }
          st.njac++;
          if (jac_warp(m, o, w, v, t_off + t_new, V.ypred, V.f0, V.J, V.tmp, V.f, V.r1g, V.r1d, lane)) {
            rc = -2;
            goto failed;
          }
          jac_current = 1;
          st.nlu++;
          c_lu = c;
          crate = 1.0;
          if (lu_factor_warp<LT>(m, lu, V.J, c, V.scale, V.wsc, LU, x, lane)) { rc = -3; goto failed; }
          rank1_setup(c);
          continue;
        }
        if (++ncf >= kMaxConvFails) { rc = -8; goto failed; }
        change_D(V.D, n, q, 0.5, lane);
        h *= 0.5;
        st.nrej++;
        continue;
      }
      safety = 0.9 * (2 * kNewtonMaxIter + 1) / (2.0 * kNewtonMaxIter + it);
      double a = 0.0;
      for (int i = lane; i < n; i += 32) {
        const double e = bc.econ[q] * V.d[i] / V.scale[i];
        a += e * e;
      }
      err_norm = sqrt(wsum(a) / n);
      if (!isfinite(err_norm)) { rc = -7; goto failed; }
      if (err_norm > 1.0) {
        if (++nef >= kMaxErrTestFails) { rc = -9; goto failed; }
        st.nrej++;
        if (nef > kErrFailsBeforeCut) {  // order and step cut (integrator.h)
          if (q > 1) {
            --q;
            change_D(V.D, n, q, kEtaMinErrFail, lane);
          } else {
            st.nrhs++;
            if (rhs_warp(m, o, w, v, t_off + t, V.D, V.tmp, lane, false, nullptr)) { rc = -6; goto failed; }
            for (int i = lane; i < n; i += 32) V.D[n + i] = V.tmp[i] * (h * kEtaMinErrFail);
            __syncwarp();
          }
          h *= kEtaMinErrFail;
          neq = 0;
          continue;
        }
        const double fac = fmax(kMinFactor, safety * pow(err_norm, -1.0 / (q + 1)));
        change_D(V.D, n, q, fac, lane);
        h *= fac;
        continue;
      }
      accepted = true;
      t = t_new;
    }
    ++nsteps;
    st.nsteps++;
    ++neq;
    jac_current = 0;
    const bool keep_prev = T_target > 0.0 && o.stop_ign && t_ign < 0.0;
    for (int i = lane; i < n; i += 32) {
      if (keep_prev) V.tmp[i] = V.D[i];  // the previous accepted state
      const double di = V.d[i];
      V.D[(q + 2) * n + i] = di - V.D[(q + 1) * n + i];
      V.D[(q + 1) * n + i] = di;
      for (int k = q; k >= 0; --k) V.D[k * n + i] += V.D[(k + 1) * n + i];
    }
    __syncwarp();
    if (T_target > 0.0) {  // first crossing of T0 + dT_ign, linear between accepted steps
      const double Tn = V.D[n - 1] * o.Tref;
      if (t_ign < 0.0 && Tn >= T_target) {
        const double frac = (Tn > T_prev) ? (T_target - T_prev) / (Tn - T_prev) : 1.0;
        t_ign = t_off + (t - h) + frac * h;
        // the callback's record of CVode's root return (solver_cvode.cpp:249-262)
        const bool cb_end = cb.rec && cb_record(cb, V.D, o.stop_ign ? V.tmp : nullptr, n, q, h,
                                                frac - 1.0, frac, t_ign, V.y, lane, 32);
        if (o.stop_ign || cb_end) {  // stop_after_ignition: the call ends at the crossing
          if (!cb_end)
            for (int i = lane; i < n; i += 32) V.y[i] = V.tmp[i] + frac * (V.D[i] - V.tmp[i]);
          __syncwarp();
          t_done = (t - h) + frac * h;
          return 0;
        }
      }
      T_prev = Tn;
    }
    if (cb.rec && cb_record(cb, V.D, nullptr, n, q, h, 0.0, 0.0, t_off + t, V.y, lane, 32)) {
      __syncwarp();  // the callback asked to stop here
      t_done = t;
      return 0;
    }
    if (neq < q + 1) continue;
    double em = INFINITY, ep = INFINITY;
    if (q > 1) {
      double a = 0.0;
      for (int i = lane; i < n; i += 32) {
        const double e = bc.econ[q - 1] * V.D[q * n + i] / V.scale[i];
        a += e * e;
      }
      em = sqrt(wsum(a) / n);
    }
    if (q < kMaxOrder) {
      double a = 0.0;
      for (int i = lane; i < n; i += 32) {
        const double e = bc.econ[q + 1] * V.D[(q + 2) * n + i] / V.scale[i];
        a += e * e;
      }
      ep = sqrt(wsum(a) / n);
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
    if (fac < kEtaKeep) fac = 1.0;  // CVODE's step-size hysteresis
    change_D(V.D, n, q, fac, lane);
    h *= fac;
    neq = 0;
  }
  for (int i = lane; i < n; i += 32) V.y[i] = V.D[i];
  __syncwarp();
  t_done = t;
  return 0;
failed:  // D[0] holds the last accepted state (step-size changes keep it)
  for (int i = lane; i < n; i += 32) V.y[i] = V.D[i];
  __syncwarp();
  t_done = t;
  return rc;
}

template <class LT>
__global__ void __launch_bounds__(384, 1) integrate_kernel(DevMech m, LUDev lu, IntegOpts o,
                                                        IntegArgs a, int rop_in_smem,
                                                        int per_warp) {
  extern __shared__ double smem_dyn[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int S = m.nsp, n = S + 1, N = m.nstep;
  double *base = smem_dyn + wid * per_warp;
  Warp w;
  w.C = base;
  w.G = base + S;
  w.U = base + 2 * S;
  double *after = base + 3 * S;
  if (rop_in_smem) {
    w.ROP = after;
    after += N;
  } else {
    const int slot = blockIdx.x * (blockDim.x >> 5) + wid;
    w.ROP = a.rop_scratch + (size_t)slot * N;
  }
  w.X = after;
  w.ysrc = nullptr;
  BdfConst bc;
  bdf_consts(bc);
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(a.queue_head, 1);
    idx = __shfl_sync(kFull, idx, 0);
    if (idx >= a.n_reactors) break;
    const int r = a.order ? a.order[idx] : idx;
    double *st = a.state + (size_t)r * a.state_stride;
    Vecs V;
    V.D = st;
    V.y = st + (kMaxOrder + 3) * n;
    V.f = V.y + n;
    V.f0 = V.f + n;
    V.ypred = V.f0 + n;
    V.psi = V.ypred + n;
    V.d = V.psi + n;
    V.scale = V.d + n;
    V.tmp = V.scale + n;
    V.J = V.tmp + n;
    V.wsc = V.J + m.nnz;
    V.K = V.wsc + n;
    V.r1g = V.K + (kMaxl + 3) * n;
    V.r1d = V.r1g + n;
    V.r1w = V.r1d + n;
    LT *LU = (LT *)a.lu + (size_t)r * a.lu_stride;
    // InitializeState (reactor_constant_volume_cpu.cpp:15-41)
    const double T0 = a.T[r], P0 = a.P[r];
    const double *Y0 = a.Y + (size_t)r * S;
    double pa = 0.0;
    for (int s = lane; s < S; s += 32) pa += Y0[s] * m.inv_mw[s];
    const double mwmix = 1.0 / wsum(pa);
    const double v = 1.0 / (P0 * mwmix / (kRuD * T0));
    w.src.dpdt = a.dpdt ? a.dpdt[r] : 0.0;
    w.src.esrc = a.esrc ? a.esrc[r] : 0.0;
    w.src.P0 = P0;
    w.src.ysrc = a.ysrc != nullptr;
    w.src.fixT = !o.always_T && a.tdel_in && !(a.tdel_in[r] > 0.0);
    w.src.T0 = T0;
    w.src.E0 = 0.0;
    if (w.src.esrc != 0.0 || w.src.fixT) {  // initial_energy_ (InitializeState)
      double cx;
      mix_energy(m, o.cp != 0, false, T0, Y0, false, 0.0, lane, 32,
                 [](double x) { return wsum(x); }, w.src.E0, cx);
    }
    for (int s = lane; s < S; s += 32) V.y[s] = Y0[s];
    if (lane == 0) V.y[S] = T0 / o.Tref;
    __syncwarp();
    ReactorStats rs = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    CbCtx cb{a.cb_rec ? a.cb_rec + (size_t)idx * a.cb_cap * (3 + 2 * (size_t)n) : nullptr, a.cb_cap,
             (a.cb_rec && a.cb_stop) ? a.cb_stop[r] : 0, 0, 0, 0.0};
    double rtol = o.rtol, atol = o.atol;
    int rc = 0;
    double t_left = a.dt, t_ign = -1.0;
    const double T_target = o.dT_ign > 0.0 ? T0 + o.dT_ign : -1.0;
    w.ysrc = a.ysrc ? a.ysrc + (size_t)r * S : nullptr;
    for (int attempt = 0;; ++attempt) {
      double t_done = 0.0;
      rc = bdf_attempt<LT>(m, lu, o, bc, w, V, LU, v, t_left, rtol, atol, rs, lane, t_done, a.dt - t_left,
                           T_target, t_ign, cb);
      if (rc == 0 || attempt + 1 >= o.max_retries) break;
      cb.ncalls++;  // the failed CVode call counts as a step
      t_left -= t_done;
      // solver_cvode.cpp:236-246: adjust tolerances and start over from the
      // last accepted state for the remaining time
      rs.retries++;
      atol *= o.retry_atol_factor;
      rtol *= o.retry_rtol_factor;
    }
    rs.status = rc;
    // GetState (reactor_constant_volume_cpu.cpp:43-61)
    if (rc == 0) {
      double pb = 0.0;
      for (int s = lane; s < S; s += 32) {
        const double ys = V.y[s];
        a.Y[(size_t)r * S + s] = ys;
        pb += ys * m.inv_mw[s];
      }
      const double mw2 = 1.0 / wsum(pb);
      const double Tn = end_temperature(m, o.cp != 0, w.src, a.dt, V.y, V.y[S] * o.Tref, lane, 32,
                                        [](double x) { return wsum(x); });
      if (lane == 0) {
        a.T[r] = Tn;
        a.P[r] = end_pressure(o.cp != 0, w.src, a.dt, Tn, mw2, v);
      }
    }
    if (lane == 0) {
      a.v[r] = v;
      if (a.stats) a.stats[r] = rs;
      if (a.cb_cnt) a.cb_cnt[r] = cb.cnt;
      if (a.t_ign) a.t_ign[r] = t_ign;
    }
    __syncwarp();
  }
}

}  // namespace

size_t integ_smem_per_warp(const DevMech &m, const LUDev &lu, bool rop_in_smem) {
  size_t d = 3 * (size_t)m.nsp + (rop_in_smem ? m.nstep : 0) + lu.n + 1;
  return ((d * sizeof(double) + 15) / 16) * 16;
}

long integ_state_doubles(const DevMech &m, const LUDev &lu) {
  const long n = m.nsp + 1;
  return (kMaxOrder + 3) * n + 8 * n + m.nnz + n + (kMaxl + 3) * n + 3 * n;
}

cudaError_t launch_integrate(const DevMech &m, const LUDev &lu, const IntegOpts &o,
                             const IntegArgs &a, int warps_per_cta, int ctas, bool rop_in_smem,
                             cudaStream_t stream) {
  const size_t smem = integ_smem_per_warp(m, lu, rop_in_smem) * warps_per_cta;
  const int pw = (int)(integ_smem_per_warp(m, lu, rop_in_smem) / sizeof(double));
  cudaError_t e;
  if (o.lu_fp32) {
    e = cudaFuncSetAttribute(integrate_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    integrate_kernel<float><<<ctas, warps_per_cta * 32, smem, stream>>>(m, lu, o, a, rop_in_smem, pw);
  } else {
    e = cudaFuncSetAttribute(integrate_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    integrate_kernel<double><<<ctas, warps_per_cta * 32, smem, stream>>>(m, lu, o, a, rop_in_smem, pw);
  }
  return cudaGetLastError();
}

}  // namespace zrk
