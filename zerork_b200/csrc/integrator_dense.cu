// integrator_dense.cu -- CTA-per-reactor BDF integration with the Newton
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
#include <cuda_runtime.h>

#include "integrator.h"
#include "kinetics_dev.cuh"

namespace zrk {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kNewtonMaxIter = 3;
constexpr double kMinFactor = 0.2;
constexpr double kMaxFactor = 10.0;
constexpr double kEtaKeep = 1.5;
constexpr int kMaxl = 5;  // Krylov dimension (SPGMR default, no restarts)

struct Smem {
  double *red;  // 2*32 reduction slots
  double *C, *G, *U, *ROP;
  double *D, *y, *f, *f0, *ypred, *psi, *d, *scale, *tmp, *yp;
  void *A;      // n x lda inverse (LT)
  int *piv;     // n
  double *colk; // n (LT-sized use)
  double *wlu;  // n: error-weight scale the stored inverse was formed with
  double *bs;   // n: scaled right-hand side
  double *V;    // FP32 path: (kMaxl + 1) Krylov vectors, then 2 work vectors
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

// ydot at y (shared vector); returns 1 if T <= 0 (all threads agree).
__device__ int rhs_cta(const DevMech &m, const IntegOpts &o, const Smem &s, double v,
                       const double *y, double *ydot, bool clamp, double *cv_out) {
  const int S = m.nsp, tid = threadIdx.x, nt = blockDim.x;
  const double yS = y[S];
  double T = yS * o.Tref;
  if (!(T > 0.0)) return 1;
  if (T > 1.0e4) T = 1.0e4;
  const double logT = log(T), invT = 1.0 / T, lprt = log(kPatmD / (kRuD * T));
  const double dens = 1.0 / v;
  double pc = 0.0, pcv = 0.0;
  for (int k = tid; k < S; k += nt) {
    double ys = y[k];
    if (clamp) ys = clamp_mass_fraction(ys, o.mmf);
    const double c = dens * m.inv_mw[k] * ys;
    s.C[k] = c;
    double cp, h, g;
    nasa_cp_h_g(m.thermo + 16 * k, T, logT, &cp, &h, &g);
    s.G[k] = g;
    s.U[k] = h - 1.0;
    pc += c;
    pcv += ((cp - 1.0) * m.ru_inv_mw[k]) * ys;
  }
  const double Csum = block_sum(pc, s.red);
  const double cv = block_sum(pcv, s.red);
  for (int r = tid; r < m.nrxn; r += nt)
    reaction_item<1, 1>(m, m.rxn[r], 0, s.C, s.G, s.ROP, &T, &logT, &invT, &lprt, &Csum, o.lim);
  __syncthreads();
  double pe = 0.0;
  for (int k = tid; k < S; k += nt) {
    double des = 0.0, cre = 0.0;
    for (int q = m.sd_ptr[k]; q < m.sd_ptr[k + 1]; ++q) des += s.ROP[m.sd_step[q]];
    for (int q = m.sc_ptr[k]; q < m.sc_ptr[k + 1]; ++q) cre += s.ROP[m.sc_step[q]];
    const double net = cre - des;
    ydot[k] = net * m.mw[k] * v;
    pe += s.U[k] * net * v;
  }
  const double es = block_sum(pe, s.red);
  if (tid == 0) ydot[S] = -es * kRuD * yS / cv + 0.0;
  if (cv_out) *cv_out = cv;
  __syncthreads();
  return 0;
}

// Reactor Jacobian (SetupJacobianSparse semantics) into J (global, nnz).
__device__ int jac_cta(const DevMech &m, const IntegOpts &o, const Smem &s, double v,
                       const double *y, const double *fy, double *J) {
  const int S = m.nsp, tid = threadIdx.x, nt = blockDim.x;
  int need = 0;
  for (int k = tid; k < S; k += nt) need |= (fabs(y[k]) < o.mmf);
  need = __syncthreads_or(need);
  double cvc;
  if (rhs_cta(m, o, s, v, y, s.tmp, need != 0, &cvc)) return 1;
  const double TdC = s.tmp[S];
  const double yS = y[S];
  const double RuTemp = kRuD * yS;
  const double multFact = -1.0 / cvc;
  double T = yS * o.Tref;
  if (T > 1.0e4) T = 1.0e4;
  for (int j = tid; j < S; j += nt) {  // one column per thread
    const double t2 = m.mw[j] / clamp_mass_fraction(y[j], o.mmf) * v;
    const int k0 = m.col_ptr[j], k1 = m.col_ptr[j + 1] - 1;
    const double wcol = m.inv_mw[j];
    double trow = 0.0;
    for (int kk = k0; kk < k1; ++kk) {
      const int row = m.row_idx[kk];
      double des = 0.0, cre = 0.0;
      for (int q = m.nzd_ptr[kk]; q < m.nzd_ptr[kk + 1]; ++q) des += s.ROP[m.nzd_step[q]];
      for (int q = m.nzc_ptr[kk]; q < m.nzc_ptr[kk + 1]; ++q) cre += s.ROP[m.nzc_step[q]];
      const double val = (0.0 - des * t2) + cre * t2;
      trow += val * s.U[row];
      J[kk] = val * (m.mw[row] * wcol);
    }
    const double cvj = (nasa_cp(m.thermo + 16 * j, T) - 1.0) * m.ru_inv_mw[j];
    double tr = trow * RuTemp;
    tr += TdC * cvj * m.mw[j];
    tr *= wcol * multFact;
    J[k1] = tr;
  }
  __syncthreads();
  const double ySp = yS + yS * o.sqrt_ur;
  const double mult = 1.0 / (ySp - yS);
  for (int k = tid; k < S; k += nt) s.yp[k] = y[k];
  if (tid == 0) s.yp[S] = ySp;
  __syncthreads();
  if (rhs_cta(m, o, s, v, s.yp, s.tmp, false, nullptr)) return 1;
  for (int kk = m.col_ptr[S] + tid; kk < m.col_ptr[S + 1]; kk += nt) {
    const int row = m.row_idx[kk];
    J[kk] = (s.tmp[row] - fy[row]) * mult;
  }
  __syncthreads();
  return 0;
}

// A <- (W (I - cJ) W^-1)^{-1} with W = diag(1/scale) the error weights of
// the current step (scale = atol + rtol |y|): the similarity transform turns
// J_ij into J_ij scale_j / scale_i, the Jacobian of relative changes, which
// is far better balanced than J for species spanning 20 decades of mass
// fraction and keeps the single-precision inverse accurate in the weighted
// norm the Newton test uses.  Gauss-Jordan with partial pivoting in shared
// memory.  Returns nonzero (all threads) for a singular or non-finite matrix.
template <class LT>
__device__ int invert_cta(const DevMech &m, const Smem &s, const double *J, double c, int n, int lda) {
  LT *A = (LT *)s.A;
  LT *colk = (LT *)s.colk;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < n * lda; i += nt) A[i] = (LT)0;
  for (int i = tid; i < n; i += nt) s.wlu[i] = s.scale[i];
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
  int bad = 0;
  for (int k = 0; k < n; ++k) {
    // pivot search: warp argmax then across warps
    double best = -1.0;
    int bi = k;
    for (int i = k + tid; i < n; i += nt) {
      const double a = fabs((double)A[i * lda + k]);
      if (a > best) { best = a; bi = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(kFull, best, o);
      const int oi = __shfl_xor_sync(kFull, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    __syncthreads();
    if ((tid & 31) == 0) {
      s.red[tid >> 5] = best;
      s.red[32 + (tid >> 5)] = (double)bi;
    }
    __syncthreads();
    if (tid == 0) {
      double b = -1.0;
      int p = k;
      for (int w = 0; w < (nt >> 5); ++w)
        if (s.red[w] > b) { b = s.red[w]; p = (int)s.red[32 + w]; }
      s.piv[k] = p;
      s.red[64] = b;
    }
    __syncthreads();
    const int p = s.piv[k];
    if (!(s.red[64] > 0.0) || !isfinite(s.red[64])) bad = 1;
    if (p != k)
      for (int j = tid; j < n; j += nt) {
        const LT t = A[k * lda + j];
        A[k * lda + j] = A[p * lda + j];
        A[p * lda + j] = t;
      }
    __syncthreads();
    const LT pinv = (LT)1 / A[k * lda + k];
    for (int i = tid; i < n; i += nt) colk[i] = A[i * lda + k];
    __syncthreads();
    for (int j = tid; j < n; j += nt) A[k * lda + j] = (j == k ? (LT)1 : A[k * lda + j]) * pinv;
    __syncthreads();
    // rank-1 update: warp w owns rows i = w (mod warps), lane l the columns
    // j = l (mod 32); rows whose multiplier is zero (untouched by the fill
    // so far) are skipped whole.
    {
      const int lane = tid & 31, nw = nt >> 5;
      const LT *Ak = A + k * lda;
      for (int i = tid >> 5; i < n; i += nw) {
        const LT f = colk[i];
        if (i == k || f == (LT)0) continue;
        LT *Ai = A + i * lda;
        for (int j = lane; j < n; j += 32) {
          const LT a = (j == k) ? (LT)0 : Ai[j];
          Ai[j] = a - f * Ak[j];
        }
      }
    }
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {  // undo the row interchanges on columns
    const int p = s.piv[k];
    if (p != k)
      for (int i = tid; i < n; i += nt) {
        const LT t = A[i * lda + k];
        A[i * lda + k] = A[i * lda + p];
        A[i * lda + p] = t;
      }
    __syncthreads();
  }
  return __syncthreads_or(bad);
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

__device__ void make_consts(Consts &b) {
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

// x = (I - c_lu J)^{-1} b = W^-1 A W b (A the stored inverse), into x (shared).
template <class LT>
__device__ void apply_inverse(const Smem &s, int n, int lda, const double *b, double *x) {
  const LT *A = (const LT *)s.A;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s.bs[i] = b[i] / s.wlu[i];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double acc = 0.0;
    const LT *row = A + (size_t)i * lda;
    for (int j = 0; j < n; ++j) acc += (double)row[j] * s.bs[j];
    x[i] = acc * s.wlu[i];
  }
  __syncthreads();
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
__device__ int gmres_cta(const DevMech &m, const Smem &s, const double *J, double c, int n, int lda,
                         double delta, const double *b, double *x) {
  const int tid = threadIdx.x, nt = blockDim.x;
  double *V = s.V, *u = s.V + (kMaxl + 1) * n, *z = u + n;
  apply_inverse<LT>(s, n, lda, b, z);
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
    for (int i = tid; i < n; i += nt) u[i] = vl[i] * s.scale[i];
    __syncthreads();
    for (int i = tid; i < n; i += nt) {  // (I - cJ) u, row i
      double jx = 0.0;
      for (int q = m.jr_ptr[i]; q < m.jr_ptr[i + 1]; ++q) jx += J[m.jr_kk[q]] * u[m.jr_col[q]];
      s.colk[i] = u[i] - c * jx;
    }
    __syncthreads();
    apply_inverse<LT>(s, n, lda, s.colk, z);
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

template <class LT>
__device__ int attempt_cta(const DevMech &m, const IntegOpts &o, const Consts &bc, const Smem &s,
                           double *J, double v, double t_end, double rtol, double atol,
                           ReactorStats &st, int lda, double &t_done) {
  const int n = m.nsp + 1, tid = threadIdx.x, nt = blockDim.x;
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
  st.nrhs++;
  if (rhs_cta(m, o, s, v, s.y, s.f0, false, nullptr)) return -1;
  for (int i = tid; i < n; i += nt) s.scale[i] = atol + fabs(s.y[i]) * rtol;
  __syncthreads();
  const double d0 = vrms(s.y, s.scale), d1 = vrms(s.f0, s.scale);
  double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
  if (h0 > t_end) h0 = t_end;
  for (int i = tid; i < n; i += nt) s.tmp[i] = s.y[i] + h0 * s.f0[i];
  __syncthreads();
  double d2 = 0.0;
  st.nrhs++;
  if (rhs_cta(m, o, s, v, s.tmp, s.f, false, nullptr) == 0) {
    for (int i = tid; i < n; i += nt) s.d[i] = s.f[i] - s.f0[i];
    __syncthreads();
    d2 = vrms(s.d, s.scale) / h0;
  }
  double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : sqrt(0.01 / fmax(d1, d2));
  double h = fmin(100.0 * h0, h1);
  h = fmin(h, o.max_dt);
  h = fmin(h, t_end);
  int q = 1, neq = 0, jac_current = 1, nsteps = 0;
  double c_lu = h / bc.alp[q], crate = 1.0;
  for (int i = tid; i < (kMaxOrder + 3) * n; i += nt) s.D[i] = 0.0;
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    s.D[i] = s.y[i];
    s.D[n + i] = s.f0[i] * h;
  }
  __syncthreads();
  st.njac++;
  if (jac_cta(m, o, s, v, s.y, s.f0, J)) { rc = -2; goto failed; }
  st.nlu++;
  if (invert_cta<LT>(m, s, J, c_lu, n, lda)) { rc = -3; goto failed; }
  while (t < t_end) {
    if (nsteps >= o.max_steps) { rc = -4; goto failed; }
    bool accepted = false;
    double safety = 0.9, err_norm = 0.0;
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
        s.scale[i] = atol + rtol * fabs(a);
        s.y[i] = a;
        s.d[i] = 0.0;
      }
      __syncthreads();
      const double c = h / bc.alp[q];
      if (fabs(c / c_lu - 1.0) > 0.3) {
        st.nlu++;
        c_lu = c;
        crate = 1.0;
        if (invert_cta<LT>(m, s, J, c, n, lda)) { rc = -3; goto failed; }
      }
      const double gscale = (c == c_lu) ? 1.0 : 2.0 / (1.0 + c / c_lu);
      bool conv = false;
      int it;
      double dnorm_old = -1.0;
      for (it = 0; it < kNewtonMaxIter; ++it) {
        st.nrhs++;
        if (rhs_cta(m, o, s, v, s.y, s.f, false, nullptr)) break;
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
          // weighted 2-norm; a reduced but unconverged residual is accepted
          // on the first Newton iteration only
          const double delta = o.eps_lin * o.nlscoef / bc.econ[q] * sqrt((double)n);
          const int lrc = gmres_cta<LT>(m, s, J, c, n, lda, delta, s.tmp, s.yp);
          if (lrc == 2 || (lrc == 1 && it > 0)) break;
          gs = 1.0;  // the Krylov solve uses the current c exactly
        } else {
          apply_inverse<LT>(s, n, lda, s.tmp, s.yp);
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
          if (rhs_cta(m, o, s, v, s.ypred, s.f0, false, nullptr)) { rc = -6; goto failed; }
          st.njac++;
          if (jac_cta(m, o, s, v, s.ypred, s.f0, J)) { rc = -2; goto failed; }
          jac_current = 1;
          st.nlu++;
          c_lu = c;
          crate = 1.0;
          if (invert_cta<LT>(m, s, J, c, n, lda)) { rc = -3; goto failed; }
          continue;
        }
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
        const double fac = fmax(kMinFactor, safety * pow(err_norm, -1.0 / (q + 1)));
        change_D_cta(s.D, n, q, fac);
        h *= fac;
        st.nrej++;
        continue;
      }
      accepted = true;
      t = t_new;
    }
    ++nsteps;
    st.nsteps++;
    ++neq;
    jac_current = 0;
    for (int i = tid; i < n; i += nt) {
      const double di = s.d[i];
      s.D[(q + 2) * n + i] = di - s.D[(q + 1) * n + i];
      s.D[(q + 1) * n + i] = di;
      for (int k = q; k >= 0; --k) s.D[k * n + i] += s.D[(k + 1) * n + i];
    }
    __syncthreads();
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
  double *g = a.rop_scratch + (size_t)blockIdx.x * ((size_t)N + (kMaxOrder + 3) * (size_t)n);
  s.red = p; p += 72;
  s.C = p; p += S;
  s.G = p; p += S;
  s.U = p; p += S;
  if (spill & 1) { s.ROP = g; } else { s.ROP = p; p += N; }
  if (spill & 2) { s.D = g + N; } else { s.D = p; p += (kMaxOrder + 3) * n; }
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
  s.piv = (int *)p; p += (n + 1) / 2 + 1;
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
    double *J = a.state + (size_t)r * a.state_stride;
    const double T0 = a.T[r], P0 = a.P[r];
    const double *Y0 = a.Y + (size_t)r * S;
    double pa = 0.0;
    for (int k = tid; k < S; k += nt) pa += Y0[k] * m.inv_mw[k];
    const double mwmix = 1.0 / block_sum(pa, s.red);
    const double v = 1.0 / (P0 * mwmix / (kRuD * T0));
    for (int k = tid; k < S; k += nt) s.y[k] = Y0[k];
    if (tid == 0) s.y[S] = T0 / o.Tref;
    __syncthreads();
    ReactorStats rs = {0, 0, 0, 0, 0, 0, 0, 0};
    double rtol = o.rtol, atol = o.atol;
    int rc = 0;
    // retries (solver_cvode.cpp:227-246): restart the method from the last
    // accepted state for the remaining time with adjusted tolerances;
    // max_steps counts per attempt
    double t_left = a.dt;
    for (int attempt = 0;; ++attempt) {
      double t_done = 0.0;
      rc = attempt_cta<LT>(m, o, bc, s, J, v, t_left, rtol, atol, rs, lda, t_done);
      if (rc == 0 || attempt + 1 >= o.max_retries) break;
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
      if (tid == 0) {
        const double Tn = s.y[S] * o.Tref;
        a.T[r] = Tn;
        a.P[r] = kRuD * Tn / (v * mw2);
      }
    }
    if (tid == 0) {
      a.v[r] = v;
      if (a.stats) a.stats[r] = rs;
    }
    __syncthreads();
  }
}

}  // namespace

size_t dense_smem_bytes(const DevMech &m, bool fp32, int *lda_out, int spill) {
  const int n = m.nsp + 1;
  const int lda = (n % 2 == 1) ? n : n + 1;  // odd row stride: conflict-free column walks
  if (lda_out) *lda_out = lda;
  size_t d = 72 + 3 * (size_t)m.nsp + 12 * (size_t)n + ((n + 1) / 2 + 1);
  if (fp32) d += (kMaxl + 3) * (size_t)n;
  if (!(spill & 1)) d += m.nstep;
  if (!(spill & 2)) d += (kMaxOrder + 3) * (size_t)n;
  size_t bytes = d * sizeof(double) + (size_t)n * lda * (fp32 ? sizeof(float) : sizeof(double));
  return ((bytes + 15) / 16) * 16;
}

size_t dense_spill_doubles(const DevMech &m) {
  return (size_t)m.nstep + (kMaxOrder + 3) * (size_t)(m.nsp + 1);
}

cudaError_t launch_integrate_dense(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                   int threads, int ctas, int spill, cudaStream_t stream) {
  int lda = 0;
  const size_t smem = dense_smem_bytes(m, o.lu_fp32 != 0, &lda, spill);
  cudaError_t e;
  if (o.lu_fp32) {
    e = cudaFuncSetAttribute(integrate_dense_kernel<float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    integrate_dense_kernel<float><<<ctas, threads, smem, stream>>>(m, o, a, lda, spill);
  } else {
    e = cudaFuncSetAttribute(integrate_dense_kernel<double>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    integrate_dense_kernel<double><<<ctas, threads, smem, stream>>>(m, o, a, lda, spill);
  }
  return cudaGetLastError();
}

}  // namespace zrk
