/*
 * zrk_bdf.c -- CPU ORACLE integrator (see zrk_oracle_bdf.h).  Test
 * infrastructure only.
 *
 * Quasi-constant step-size BDF, orders 1-5 (Shampine & Reichelt 1997):
 * backward differences D[0..q+2] carried between steps, step-size change by
 * D <- (R(factor) U)^T D, predictor sum(D[0..q]), corrector by modified
 * Newton on  y - c f(y) - psi = 0 with c = h/alpha_q, local error
 * error_const[q] * d, order choice among q-1, q, q+1 after q+1 equal steps.
 * Newton matrices are reused while c stays within 30 % of the factored value
 * (the correction is then scaled by 2/(1+c/c_lu)); a fresh Jacobian is taken
 * after a failed Newton iteration, as CVODE does.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "zrk_oracle_bdf.h"

#define MAXO 5
#define NEWTON_MAXITER 3
#define MIN_FACTOR 0.2
#define MAX_FACTOR 10.0
#define ETA_KEEP 1.5
/* CVODE's default per-step failure limits (the plugin sets neither
 * CVodeSetMaxErrTestFails nor CVodeSetMaxConvFails): the 7th error-test
 * failure or the 10th convergence failure within one step fails the attempt */
#define MAX_NEF 7
#define MAX_NCF 10
#define MXNEF1 3       /* error-test failures before the order/step cut below */
#define ETA_MIN_EF 0.1 /* step factor of that cut */

static const double KAPPA[MAXO + 1] = {0.0, -0.1850, -1.0 / 9.0, -0.0823, -0.0415, 0.0};

void zo_bdf_default_opts(zo_bdf_opts *o) {
  /* cfd_plugin defaults, zerork_reactor_manager.cpp:49-101 */
  o->rtol = 1.0e-8;
  o->atol = 1.0e-20;
  o->max_dt = 0.05;
  o->nlscoef = 0.05;
  o->max_steps = 5000;
  o->Tref = 1.0;
  o->min_mass_frac = 1.0e-30;
  o->step_limiter = 1.0e22;
  o->analytic = 1;
  o->max_retries = 5;
  o->retry_atol = 0.1;
  o->retry_rtol = 1.0;
  o->dT_ign = 0.0;
  o->constant_volume = 1;
  o->stop_ign = 0;
  o->abstol_dens = 0;
  o->fail_caps = 1;
}

typedef struct {
  int n, nnz;
  zo_reactor *r;
  const zo_jac_pattern *p;
  const zo_bdf_opts *o;
  double gam[MAXO + 2], alp[MAXO + 2], econ[MAXO + 2];
  double *D;       /* (MAXO+3) x n */
  double *jac;     /* nnz sparse values */
  double *A;       /* n x n dense Newton matrix, LU in place */
  double *Jd;      /* n x n dense divided-difference Jacobian (analytic = 0) */
  /* energy source: the right-hand side takes T from the energy, T* =
   * T(E0 + e_src t, Y), so it depends on Y through T* as well; the Newton
   * matrix adds that coupling as the rank-one term g d^T with g = df/dT*
   * and d_j = dT* by dY_j = -e_j / c_x (r1 = 1 when set) */
  double *r1g, *r1d;
  int r1;
  int *piv;
  double *y, *f, *f0, *ypred, *psi, *d, *dy, *scale, *rhs, *err, *tmp;
  double c_lu, crate;
  int jac_current;
  zo_bdf_stats st;
  /* ignition time: target temperature (<= 0: off), the attempt's start time
   * within the call, the temperature at the last accepted step */
  double T_target, t_off, T_prev;
  double *t_ign;
  double v0; /* initial inverse density (abstol_dens) */
} bdf_t;

/* absolute tolerance of component i (abstol_dens: reactor_nvector_serial.cpp:
 * 107-119, correction 1 / (rho * (1 / W_k) * 1e-3)) */
static double atol_of(const bdf_t *b, double atol, int i) {
  if (!b->o->abstol_dens || i >= b->n - 1) return atol;
  return atol * (1.0 / ((1.0 / b->v0) * (1.0 / b->r->t->mw[i]) * 1.0e-3));
}

static double rms(const double *x, const double *s, int n) {
  double a = 0.0;
  for (int i = 0; i < n; ++i) {
    double v = x[i] / s[i];
    a += v * v;
  }
  return sqrt(a / n);
}

/* f = ydot(t, y), t local to the attempt (the reactor's sources see the
 * time from the start of the call) */
static int rhs(bdf_t *b, double t, const double *y, double *f) {
  b->st.nrhs++;
  b->r->time = b->t_off + t;
  if (zo_reactor_rhs(b->r, y, f)) return 1;
  for (int i = 0; i < b->n; ++i)
    if (!isfinite(f[i])) return 1;
  return 0;
}

/* Jacobian at y with f = f(y), then Newton matrix A = I - c J, LU. */
static int take_jacobian(bdf_t *b, double t, const double *y, const double *f) {
  b->st.njac++;
  b->r->time = b->t_off + t;
  if (!b->o->analytic) {
    /* forward differences, increment sqrt(uround) * max(|y_j|, 1/w_j) */
    const int n = b->n;
    double *yp = b->tmp + n, *fp = b->tmp + 2 * n;
    memcpy(yp, y, sizeof(double) * n);
    for (int j = 0; j < n; ++j) {
      double inc = sqrt(2.220446049250313e-16) * fmax(fabs(y[j]), b->o->atol + b->o->rtol * fabs(y[j]) + 1e-10);
      yp[j] = y[j] + inc;
      inc = yp[j] - y[j];
      if (rhs(b, t, yp, fp)) return 1;
      for (int i = 0; i < n; ++i) b->Jd[i * n + j] = (fp[i] - f[i]) / inc;
      yp[j] = y[j];
    }
    b->jac_current = 1;
    return 0;
  }
  if (zo_jac_values(b->r, b->p, y, f, b->jac, NULL)) return 1;
  for (int i = 0; i < b->nnz; ++i)
    if (!isfinite(b->jac[i])) return 1;
  b->r1 = 0;
  if (b->r->e_src != 0.0) {
    const int n = b->n, ns = n - 1;
    double *f1 = b->tmp + n, *f2 = b->tmp + 2 * n;
    if (rhs(b, t, y, f1)) return 1;
    const double Ts = b->r->T_used, cx = b->r->mean_cv;
    for (int j = 0; j < ns; ++j)
      b->r1d[j] = -(b->r->u_RT[j] * (ZO_RU / b->r->t->mw[j] * Ts)) / cx;
    b->r1d[ns] = 0.0;
    const double Tp = Ts + Ts * sqrt(2.220446049250313e-16);
    b->r->T_force = Tp;
    const int bad = rhs(b, t, y, f2);
    b->r->T_force = 0.0;
    if (bad) return 1;
    for (int i = 0; i < n; ++i) b->r1g[i] = (f2[i] - f1[i]) / (Tp - Ts);
    b->r1 = 1;
  }
  b->jac_current = 1;
  return 0;
}

static int factor(bdf_t *b, double c) {
  const int n = b->n;
  b->st.nlu++;
  double *A = b->A;
  memset(A, 0, sizeof(double) * n * n);
  if (!b->o->analytic) {
    for (int i = 0; i < n * n; ++i) A[i] = -c * b->Jd[i];
  } else {
    for (int j = 0; j < n; ++j)
      for (int k = b->p->col_ptr[j]; k < b->p->col_ptr[j + 1]; ++k)
        A[b->p->row_idx[k] * n + j] = -c * b->jac[k];
  }
  if (b->o->analytic && b->r1)
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) A[i * n + j] -= c * b->r1g[i] * b->r1d[j];
  for (int i = 0; i < n; ++i) A[i * n + i] += 1.0;
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double mx = fabs(A[k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (fabs(A[i * n + k]) > mx) { mx = fabs(A[i * n + k]); pr = i; }
    b->piv[k] = pr;
    if (mx == 0.0) return 1;
    if (pr != k)
      for (int j = 0; j < n; ++j) { double t = A[k * n + j]; A[k * n + j] = A[pr * n + j]; A[pr * n + j] = t; }
    const double inv = 1.0 / A[k * n + k];
    for (int i = k + 1; i < n; ++i) {
      double l = A[i * n + k] * inv;
      A[i * n + k] = l;
      if (l != 0.0)
        for (int j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
    }
  }
  b->c_lu = c;
  b->crate = 1.0;
  return 0;
}

static void lu_solve(bdf_t *b, double *x) {
  const int n = b->n;
  const double *A = b->A;
  for (int k = 0; k < n; ++k) {
    int pr = b->piv[k];
    if (pr != k) { double t = x[k]; x[k] = x[pr]; x[pr] = t; }
  }
  for (int i = 1; i < n; ++i) {
    double s = x[i];
    for (int j = 0; j < i; ++j) s -= A[i * n + j] * x[j];
    x[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * x[j];
    x[i] = s / A[i * n + i];
  }
}

/* R(order, factor): M[i][j] = (i - 1 - factor*j)/i (i,j >= 1), M[0][*] = 1,
 * R = column-wise cumulative product over rows. */
static void compute_R(int order, double fac, double R[MAXO + 1][MAXO + 1]) {
  double M[MAXO + 1][MAXO + 1];
  for (int i = 0; i <= order; ++i)
    for (int j = 0; j <= order; ++j) M[i][j] = (i == 0) ? 1.0 : (j == 0 ? 0.0 : (i - 1 - fac * j) / i);
  for (int j = 0; j <= order; ++j) {
    R[0][j] = M[0][j];
    for (int i = 1; i <= order; ++i) R[i][j] = R[i - 1][j] * M[i][j];
  }
}

static void change_D(bdf_t *b, int order, double fac) {
  double R[MAXO + 1][MAXO + 1], U[MAXO + 1][MAXO + 1], RU[MAXO + 1][MAXO + 1];
  compute_R(order, fac, R);
  compute_R(order, 1.0, U);
  for (int i = 0; i <= order; ++i)
    for (int j = 0; j <= order; ++j) {
      double s = 0.0;
      for (int k = 0; k <= order; ++k) s += R[i][k] * U[k][j];
      RU[i][j] = s;
    }
  const int n = b->n;
  double *Dn = b->tmp;  /* (MAXO+1)*n scratch */
  for (int i = 0; i <= order; ++i)
    for (int m = 0; m < n; ++m) {
      double s = 0.0;
      for (int k = 0; k <= order; ++k) s += RU[k][i] * b->D[k * n + m];
      Dn[i * n + m] = s;
    }
  memcpy(b->D, Dn, sizeof(double) * (order + 1) * n);
}

/* One attempt (one CVodeReInit..failure span): integrates y0 over
 * [0, t_end].  On failure y0 receives the last accepted state and *t_done
 * the time it was reached (D[0], which step-size changes leave unchanged). */
static int integrate(bdf_t *b, double *y0, double t_end, double rtol, double atol, double *t_done) {
  const int n = b->n;
  const zo_bdf_opts *o = b->o;
  double t = 0.0;
  int rc = 0, nsteps_att = 0;
  *t_done = 0.0;
  b->T_prev = y0[n - 1] * o->Tref;
  memcpy(b->y, y0, sizeof(double) * n);
  if (rhs(b, 0.0, b->y, b->f0)) return -1;
  /* initial step: Hairer-Norsett-Wanner estimate (first order) */
  for (int i = 0; i < n; ++i) b->scale[i] = atol_of(b, atol, i) + fabs(b->y[i]) * rtol;
  double d0 = rms(b->y, b->scale, n), d1 = rms(b->f0, b->scale, n);
  double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
  if (h0 > t_end) h0 = t_end;
  for (int i = 0; i < n; ++i) b->tmp[i] = b->y[i] + h0 * b->f0[i];
  double d2 = 0.0;
  if (rhs(b, h0, b->tmp, b->f) == 0) {
    for (int i = 0; i < n; ++i) b->dy[i] = b->f[i] - b->f0[i];
    d2 = rms(b->dy, b->scale, n) / h0;
  }
  double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : sqrt(0.01 / fmax(d1, d2));
  double h = fmin(100.0 * h0, h1);
  h = fmin(h, o->max_dt);
  h = fmin(h, t_end);
  int q = 1, neq = 0;
  memset(b->D, 0, sizeof(double) * (MAXO + 3) * n);
  memcpy(b->D, b->y, sizeof(double) * n);
  for (int i = 0; i < n; ++i) b->D[n + i] = b->f0[i] * h;
  if (take_jacobian(b, 0.0, b->y, b->f0)) { rc = -2; goto failed; }
  if (factor(b, h / b->alp[q])) { rc = -3; goto failed; }
  while (t < t_end) {
    if (nsteps_att >= o->max_steps) { rc = -4; goto failed; }
    int accepted = 0;
    double safety = 0.9, err_norm = 0.0;
    int nef = 0, ncf = 0; /* this step's error-test and convergence failures */
    while (!accepted) {
      if (h > o->max_dt) { change_D(b, q, o->max_dt / h); h = o->max_dt; }
      if (t + h > t_end) {
        double fac = (t_end - t) / h;
        change_D(b, q, fac);
        h = t_end - t;
      }
      if (!(t + h > t)) { rc = -5; goto failed; } /* no progress (or h not finite) */
      const double t_new = t + h;
      for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int k = 0; k <= q; ++k) s += b->D[k * n + i];
        b->ypred[i] = s;
        double ps = 0.0;
        for (int k = 1; k <= q; ++k) ps += b->gam[k] * b->D[k * n + i];
        b->psi[i] = ps / b->alp[q];
        b->scale[i] = atol_of(b, atol, i) + rtol * fabs(s);
      }
      const double c = h / b->alp[q];
      if (fabs(c / b->c_lu - 1.0) > 0.3)
        if (factor(b, c)) { rc = -3; goto failed; }
      /* modified Newton, CVODE-style convergence test (Hindmarsh et al.,
       * ACM TOMS 31 (2005) 363-396, sec. 2.1): rate estimate carried across
       * steps, converged when econ * |delta| * min(1, rate) <= nlscoef,
       * at most NEWTON_MAXITER iterations, divergence when |delta| doubles. */
      memcpy(b->y, b->ypred, sizeof(double) * n);
      memset(b->d, 0, sizeof(double) * n);
      int conv = 0, it;
      double dnorm_old = -1.0;
      const double gscale = (c == b->c_lu) ? 1.0 : 2.0 / (1.0 + c / b->c_lu);
      for (it = 0; it < NEWTON_MAXITER; ++it) {
        if (rhs(b, t_new, b->y, b->f)) break;
        if (it == 0) memcpy(b->f0, b->f, sizeof(double) * n);
        b->st.nnewt++;
        for (int i = 0; i < n; ++i) b->dy[i] = c * b->f[i] - b->psi[i] - b->d[i];
        lu_solve(b, b->dy);
        for (int i = 0; i < n; ++i) b->dy[i] *= gscale;
        const double dn = rms(b->dy, b->scale, n);
        for (int i = 0; i < n; ++i) { b->y[i] += b->dy[i]; b->d[i] += b->dy[i]; }
        if (dnorm_old > 0.0) b->crate = fmax(0.3 * b->crate, dn / dnorm_old);
        if (b->econ[q] * dn * fmin(1.0, b->crate) <= o->nlscoef) { conv = 1; ++it; break; }
        if (dnorm_old > 0.0 && dn > 2.0 * dnorm_old) break;
        dnorm_old = dn;
      }
      if (!conv) {
        if (!b->jac_current) {
          if (rhs(b, t_new, b->ypred, b->f0)) { rc = -6; goto failed; }
          if (take_jacobian(b, t_new, b->ypred, b->f0)) { rc = -2; goto failed; }
          if (factor(b, c)) { rc = -3; goto failed; }
          continue;
        }
        if (++ncf >= MAX_NCF && o->fail_caps) { rc = -8; goto failed; }
        change_D(b, q, 0.5);
        h *= 0.5;
        b->st.nrej++;
        continue;
      }
      safety = 0.9 * (2 * NEWTON_MAXITER + 1) / (2.0 * NEWTON_MAXITER + it);
      for (int i = 0; i < n; ++i) b->err[i] = b->econ[q] * b->d[i];
      err_norm = rms(b->err, b->scale, n);
      if (!isfinite(err_norm)) { rc = -7; goto failed; }
      if (err_norm > 1.0) {
        if (++nef >= MAX_NEF && o->fail_caps) { rc = -9; goto failed; }
        b->st.nrej++;
        if (nef > MXNEF1 && o->fail_caps) {
          /* repeated failures (CVODE's rule, user guide sec. 2.1): order one
           * lower and a tenth of the step; at order 1 the first difference
           * is reloaded from f at the last accepted state */
          if (q > 1) {
            --q;
            change_D(b, q, ETA_MIN_EF);
          } else {
            if (rhs(b, t, b->D, b->tmp)) { rc = -6; goto failed; }
            for (int i = 0; i < n; ++i) b->D[n + i] = b->tmp[i] * (h * ETA_MIN_EF);
          }
          h *= ETA_MIN_EF;
          neq = 0;
          continue;
        }
        double fac = fmax(MIN_FACTOR, safety * pow(err_norm, -1.0 / (q + 1)));
        change_D(b, q, fac);
        h *= fac;
        continue;
      }
      accepted = 1;
      t = t_new;
    }
    b->st.nsteps++;
    nsteps_att++;
    neq++;
    b->jac_current = 0;
    /* update differences (stop_after_ignition keeps the previous state) */
    const int keep_prev = b->t_ign && b->T_target > 0.0 && o->stop_ign && *b->t_ign < 0.0;
    if (keep_prev) memcpy(b->tmp, b->D, sizeof(double) * n);
    for (int i = 0; i < n; ++i) {
      b->D[(q + 2) * n + i] = b->d[i] - b->D[(q + 1) * n + i];
      b->D[(q + 1) * n + i] = b->d[i];
    }
    for (int k = q; k >= 0; --k)
      for (int i = 0; i < n; ++i) b->D[k * n + i] += b->D[(k + 1) * n + i];
    if (b->t_ign && b->T_target > 0.0) { /* first crossing of T0 + dT_ign */
      const double Tn = b->D[n - 1] * o->Tref;
      if (*b->t_ign < 0.0 && Tn >= b->T_target) {
        const double frac = (Tn > b->T_prev) ? (b->T_target - b->T_prev) / (Tn - b->T_prev) : 1.0;
        *b->t_ign = b->t_off + (t - h) + frac * h;
        if (o->stop_ign) { /* solver_cvode.cpp:259-263: the call ends at the crossing */
          for (int i = 0; i < n; ++i) y0[i] = b->tmp[i] + frac * (b->D[i] - b->tmp[i]);
          *t_done = (t - h) + frac * h;
          return 0;
        }
      }
      b->T_prev = Tn;
    }
    if (neq < q + 1) continue;
    double em = INFINITY, ep = INFINITY;
    if (q > 1) {
      for (int i = 0; i < n; ++i) b->err[i] = b->econ[q - 1] * b->D[q * n + i];
      em = rms(b->err, b->scale, n);
    }
    if (q < MAXO) {
      for (int i = 0; i < n; ++i) b->err[i] = b->econ[q + 1] * b->D[(q + 2) * n + i];
      ep = rms(b->err, b->scale, n);
    }
    double fm = (q > 1) ? pow(em, -1.0 / q) : 0.0;
    double f0 = pow(err_norm, -1.0 / (q + 1));
    double fp = (q < MAXO) ? pow(ep, -1.0 / (q + 2)) : 0.0;
    int dq = 0;
    double best = f0;
    if (fm > best) { best = fm; dq = -1; }
    if (fp > best) { best = fp; dq = 1; }
    q += dq;
    double fac = fmin(MAX_FACTOR, safety * best);
    /* CVODE's step-size hysteresis (eta < 1.5 keeps h): fewer matrix updates */
    if (fac < ETA_KEEP) fac = 1.0;
    change_D(b, q, fac);
    h *= fac;
    neq = 0;
  }
  memcpy(y0, b->D, sizeof(double) * n); /* D[0] holds y at t_end */
  *t_done = t;
  return 0;
failed:
  memcpy(y0, b->D, sizeof(double) * n);
  *t_done = t;
  return rc;
}

int zo_reactor_solve(const zo_tables *t, const zo_jac_pattern *p, const zo_kinetics *kin,
                     const zo_bdf_opts *o, double dt, double *T, double *P, double *Y,
                     const double *y_src, double dpdt, double e_src, int fix_T, double *t_ign,
                     zo_bdf_stats *st) {
  bdf_t b;
  memset(&b, 0, sizeof(b));
  const int ns = t->nsp, n = ns + 1;
  b.n = n;
  b.nnz = p->nnz;
  b.p = p;
  b.o = o;
  b.r = zo_reactor_new(t, kin, o->Tref, o->min_mass_frac, o->step_limiter);
  for (int k = 0; k <= MAXO + 1; ++k) {
    double g = 0.0;
    for (int i = 1; i <= k; ++i) g += 1.0 / i;
    b.gam[k] = g;
    double kap = (k <= MAXO) ? KAPPA[k] : 0.0;
    b.alp[k] = (1.0 - kap) * g;
    b.econ[k] = kap * g + 1.0 / (k + 1);
  }
  b.D = (double *)calloc((size_t)(MAXO + 3) * n, sizeof(double));
  b.jac = (double *)calloc(p->nnz, sizeof(double));
  b.A = (double *)calloc((size_t)n * n, sizeof(double));
  b.Jd = (double *)calloc((size_t)n * n, sizeof(double));
  b.piv = (int *)calloc(n, sizeof(int));
  double *w = (double *)calloc((size_t)n * 12 + (size_t)(MAXO + 1) * n, sizeof(double));
  b.y = w; b.f = w + n; b.f0 = w + 2 * n; b.ypred = w + 3 * n; b.psi = w + 4 * n;
  b.d = w + 5 * n; b.dy = w + 6 * n; b.scale = w + 7 * n; b.rhs = w + 8 * n; b.err = w + 9 * n;
  b.tmp = w + 10 * n;
  b.r1g = (double *)calloc((size_t)2 * n, sizeof(double));
  b.r1d = b.r1g + n;
  double *y = (double *)calloc(n, sizeof(double));
  b.r->cp = o->constant_volume == 0;
  b.r->fix_T = fix_T;
  zo_reactor_init_state(b.r, *T, *P, Y, dpdt, e_src, y_src);
  b.v0 = b.r->inv_density;
  b.t_ign = t_ign;
  if (t_ign) *t_ign = -1.0;
  b.T_target = o->dT_ign > 0.0 ? *T + o->dT_ign : -1.0;
  for (int j = 0; j < ns; ++j) y[j] = Y[j];
  y[ns] = *T / o->Tref;
  /* retry loop, solver_cvode.cpp:227-246: a failed attempt restarts the
   * method (order 1, new initial step) from the last accepted state with
   * adjusted tolerances; max_steps counts per attempt, as CVodeReInit
   * resets CVODE's step counter */
  double *ystart = (double *)calloc(n, sizeof(double));
  memcpy(ystart, y, sizeof(double) * n);
  double rtol = o->rtol, atol = o->atol, t_left = dt;
  int rc = 0;
  for (int attempt = 0;; ++attempt) {
    double t_done = 0.0;
    b.t_off = dt - t_left;
    rc = integrate(&b, y, t_left, rtol, atol, &t_done);
    if (rc == 0 || attempt + 1 >= o->max_retries) break;
    b.st.retries++;
    t_left -= t_done;
    atol *= o->retry_atol;
    rtol *= o->retry_rtol;
  }
  if (rc != 0) memcpy(y, ystart, sizeof(double) * n);
  free(ystart);
  b.st.status = rc;
  if (rc == 0) {
    for (int j = 0; j < ns; ++j) Y[j] = y[j];
    *T = zo_reactor_end_temperature(b.r, dt, Y, y[ns] * o->Tref);
    *P = zo_reactor_pressure(b.r, dt, *T, Y);
  }
  if (st) *st = b.st;
  free(y); free(w); free(b.r1g); free(b.piv); free(b.A); free(b.Jd); free(b.jac); free(b.D);
  zo_reactor_free(b.r);
  return rc;
}

int zo_reactor_solve_batch(const zo_tables *t, const zo_jac_pattern *p, const zo_bdf_opts *o,
                           int nthreads, int n, double dt, double *T, double *P, double *Y,
                           const double *y_src, const double *dpdt, const double *e_src,
                           const int *fix_T, double *t_ign, zo_bdf_stats *stats) {
  int nfail = 0;
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) reduction(+ : nfail)
  for (int r = 0; r < n; ++r) {
    zo_kinetics kin;
    zo_kinetics_oracle(t, &kin);
    zo_bdf_stats st;
    if (zo_reactor_solve(t, p, &kin, o, dt, &T[r], &P[r], &Y[(size_t)r * t->nsp],
                         y_src ? &y_src[(size_t)r * t->nsp] : NULL, dpdt ? dpdt[r] : 0.0,
                         e_src ? e_src[r] : 0.0, fix_T ? fix_T[r] : 0, t_ign ? &t_ign[r] : NULL,
                         &st))
      ++nfail;
    if (stats) stats[r] = st;
  }
  return nfail;
}
