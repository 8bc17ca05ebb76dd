/*
 * zrk_oracle.c -- CPU ORACLE (test infrastructure only; see zrk_oracle.h).
 *
 * Restates, operation for operation, the reference's CPU rate path so that it
 * agrees with the reference library built with ZERORK_EXP_LIBC to rounding.
 * Citations are to files of the Zero-RK checkout.
 */
#include "zrk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static void *zcalloc(size_t n, size_t sz) { return calloc(n > 0 ? n : 1, sz); }

zo_tables *zo_tables_alloc(const int s[14]) {
  zo_tables *t = (zo_tables *)zcalloc(1, sizeof(zo_tables));
  t->nsp = s[0]; t->nrxn = s[1]; t->nstep = s[2];
  t->tot_reac = s[3]; t->tot_prod = s[4];
  t->n_arr = s[5]; t->n_keq = s[6]; t->n_tb = s[7]; t->n_fo = s[8];
  t->n_tb_eff = s[9]; t->n_fo_eff = s[10];
  t->mw = (double *)zcalloc(t->nsp, sizeof(double));
  t->thermo = (double *)zcalloc((size_t)t->nsp * 16, sizeof(double));
  t->step_rxn = (int *)zcalloc(t->nstep, sizeof(int));
  t->step_dir = (int *)zcalloc(t->nstep, sizeof(int));
  t->reac_ptr = (int *)zcalloc(t->nstep + 1, sizeof(int));
  t->reac_spc = (int *)zcalloc(t->tot_reac, sizeof(int));
  t->prod_ptr = (int *)zcalloc(t->nstep + 1, sizeof(int));
  t->prod_spc = (int *)zcalloc(t->tot_prod, sizeof(int));
  t->arr_step = (int *)zcalloc(t->n_arr, sizeof(int));
  t->arr_lnA = (double *)zcalloc(t->n_arr, sizeof(double));
  t->arr_n = (double *)zcalloc(t->n_arr, sizeof(double));
  t->arr_Ta = (double *)zcalloc(t->n_arr, sizeof(double));
  t->keq_step = (int *)zcalloc(t->n_keq, sizeof(int));
  t->keq_fwd = (int *)zcalloc(t->n_keq, sizeof(int));
  t->keq_dn = (double *)zcalloc(t->n_keq, sizeof(double));
  t->tb_fwd = (int *)zcalloc(t->n_tb, sizeof(int));
  t->tb_rev = (int *)zcalloc(t->n_tb, sizeof(int));
  t->tb_ptr = (int *)zcalloc(t->n_tb + 1, sizeof(int));
  t->tb_spc = (int *)zcalloc(t->n_tb_eff, sizeof(int));
  t->tb_alpha = (double *)zcalloc(t->n_tb_eff, sizeof(double));
  t->fo_fwd = (int *)zcalloc(t->n_fo, sizeof(int));
  t->fo_rev = (int *)zcalloc(t->n_fo, sizeof(int));
  t->fo_type = (int *)zcalloc(t->n_fo, sizeof(int));
  t->fo_spc = (int *)zcalloc(t->n_fo, sizeof(int));
  t->fo_ptr = (int *)zcalloc(t->n_fo + 1, sizeof(int));
  t->fo_eff_spc = (int *)zcalloc(t->n_fo_eff, sizeof(int));
  t->fo_alpha = (double *)zcalloc(t->n_fo_eff, sizeof(double));
  t->fo_par = (double *)zcalloc((size_t)t->n_fo * 8, sizeof(double));
  t->n_plog = s[11]; t->n_plog_pt = s[12]; t->n_plog_ln = s[13];
  t->plog_step = (int *)zcalloc(t->n_plog, sizeof(int));
  t->plog_pt_ptr = (int *)zcalloc(t->n_plog + 1, sizeof(int));
  t->plog_ln_ptr = (int *)zcalloc(t->n_plog_pt + 1, sizeof(int));
  t->plog_p = (double *)zcalloc(t->n_plog_pt, sizeof(double));
  t->plog_lnp = (double *)zcalloc(t->n_plog_pt, sizeof(double));
  t->plog_lnA = (double *)zcalloc(t->n_plog_ln, sizeof(double));
  t->plog_sgn = (double *)zcalloc(t->n_plog_ln, sizeof(double));
  t->plog_n = (double *)zcalloc(t->n_plog_ln, sizeof(double));
  t->plog_Ta = (double *)zcalloc(t->n_plog_ln, sizeof(double));
  return t;
}

void zo_tables_free(zo_tables *t) {
  if (!t) return;
  free(t->mw); free(t->thermo); free(t->step_rxn); free(t->step_dir);
  free(t->reac_ptr); free(t->reac_spc); free(t->prod_ptr); free(t->prod_spc);
  free(t->arr_step); free(t->arr_lnA); free(t->arr_n); free(t->arr_Ta);
  free(t->keq_step); free(t->keq_fwd); free(t->keq_dn);
  free(t->tb_fwd); free(t->tb_rev); free(t->tb_ptr); free(t->tb_spc); free(t->tb_alpha);
  free(t->fo_fwd); free(t->fo_rev); free(t->fo_type); free(t->fo_spc); free(t->fo_ptr);
  free(t->fo_eff_spc); free(t->fo_alpha); free(t->fo_par);
  free(t->plog_step); free(t->plog_pt_ptr); free(t->plog_ln_ptr); free(t->plog_p);
  free(t->plog_lnp); free(t->plog_lnA); free(t->plog_sgn); free(t->plog_n); free(t->plog_Ta);
  free(t);
}

/* ------------------------------------------------------------------ thermo */
/* nasa_poly.cpp:50-76 getCp_R */
void zo_cp_R(const zo_tables *t, double T, double *cp_R) {
  for (int j = 0; j < t->nsp; ++j) {
    const double *c = t->thermo + 16 * j;
    if (T < c[0])
      cp_R[j] = c[1] + T * (c[2] + T * (c[3] + T * (c[4] + T * c[5])));
    else
      cp_R[j] = c[8] + T * (c[9] + T * (c[10] + T * (c[11] + T * c[12])));
  }
}

/* nasa_poly.cpp:78-117 getH_RT */
void zo_h_RT(const zo_tables *t, double T, double *h_RT) {
  double invT = 1.0 / T, m[4];
  m[0] = T; m[1] = T * m[0]; m[2] = T * m[1]; m[3] = T * m[2];
  m[0] *= 0.50000000000000000000;
  m[1] *= 0.33333333333333333333;
  m[2] *= 0.25000000000000000000;
  m[3] *= 0.20000000000000000000;
  for (int j = 0; j < t->nsp; ++j) {
    const double *c = t->thermo + 16 * j;
    if (T < c[0])
      h_RT[j] = c[1] + c[2] * m[0] + c[3] * m[1] + c[4] * m[2] + c[5] * m[3] + c[6] * invT;
    else
      h_RT[j] = c[8] + c[9] * m[0] + c[10] * m[1] + c[11] * m[2] + c[12] * m[3] + c[13] * invT;
  }
}

/* nasa_poly.cpp:118-172 getG_RT */
void zo_g_RT(const zo_tables *t, double T, double *g_RT) {
  double invT = 1.0 / T, m[5];
  m[0] = 1.0 - log(T);
  m[1] = T; m[2] = T * m[1]; m[3] = T * m[2]; m[4] = T * m[3];
  m[1] *= -0.50000000000000000000;
  m[2] *= -0.16666666666666666667;
  m[3] *= -0.08333333333333333333;
  m[4] *= -0.05000000000000000000;
  for (int j = 0; j < t->nsp; ++j) {
    const double *c = t->thermo + 16 * j;
    if (T < c[0])
      g_RT[j] = c[1] * m[0] + c[2] * m[1] + c[3] * m[2] + c[4] * m[3] + c[5] * m[4] +
                c[6] * invT - c[7];
    else
      g_RT[j] = c[8] * m[0] + c[9] * m[1] + c[10] * m[2] + c[11] * m[3] + c[12] * m[4] +
                c[13] * invT - c[14];
  }
}

/* ------------------------------------------------------- rate coefficients */
/* A PLOG reaction at (T, P): plog_reaction.cpp:166-185 (the Arrhenius lines
 * of one pressure, summed with the sign of A) and :187-300 (no
 * extrapolation: the end pressures' values outside [p_min, p_max];
 * logarithmic interpolation inside; zero for T or P <= 0 or a non-positive
 * bracketing value). */
static double plog_at(const zo_tables *t, int q, double invT, double logT) {
  double k = 0.0;
  for (int l = t->plog_ln_ptr[q]; l < t->plog_ln_ptr[q + 1]; ++l)
    k += t->plog_sgn[l] * exp(t->plog_lnA[l] + logT * t->plog_n[l] - invT * t->plog_Ta[l]);
  return k;
}

double zo_plog_k(const zo_tables *t, int j, double T, double invT, double logT, double P) {
  const int q0 = t->plog_pt_ptr[j], q1 = t->plog_pt_ptr[j + 1];
  if (T <= 0.0 || P <= 0.0) return 0.0;
  if (q1 - q0 == 1) return plog_at(t, q0, invT, logT);
  if (P <= t->plog_p[q0]) return plog_at(t, q0, invT, logT);
  if (P >= t->plog_p[q1 - 1]) return plog_at(t, q1 - 1, invT, logT);
  int r = q0;
  while (r + 1 < q1 - 1 && !(t->plog_p[r] <= P && P < t->plog_p[r + 1])) ++r;
  const double k1 = plog_at(t, r, invT, logT);
  if (k1 <= 0.0) return 0.0;
  const double k2 = plog_at(t, r + 1, invT, logT);
  if (k2 <= 0.0) return 0.0;
  const double e = log(k2 / k1) / (t->plog_lnp[r + 1] - t->plog_lnp[r]);
  return k1 * pow(P / t->plog_p[r], e);
}

/* rate_const.cpp:539-582 updateK, with updateArrheniusStep (:669-687),
 * updateFromKeqStep (:690-731), updateThirdBodyRxn (:862-888) and
 * updateFalloffRxn (:890-1012).  Exponentials use libc exp (the
 * ZERORK_EXP_LIBC build, fast_exps.cpp). */
void zo_rate_coefs(const zo_tables *t, double T, const double *C, double *K) {
  const int nsp = t->nsp;
  for (int j = 0; j < t->nstep; ++j) K[j] = 0.0;
  const double logT = log(T);
  const double invT = 1.0 / T;
  const double log_PatmInvRuT = log(ZO_PATM / (ZO_RU * T));
  double Csum = 0.0;
  for (int j = 0; j < nsp; ++j) Csum += C[j];

  for (int j = 0; j < t->n_arr; ++j) {
    double a = t->arr_lnA[j] + t->arr_n[j] * logT - t->arr_Ta[j] * invT;
    K[t->arr_step[j]] = exp(a);
  }
  /* PLOG steps before the reverse rates (rate_const.cpp:565-567), at the
   * pressure of the concentrations, Csum Ru T */
  for (int j = 0; j < t->n_plog; ++j)
    K[t->plog_step[j]] = zo_plog_k(t, j, T, invT, logT, Csum * ZO_RU * T);
  if (t->n_keq > 0) {
    double *g = (double *)malloc(sizeof(double) * nsp);
    zo_g_RT(t, T, g);
    for (int j = 0; j < t->n_keq; ++j) {
      const int f = t->keq_fwd[j];
      double s = 0.0;
      for (int k = t->prod_ptr[f]; k < t->prod_ptr[f + 1]; ++k) s += g[t->prod_spc[k]];
      for (int k = t->reac_ptr[f]; k < t->reac_ptr[f + 1]; ++k) s -= g[t->reac_spc[k]];
      double keq = exp(s - t->keq_dn[j] * log_PatmInvRuT);
      K[t->keq_step[j]] = keq * K[f];
    }
    free(g);
  }
  for (int j = 0; j < t->n_tb; ++j) {
    double Cmult = Csum;
    for (int k = t->tb_ptr[j]; k < t->tb_ptr[j + 1]; ++k) Cmult += C[t->tb_spc[k]] * t->tb_alpha[k];
    K[t->tb_fwd[j]] *= Cmult;
    if (t->tb_rev[j] >= 0) K[t->tb_rev[j]] *= Cmult;
  }
  for (int j = 0; j < t->n_fo; ++j) {
    const double *p = t->fo_par + 8 * j;
    double Klow = exp(p[0] + p[1] * logT - p[2] * invT);
    double Cmult;
    if (t->fo_spc[j] >= 0) {
      Cmult = C[t->fo_spc[j]];
    } else {
      Cmult = Csum;
      for (int k = t->fo_ptr[j]; k < t->fo_ptr[j + 1]; ++k)
        Cmult += C[t->fo_eff_spc[k]] * t->fo_alpha[k];
    }
    double Pr = Klow * Cmult / K[t->fo_fwd[j]];
    if (Pr < 1.0e-300) Pr = 1.0e-300;
    double lPr = log10(Pr);
    double fTerm = 1.0;
    const int ty = t->fo_type[j];
    if (ty == ZO_FO_TROE3 || ty == ZO_FO_TROE4) {
      double Fc = 0.0;
      if (p[4] != 0) Fc += (1.0 - p[3]) * exp(-T / p[4]);
      if (p[5] != 0) Fc += p[3] * exp(-T / p[5]);
      if (ty == ZO_FO_TROE4) Fc += exp(-p[6] * invT);
      if (Fc < 1.0e-300) Fc = 1.0e-300;
      fTerm = log10(Fc);
      double nTerm = 0.75 - 1.27 * fTerm;
      lPr -= (0.4 + 0.67 * fTerm);
      lPr = lPr / (nTerm - 0.14 * lPr);
      lPr *= lPr;
      fTerm /= (1.0 + lPr);
      fTerm = pow(10.0, fTerm);
    } else if (ty == ZO_FO_SRI) {
      const double x_power = 1.0 / (1.0 + lPr * lPr);
      fTerm = p[3] * exp(-p[4] * invT);
      if (p[5] > 0) fTerm += exp(-T * p[5]);
      fTerm = pow(fTerm, x_power);
      fTerm *= p[6];
      fTerm *= pow(T, p[7]);
    }
    double Pcorr = fTerm * Pr / (1.0 + Pr);
    K[t->fo_fwd[j]] *= Pcorr;
    if (t->fo_rev[j] >= 0) K[t->fo_rev[j]] *= Pcorr;
  }
}

/* perf_net.cpp:190-274 calcRatesFromTC_StepLimiter (lim != NULL) and
 * perf_net.cpp:126-188 calcRatesFromTC (lim == NULL). */
void zo_rates(const zo_tables *t, double T, const double *C, const double *lim,
              double *net, double *cre, double *des, double *rop) {
  zo_rate_coefs(t, T, C, rop);
  if (lim) {
    for (int j = 0; j < t->nstep; ++j)
      if (0.0 < lim[j] && lim[j] < 1.0e+300) rop[j] *= lim[j] / (lim[j] + rop[j]);
  }
  for (int j = 0; j < t->nstep; ++j)
    for (int k = t->reac_ptr[j]; k < t->reac_ptr[j + 1]; ++k) rop[j] *= C[t->reac_spc[k]];
  memset(cre, 0, sizeof(double) * t->nsp);
  memset(des, 0, sizeof(double) * t->nsp);
  for (int j = 0; j < t->nstep; ++j)
    for (int k = t->reac_ptr[j]; k < t->reac_ptr[j + 1]; ++k) des[t->reac_spc[k]] += rop[j];
  for (int j = 0; j < t->nstep; ++j)
    for (int k = t->prod_ptr[j]; k < t->prod_ptr[j + 1]; ++k) cre[t->prod_spc[k]] += rop[j];
  for (int j = 0; j < t->nsp; ++j) net[j] = cre[j] - des[j];
}

/* ------------------------------------------ oracle kinetics provider */
static void ok_rates(void *ctx, double T, const double *C, const double *lim, double *net,
                     double *cre, double *des, double *rop) {
  zo_rates((const zo_tables *)ctx, T, C, lim, net, cre, des, rop);
}
/* mechanism.cpp:374-379 getIntEnergy_RT */
static void ok_u_RT(void *ctx, double T, double *u) {
  const zo_tables *t = (const zo_tables *)ctx;
  zo_h_RT(t, T, u);
  for (int j = 0; j < t->nsp; ++j) u[j] -= 1.0;
}
/* mechanism.cpp:421-434 getMassCvFromTY */
static double ok_mass_cv(void *ctx, double T, const double *y, double *cv) {
  const zo_tables *t = (const zo_tables *)ctx;
  double mix = 0.0;
  zo_cp_R(t, T, cv);
  for (int j = 0; j < t->nsp; ++j) {
    cv[j] -= 1.0;
    cv[j] *= ZO_RU / t->mw[j];
    mix += cv[j] * y[j];
  }
  return mix;
}
/* mechanism.cpp:267-283 getMolWtMixFromY / getDensityFromTPY */
static double ok_density(void *ctx, double T, double P, const double *y) {
  const zo_tables *t = (const zo_tables *)ctx;
  double s = 0.0;
  for (int j = 0; j < t->nsp; ++j) s += y[j] * (1.0 / t->mw[j]);
  double mwmix = 1.0 / s;
  return P * mwmix / (ZO_RU * T);
}
/* mechanism.cpp:321-327 getCfromVY */
static void ok_c_from_vy(void *ctx, double v, const double *y, double *c) {
  const zo_tables *t = (const zo_tables *)ctx;
  double dens = 1.0 / v;
  for (int j = 0; j < t->nsp; ++j) c[j] = dens * (1.0 / t->mw[j]) * y[j];
}

/* mechanism.cpp:366-367 getEnthalpy_RT */
static void ok_h_RT(void *ctx, double T, double *h) { zo_h_RT((const zo_tables *)ctx, T, h); }
/* mechanism.cpp:408-420 getMassCpFromTY */
static double ok_mass_cp(void *ctx, double T, const double *y, double *cp) {
  const zo_tables *t = (const zo_tables *)ctx;
  double mix = 0.0;
  zo_cp_R(t, T, cp);
  for (int j = 0; j < t->nsp; ++j) {
    cp[j] *= ZO_RU / t->mw[j];
    mix += cp[j] * y[j];
  }
  return mix;
}
/* mechanism.cpp:355-367 getMassIntEnergyFromTY */
static double ok_mass_u(void *ctx, double T, const double *y) {
  const zo_tables *t = (const zo_tables *)ctx;
  double *u = (double *)zcalloc(t->nsp, sizeof(double)), mix = 0.0;
  zo_h_RT(t, T, u);
  for (int j = 0; j < t->nsp; ++j) {
    u[j] -= 1.0;
    u[j] *= ZO_RU / t->mw[j] * T;
    mix += u[j] * y[j];
  }
  free(u);
  return mix;
}
/* mechanism.cpp:336-347 getMassEnthalpyFromTY */
static double ok_mass_h(void *ctx, double T, const double *y) {
  const zo_tables *t = (const zo_tables *)ctx;
  double *h = (double *)zcalloc(t->nsp, sizeof(double)), mix = 0.0;
  zo_h_RT(t, T, h);
  for (int j = 0; j < t->nsp; ++j) {
    h[j] *= ZO_RU / t->mw[j] * T;
    mix += h[j] * y[j];
  }
  free(h);
  return mix;
}
/* mechanism.cpp:292-297 getPressureFromTVY */
static double ok_pressure(void *ctx, double T, double v, const double *y) {
  const zo_tables *t = (const zo_tables *)ctx;
  double s = 0.0;
  for (int j = 0; j < t->nsp; ++j) s += y[j] * (1.0 / t->mw[j]);
  double mwmix = 1.0 / s;
  return ZO_RU * T / (v * mwmix);
}
/* mechanism.cpp:477-547 getTemperatureFromEY / getTemperatureFromHY: Newton
 * on the mixture energy between 100 K and 5000 K (linear extrapolation
 * outside), steps clipped to +-100 K, stop below 1e-6 K or when the step no
 * longer changes T, at most 400 iterations.  Both iterations divide by the
 * mixture c_v, and so does the extrapolation above 5000 K; only the
 * enthalpy extrapolation below 100 K uses c_p. */
static double ok_temp_from(void *ctx, int enthalpy, double E, const double *y, double Tg) {
  const zo_tables *t = (const zo_tables *)ctx;
  const double Tmin = 100.0, Tmax = 5000.0;
  double *tmp = (double *)zcalloc(t->nsp, sizeof(double));
  double (*energy)(void *, double, const double *) = enthalpy ? ok_mass_h : ok_mass_u;
  const double Emin = energy(ctx, Tmin, y), Emax = energy(ctx, Tmax, y);
  double T;
  if (E < Emin) {
    const double c = enthalpy ? ok_mass_cp(ctx, Tmin, y, tmp) : ok_mass_cv(ctx, Tmin, y, tmp);
    T = Tmin - (Emin - E) / c;
  } else if (E > Emax) {
    T = Tmax - (Emax - E) / ok_mass_cv(ctx, Tmax, y, tmp);
  } else {
    T = Tg;
    if (T < Tmin || T > Tmax) T = Tmin + (Tmax - Tmin) / (Emax - Emin) * (E - Emin);
    for (int i = 0; i < 400; ++i) {
      const double Ei = energy(ctx, T, y);
      const double c = ok_mass_cv(ctx, T, y, tmp);
      const double dT = fmin(fmax((E - Ei) / c, -100.0), 100.0);
      if (fabs(dT) < 1.0e-6 || T + dT == T) break;
      T += dT;
    }
  }
  free(tmp);
  return T;
}
static double ok_temp_from_E(void *ctx, double E, const double *y, double Tg) {
  return ok_temp_from(ctx, 0, E, y, Tg);
}
static double ok_temp_from_H(void *ctx, double H, const double *y, double Tg) {
  return ok_temp_from(ctx, 1, H, y, Tg);
}

void zo_kinetics_oracle(const zo_tables *t, zo_kinetics *k) {
  k->ctx = (void *)t;
  k->rates_limiter = ok_rates;
  k->int_energy_RT = ok_u_RT;
  k->mass_cv = ok_mass_cv;
  k->density_TPY = ok_density;
  k->c_from_vy = ok_c_from_vy;
  k->enthalpy_RT = ok_h_RT;
  k->mass_cp = ok_mass_cp;
  k->mass_int_energy = ok_mass_u;
  k->mass_enthalpy = ok_mass_h;
  k->pressure_TVY = ok_pressure;
  k->temp_from_EY = ok_temp_from_E;
  k->temp_from_HY = ok_temp_from_H;
}

/* ------------------------------------------------------------- reactor */
zo_reactor *zo_reactor_new(const zo_tables *t, const zo_kinetics *kin, double Tref,
                           double min_mass_frac, double step_limiter) {
  zo_reactor *r = (zo_reactor *)zcalloc(1, sizeof(zo_reactor));
  r->t = t;
  r->kin = *kin;
  r->nsp = t->nsp;
  r->nstep = t->nstep;
  r->Tref = Tref;
  r->min_mass_frac = min_mass_frac;
  r->inv_density = 1.0;
  const int n = t->nsp, m = t->nstep;
  r->lim = (double *)zcalloc(m, sizeof(double));
  for (int j = 0; j < m; ++j) r->lim[j] = step_limiter; /* reactor_nvector_serial.cpp:56 */
  r->C = (double *)zcalloc(n, sizeof(double));
  r->net = (double *)zcalloc(n, sizeof(double));
  r->cre = (double *)zcalloc(n, sizeof(double));
  r->des = (double *)zcalloc(n, sizeof(double));
  r->rop = (double *)zcalloc(m, sizeof(double));
  r->u_RT = (double *)zcalloc(n, sizeof(double));
  r->cv_spc = (double *)zcalloc(n, sizeof(double));
  r->tmp1 = (double *)zcalloc(n + 1, sizeof(double));
  r->tmp2 = (double *)zcalloc(n + 1, sizeof(double));
  r->tmp3 = (double *)zcalloc(n + 1, sizeof(double));
  r->yscale = (double *)zcalloc(n + 1, sizeof(double));
  r->fscale = (double *)zcalloc(n + 1, sizeof(double));
  return r;
}

void zo_reactor_free(zo_reactor *r) {
  if (!r) return;
  free(r->lim); free(r->C); free(r->net); free(r->cre); free(r->des); free(r->rop);
  free(r->u_RT); free(r->cv_spc); free(r->tmp1); free(r->tmp2); free(r->tmp3);
  free(r->yscale); free(r->fscale);
  free(r);
}

/* reactor_constant_volume_cpu.cpp:27 */
void zo_reactor_set_density(zo_reactor *r, double T, double P, const double *Y) {
  r->inv_density = 1.0 / r->kin.density_TPY(r->kin.ctx, T, P, Y);
}

void zo_reactor_init_state(zo_reactor *r, double T, double P, const double *Y, double dpdt,
                           double e_src, const double *y_src) {
  r->time = 0.0;
  r->P0 = P;
  r->T0 = T;
  r->inv_density = 1.0 / r->kin.density_TPY(r->kin.ctx, T, P, Y);
  r->E0 = r->cp ? r->kin.mass_enthalpy(r->kin.ctx, T, Y) : r->kin.mass_int_energy(r->kin.ctx, T, Y);
  r->dpdt = dpdt;
  r->e_src = e_src;
  r->y_src = y_src;
}

double zo_reactor_end_temperature(const zo_reactor *r, double t, const double *Y, double T_state) {
  if (!r->fix_T) return T_state;
  const double E = r->E0 + r->e_src * t;
  return r->cp ? r->kin.temp_from_HY(r->kin.ctx, E, Y, r->T0)
               : r->kin.temp_from_EY(r->kin.ctx, E, Y, r->T0);
}

double zo_reactor_pressure(const zo_reactor *r, double t, double T, const double *Y) {
  if (r->cp && !r->y_src) return r->P0 + r->dpdt * t;
  const double P = r->kin.pressure_TVY(r->kin.ctx, T, r->inv_density, Y);
  return r->cp ? P : P + r->dpdt * t;
}

/* GetTimeDerivative: reactor_constant_volume_cpu.cpp:64-128 (cp = 0) and
 * reactor_constant_pressure_cpu.cpp:71-135 (cp = 1).  The constant-pressure
 * reactor updates inv_density from the current pressure unless mass sources
 * are set, as the reference's member does; the constant-volume reactor
 * keeps it and uses the pressure-rate corrected density locally. */
int zo_reactor_rhs(zo_reactor *r, const double *y, double *ydot) {
  const int n = r->nsp;
  const double dt = r->time;
  double T = r->fix_T ? r->T0 : y[n] * r->Tref;
  if (T <= 0.0) return 1;
  if (T > 1.0e4) T = 1.0e4;
  double v = r->inv_density;
  if (r->cp) {
    if (!r->y_src) {
      const double Pc = r->P0 + r->dpdt * dt;
      r->inv_density = 1.0 / r->kin.density_TPY(r->kin.ctx, T, Pc, y);
      v = r->inv_density;
    }
    if (r->T_force > 0.0) T = r->T_force;
    else if (r->e_src != 0.0) T = r->kin.temp_from_HY(r->kin.ctx, r->E0 + r->e_src * dt, y, T);
    r->kin.enthalpy_RT(r->kin.ctx, T, r->u_RT);
    r->mean_cv = r->kin.mass_cp(r->kin.ctx, T, y, r->cv_spc);
  } else {
    if (r->T_force > 0.0) T = r->T_force;
    else if (r->e_src != 0.0) T = r->kin.temp_from_EY(r->kin.ctx, r->E0 + r->e_src * dt, y, T);
    r->kin.int_energy_RT(r->kin.ctx, T, r->u_RT);
    r->mean_cv = r->kin.mass_cv(r->kin.ctx, T, y, r->cv_spc);
    if (r->dpdt != 0.0) {
      const double Pc = r->kin.pressure_TVY(r->kin.ctx, T, r->inv_density, y) + r->dpdt * dt;
      v = 1.0 / r->kin.density_TPY(r->kin.ctx, T, Pc, y);
    }
  }
  r->T_used = T;
  r->kin.c_from_vy(r->kin.ctx, v, y, r->C);
  r->kin.rates_limiter(r->kin.ctx, T, r->C, r->lim, r->net, r->cre, r->des, r->rop);
  double esum = 0.0;
  if (r->y_src) { /* reactor_constant_volume_cpu.cpp:108-113 */
    for (int j = 0; j < n; ++j) {
      ydot[j] = (r->net[j] * r->t->mw[j] * v + r->y_src[j]);
      esum += r->u_RT[j] * (r->net[j] * v + r->y_src[j] * (1.0 / r->t->mw[j]));
    }
  } else {
    for (int j = 0; j < n; ++j) {
      ydot[j] = (r->net[j] * r->t->mw[j] * v);
      esum += r->u_RT[j] * r->net[j] * v;
    }
  }
  double dT_dt = -esum * ZO_RU * y[n] / r->mean_cv;
  ydot[n] = r->fix_T ? 0.0 : dT_dt + (r->e_src + r->dpdt * v) / (r->mean_cv * r->Tref);
  double es = 0.0;
  for (int j = 0; j < n; ++j) {
    double m = fabs(r->cre[j]) + fabs(r->des[j]);
    r->yscale[j] = m * r->t->mw[j] * v;
    es += fabs(r->u_RT[j]) * m * v;
  }
  r->yscale[n] = es * ZO_RU * fabs(y[n]) / fabs(r->mean_cv);
  return 0;
}

void zo_mix_thermo(const zo_kinetics *k, int nsp, int n, const double *T, const double *P,
                   const double *Y, const double *E, const double *H, double *out) {
  double *tmp = (double *)zcalloc(nsp, sizeof(double));
  for (int s = 0; s < n; ++s) {
    const double *y = Y + (size_t)s * nsp;
    double *o = out + 7 * (size_t)s;
    o[0] = k->density_TPY(k->ctx, T[s], P[s], y);
    o[1] = k->pressure_TVY(k->ctx, T[s], 1.0 / o[0], y);
    o[2] = k->mass_int_energy(k->ctx, T[s], y);
    o[3] = k->mass_enthalpy(k->ctx, T[s], y);
    o[4] = k->mass_cp(k->ctx, T[s], y, tmp);
    o[5] = k->temp_from_EY(k->ctx, E[s], y, T[s]);
    o[6] = k->temp_from_HY(k->ctx, H[s], y, T[s]);
  }
  free(tmp);
}

int zo_reactor_rhs_batch(const zo_tables *t, const zo_kinetics *k, int cp, int n,
                         const double *T0, const double *P0, const double *Y0,
                         const double *dpdt, const double *e_src, const double *y_src,
                         const double *tm, const double *y, double *ydot) {
  const int ns = t->nsp;
  int nfail = 0;
  zo_reactor *r = zo_reactor_new(t, k, 1.0, 1.0e-30, 1.0e22);
  r->cp = cp;
  for (int s = 0; s < n; ++s) {
    zo_reactor_init_state(r, T0[s], P0[s], Y0 + (size_t)s * ns, dpdt ? dpdt[s] : 0.0,
                          e_src ? e_src[s] : 0.0, y_src ? y_src + (size_t)s * ns : NULL);
    r->time = tm[s];
    if (zo_reactor_rhs(r, y + (size_t)s * (ns + 1), ydot + (size_t)s * (ns + 1))) ++nfail;
  }
  zo_reactor_free(r);
  return nfail;
}

/* ------------------------------------------------------ Jacobian pattern */
/* reactor_nvector_serial.cpp:122-281 SetupSparseJacobianArrays */
zo_jac_pattern *zo_jac_pattern_new(const zo_tables *t) {
  const int ns = t->nsp, nv = ns + 1;
  int *nzf = (int *)zcalloc((size_t)nv * nv, sizeof(int)); /* [col*nv+row] */
  for (int j = 0; j < ns; ++j) {
    nzf[j * nv + j] = 1;
    nzf[j * nv + ns] = 1;
  }
  for (int k = 0; k < nv; ++k) nzf[ns * nv + k] = 1;
  int nd = 0, nc = 0;
  for (int j = 0; j < t->nstep; ++j) {
    int nr = t->reac_ptr[j + 1] - t->reac_ptr[j];
    int np = t->prod_ptr[j + 1] - t->prod_ptr[j];
    nd += nr * nr;
    nc += nr * np;
  }
  zo_jac_pattern *p = (zo_jac_pattern *)zcalloc(1, sizeof(zo_jac_pattern));
  p->n = nv;
  p->n_des = nd;
  p->n_cre = nc;
  p->des_conc = (int *)zcalloc(nd, sizeof(int));
  p->des_step = (int *)zcalloc(nd, sizeof(int));
  p->des_nz = (int *)zcalloc(nd, sizeof(int));
  p->cre_conc = (int *)zcalloc(nc, sizeof(int));
  p->cre_step = (int *)zcalloc(nc, sizeof(int));
  p->cre_nz = (int *)zcalloc(nc, sizeof(int));
  int id = 0, ic = 0;
  for (int j = 0; j < t->nstep; ++j) {
    for (int k = t->reac_ptr[j]; k < t->reac_ptr[j + 1]; ++k) {
      int col = t->reac_spc[k];
      for (int m = t->reac_ptr[j]; m < t->reac_ptr[j + 1]; ++m) {
        int row = t->reac_spc[m];
        nzf[col * nv + row] = 1;
        p->des_conc[id] = col; p->des_step[id] = j; p->des_nz[id] = row; ++id;
      }
      for (int m = t->prod_ptr[j]; m < t->prod_ptr[j + 1]; ++m) {
        int row = t->prod_spc[m];
        nzf[col * nv + row] = 1;
        p->cre_conc[ic] = col; p->cre_step[ic] = j; p->cre_nz[ic] = row; ++ic;
      }
    }
  }
  int cnt = 1;
  p->col_ptr = (int *)zcalloc(nv + 1, sizeof(int));
  for (int j = 0; j < nv; ++j) {
    for (int k = 0; k < nv; ++k)
      if (nzf[j * nv + k] == 1) nzf[j * nv + k] = cnt++;
    p->col_ptr[j + 1] = cnt - 1;
  }
  p->nnz = cnt - 1;
  p->row_idx = (int *)zcalloc(p->nnz, sizeof(int));
  p->last_row = (int *)zcalloc(nv, sizeof(int));
  for (int j = 0; j < nv; ++j) {
    for (int k = 0; k < nv; ++k) {
      int a = nzf[j * nv + k];
      if (a > 0) p->row_idx[a - 1] = k;
    }
    p->last_row[j] = nzf[(j + 1) * nv - 1] - 1;
  }
  for (int i = 0; i < nd; ++i) p->des_nz[i] = nzf[p->des_conc[i] * nv + p->des_nz[i]] - 1;
  for (int i = 0; i < nc; ++i) p->cre_nz[i] = nzf[p->cre_conc[i] * nv + p->cre_nz[i]] - 1;
  free(nzf);
  return p;
}

void zo_jac_pattern_free(zo_jac_pattern *p) {
  if (!p) return;
  free(p->col_ptr); free(p->row_idx); free(p->last_row);
  free(p->des_conc); free(p->des_step); free(p->des_nz);
  free(p->cre_conc); free(p->cre_step); free(p->cre_nz);
  free(p);
}

/* reactor_nvector_serial.cpp:610-771 SetupJacobianSparse (integer network,
 * temperature solved).  UNIT_ROUNDOFF is DBL_EPSILON (SUNDIALS realtype). */
int zo_jac_values(zo_reactor *r, const zo_jac_pattern *p, const double *y, const double *fy,
                  double *jac, double *scale) {
  const int ns = r->nsp, nv = ns + 1;
  const double *mw = r->t->mw;
  double *t1 = r->tmp1, *t2 = r->tmp2, *t3 = r->tmp3;
  const double mmf = r->min_mass_frac;
  const double sqrt_ur = sqrt(2.2204460492503131e-16);
  for (int j = 0; j < ns; ++j) {
    t1[j] = y[j];
    if (fabs(t1[j]) < mmf) t1[j] = (t1[j] < 0.0) ? -mmf : mmf;
    t2[j] = mw[j] / t1[j] * r->inv_density;
  }
  t1[ns] = y[ns];
  if (zo_reactor_rhs(r, t1, t3)) return 1;
  for (int k = 0; k < p->nnz; ++k) jac[k] = 0.0;
  if (scale)
    for (int k = 0; k < p->nnz; ++k) scale[k] = 0.0;
  for (int i = 0; i < p->n_des; ++i) {
    double v = r->rop[p->des_step[i]] * t2[p->des_conc[i]];
    jac[p->des_nz[i]] -= v;
    if (scale) scale[p->des_nz[i]] += fabs(v);
  }
  for (int i = 0; i < p->n_cre; ++i) {
    double v = r->rop[p->cre_step[i]] * t2[p->cre_conc[i]];
    jac[p->cre_nz[i]] += v;
    if (scale) scale[p->cre_nz[i]] += fabs(v);
  }
  /* d(Tdot)/dy_j */
  const double RuTemp = ZO_RU * y[ns];
  for (int j = 0; j < ns; ++j) {
    int lr = p->last_row[j];
    jac[lr] = 0.0;
    double sc = 0.0;
    for (int k = p->col_ptr[j]; k < p->col_ptr[j + 1] - 1; ++k) {
      jac[lr] += jac[k] * r->u_RT[p->row_idx[k]];
      if (scale) sc += scale[k] * fabs(r->u_RT[p->row_idx[k]]);
    }
    jac[lr] *= RuTemp;
    if (scale) scale[lr] = sc * fabs(RuTemp);
  }
  /* the Tdot term carries Tdot's own rounding: its scale is the magnitude
   * sum of Tdot's terms (yscale of the clamped evaluation), not |Tdot|, which
   * cancellation can make far smaller */
  for (int j = 0; j < ns; ++j) {
    int lr = p->last_row[j];
    double add = t3[ns] * r->cv_spc[j] * mw[j];
    jac[lr] += add;
    if (scale) scale[lr] += fabs(r->yscale[ns] * r->cv_spc[j] * mw[j]);
  }
  const double multFact = -1.0 / (r->mean_cv);
  for (int j = 0; j < ns; ++j) {
    int lr = p->last_row[j];
    jac[lr] *= (1.0 / mw[j]) * multFact;
    if (scale) scale[lr] *= fabs((1.0 / mw[j]) * multFact);
    if (r->fix_T) jac[lr] = 0.0; /* no temperature row without solve_temperature_ */
  }
  /* d(ydot)/dT by forward difference */
  double dT = y[ns] * sqrt_ur;
  t1[ns] += dT;
  dT = t1[ns] - y[ns];
  const double mult = 1.0 / dT;
  for (int j = 0; j < ns; ++j) t1[j] = y[j];
  if (zo_reactor_rhs(r, t1, t3)) return 1;
  for (int k = p->col_ptr[ns]; k < p->col_ptr[nv]; ++k) {
    int row = p->row_idx[k];
    jac[k] = (t3[row] - fy[row]) * mult;
    /* forward-difference rounding scale: term magnitudes of both RHS / dT */
    if (scale) scale[k] = (r->yscale[row] + r->fscale[row]) * fabs(mult);
  }
  /* dC -> dY conversion */
  for (int j = 0; j < ns; ++j) {
    for (int k = p->col_ptr[j]; k < p->col_ptr[j + 1]; ++k) {
      const int row = p->row_idx[k];
      if (row < ns) {
        jac[k] *= mw[row] * (1.0 / mw[j]);
        if (scale) scale[k] *= mw[row] * (1.0 / mw[j]);
      }
    }
  }
  return 0;
}

/* ------------------------------------------------------- batched driver */
int zo_batch_rates_jac(const zo_tables *t, const zo_jac_pattern *p, const zo_kinetics *kins,
                       int nthreads, int nstates, const double *T, const double *P,
                       const double *Y, double Tref, double min_mass_frac,
                       double step_limiter, double *wdot, double *jac, double *ydot) {
  const int ns = t->nsp, nv = ns + 1;
  int nfail = 0;
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads) reduction(+ : nfail)
  {
    int tid = 0, nth = 1;
#ifdef _OPENMP
    tid = omp_get_thread_num();
    nth = omp_get_num_threads();
#endif
    zo_reactor *r = zo_reactor_new(t, &kins[tid], Tref, min_mass_frac, step_limiter);
    double *y = (double *)zcalloc(nv, sizeof(double));
    double *fy = (double *)zcalloc(nv, sizeof(double));
    long lo = (long)nstates * tid / nth, hi = (long)nstates * (tid + 1) / nth;
    for (long s = lo; s < hi; ++s) {
      const double *Ys = Y + s * ns;
      zo_reactor_set_density(r, T[s], P[s], Ys);
      for (int j = 0; j < ns; ++j) y[j] = Ys[j];
      y[ns] = T[s] / Tref;
      if (zo_reactor_rhs(r, y, fy)) { ++nfail; continue; }
      if (wdot) memcpy(wdot + s * ns, r->net, sizeof(double) * ns);
      if (ydot) memcpy(ydot + s * nv, fy, sizeof(double) * nv);
      if (jac && zo_jac_values(r, p, y, fy, jac + s * (long)p->nnz, NULL)) ++nfail;
    }
    free(y); free(fy);
    zo_reactor_free(r);
  }
  return nfail;
}

int zo_batch_rates_jac_scaled(const zo_tables *t, const zo_jac_pattern *p, int nstates,
                              const double *T, const double *P, const double *Y, double Tref,
                              double min_mass_frac, double step_limiter, double *wdot,
                              double *jac, double *wscale, double *jscale) {
  const int ns = t->nsp, nv = ns + 1;
  zo_kinetics kin;
  zo_kinetics_oracle(t, &kin);
  zo_reactor *r = zo_reactor_new(t, &kin, Tref, min_mass_frac, step_limiter);
  double *y = (double *)zcalloc(nv, sizeof(double));
  double *fy = (double *)zcalloc(nv, sizeof(double));
  int nfail = 0;
  for (long s = 0; s < nstates; ++s) {
    const double *Ys = Y + s * ns;
    zo_reactor_set_density(r, T[s], P[s], Ys);
    for (int j = 0; j < ns; ++j) y[j] = Ys[j];
    y[ns] = T[s] / Tref;
    if (zo_reactor_rhs(r, y, fy)) { ++nfail; continue; }
    memcpy(wdot + s * ns, r->net, sizeof(double) * ns);
    for (int j = 0; j < ns; ++j) wscale[s * ns + j] = fabs(r->cre[j]) + fabs(r->des[j]);
    memcpy(r->fscale, r->yscale, sizeof(double) * nv);
    if (zo_jac_values(r, p, y, fy, jac + s * (long)p->nnz, jscale + s * (long)p->nnz)) ++nfail;
  }
  free(y); free(fy);
  zo_reactor_free(r);
  return nfail;
}
