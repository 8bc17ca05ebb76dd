// ref_shim.cpp -- ORACLE test infrastructure: a thin C interface over the
// reference's own zerork::mechanism library, compiled from the reference
// sources by oracle/Makefile into oracle/_ref.  It exposes
//  * the mechanism tables the reference builds internally (rate_const.h:98-170,
//    info_net.h accessors) so the product's own CHEMKIN loader can be checked
//    against them element by element;
//  * the reference's rate, thermo and Kfwd/Krev entry points (mechanism.h:114-160);
//  * a kinetics provider so the plugin-level RHS/Jacobian restatement in
//    zrk_oracle.c runs on top of the reference library (the CPU baseline).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include <stdexcept>

// The reference keeps its tables in protected members; the oracle reads them.
#define protected public
#define private public
#include "zerork/mechanism.h"
#undef protected
#undef private

#include "zrk_oracle.h"

using zerork::mechanism;

extern "C" {

void *zrkref_load(const char *mech, const char *therm, const char *log, int verbosity) {
  try {
    return new mechanism(mech, therm, log, verbosity);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "zrkref_load: %s\n", e.what());
    return nullptr;
  }
}

void zrkref_free(void *h) { delete static_cast<mechanism *>(h); }

int zrkref_num_species(void *h) { return static_cast<mechanism *>(h)->getNumSpecies(); }
int zrkref_num_reactions(void *h) { return static_cast<mechanism *>(h)->getNumReactions(); }
int zrkref_num_steps(void *h) { return static_cast<mechanism *>(h)->getNumSteps(); }
const char *zrkref_species_name(void *h, int i) {
  return static_cast<mechanism *>(h)->getSpeciesName(i);
}

// Dump the reference's internal tables in the oracle's layout.
zo_tables *zrkref_tables(void *hp) {
  mechanism *m = static_cast<mechanism *>(hp);
  zerork::info_net *inf = m->infoNet;
  zerork::rate_const *rc = m->Kconst;
  const int nsp = m->getNumSpecies(), nstep = m->getNumSteps();
  int s[14];
  s[0] = nsp;
  s[1] = m->getNumReactions();
  s[2] = nstep;
  s[3] = inf->getTotalReactants();
  s[4] = inf->getTotalProducts();
  s[5] = rc->nArrheniusStep;
  s[6] = rc->nFromKeqStep;
  s[7] = rc->nThirdBodyRxn;
  s[8] = rc->nFalloffRxn;
  int ntbe = 0, nfoe = 0;
  for (int j = 0; j < rc->nThirdBodyRxn; ++j) ntbe += rc->thirdBodyRxnList[j].nEnhanced;
  for (int j = 0; j < rc->nFalloffRxn; ++j)
    if (rc->falloffRxnList[j].falloffSpcIdx < 0) nfoe += rc->falloffRxnList[j].nEnhanced;
  s[9] = ntbe;
  s[10] = nfoe;
  // PLOG reactions: the reference's PLogReaction objects (plog_reaction.h)
  int npt = 0, nln = 0;
  for (int j = 0; j < rc->nPLogInterpolationStep; ++j) {
    npt += rc->plogInterpolationStepList[j].num_pressure_points_;
    nln += rc->plogInterpolationStepList[j].total_arrhenius_lines_;
  }
  s[11] = rc->nPLogInterpolationStep;
  s[12] = npt;
  s[13] = nln;
  zo_tables *t = zo_tables_alloc(s);
  m->getMolWtSpc(t->mw);
  std::vector<double> coef(nsp * 16);
  m->getThermoCoeffs(coef.data());
  for (int j = 0; j < nsp * 16; ++j) t->thermo[j] = coef[j];
  int rr = 0, pp = 0;
  for (int j = 0; j < nstep; ++j) {
    t->step_rxn[j] = inf->getRxnIdxOfStep(j);
    t->step_dir[j] = inf->getRxnDirOfStep(j);
    t->reac_ptr[j] = rr;
    t->prod_ptr[j] = pp;
    for (int k = 0; k < inf->getOrderOfStep(j); ++k) t->reac_spc[rr++] = inf->getSpecIdxOfStepReactant(j, k);
    for (int k = 0; k < inf->getNumProductsOfStep(j); ++k) t->prod_spc[pp++] = inf->getSpecIdxOfStepProduct(j, k);
  }
  t->reac_ptr[nstep] = rr;
  t->prod_ptr[nstep] = pp;
  // Arrhenius steps, re-listed in ascending step order.
  std::vector<std::pair<int, int>> arr;
  for (int j = 0; j < rc->nArrheniusStep; ++j)
    arr.push_back({rc->arrheniusStepList[j].stepIdx, rc->arrheniusStepList[j].arrheniusIdx});
  std::sort(arr.begin(), arr.end());
  for (size_t j = 0; j < arr.size(); ++j) {
    t->arr_step[j] = arr[j].first;
    t->arr_lnA[j] = rc->distinctArrheniusLogAfact[arr[j].second];
    t->arr_n[j] = rc->distinctArrheniusTpow[arr[j].second];
    t->arr_Ta[j] = rc->distinctArrheniusTact[arr[j].second];
  }
  for (int j = 0; j < rc->nFromKeqStep; ++j) {
    t->keq_step[j] = rc->fromKeqStepList[j].stepIdx;
    t->keq_fwd[j] = rc->fromKeqStepList[j].fwdStepIdx;
    t->keq_dn[j] = rc->fromKeqStepList[j].nDelta;
  }
  int e = 0;
  for (int j = 0; j < rc->nThirdBodyRxn; ++j) {
    const zerork::thirdBodyRxn &tb = rc->thirdBodyRxnList[j];
    t->tb_fwd[j] = tb.fwdStepIdx;
    t->tb_rev[j] = tb.revStepIdx < 0 ? -1 : tb.revStepIdx;
    t->tb_ptr[j] = e;
    for (int k = 0; k < tb.nEnhanced; ++k) {
      t->tb_spc[e] = tb.etbSpcIdx[k];
      t->tb_alpha[e] = tb.etbSpcEff[k];
      ++e;
    }
  }
  t->tb_ptr[rc->nThirdBodyRxn] = e;
  e = 0;
  for (int j = 0; j < rc->nFalloffRxn; ++j) {
    const zerork::falloffRxn &fo = rc->falloffRxnList[j];
    t->fo_fwd[j] = fo.fwdStepIdx;
    t->fo_rev[j] = fo.revStepIdx < 0 ? -1 : fo.revStepIdx;
    t->fo_spc[j] = fo.falloffSpcIdx < 0 ? -1 : fo.falloffSpcIdx;
    t->fo_ptr[j] = e;
    if (fo.falloffSpcIdx < 0) {
      for (int k = 0; k < fo.nEnhanced; ++k) {
        t->fo_eff_spc[e] = fo.etbSpcIdx[k];
        t->fo_alpha[e] = fo.etbSpcEff[k];
        ++e;
      }
    }
    double *p = t->fo_par + 8 * j;
    for (int k = 0; k < 8; ++k) p[k] = 0.0;
    for (size_t k = 0; k < fo.param.size() && k < 8; ++k) p[k] = fo.param[k];
    switch (fo.falloffType) {
      case zerork::LINDEMANN: t->fo_type[j] = ZO_FO_LINDEMANN; break;
      case zerork::TROE_THREE_PARAMS: t->fo_type[j] = ZO_FO_TROE3; break;
      case zerork::TROE_FOUR_PARAMS: t->fo_type[j] = ZO_FO_TROE4; break;
      case zerork::SRI:
        t->fo_type[j] = ZO_FO_SRI;
        if (fo.param.size() < 7) p[6] = 1.0;
        if (fo.param.size() < 8) p[7] = 0.0;
        break;
    }
  }
  t->fo_ptr[rc->nFalloffRxn] = e;
  int q = 0, l = 0;
  for (int j = 0; j < rc->nPLogInterpolationStep; ++j) {
    const zerork::PLogReaction &pr = rc->plogInterpolationStepList[j];
    t->plog_step[j] = pr.step_index_;
    t->plog_pt_ptr[j] = q;
    for (int k = 0; k < pr.num_pressure_points_; ++k, ++q) {
      t->plog_p[q] = pr.pressure_points_[k];
      t->plog_lnp[q] = pr.log_e_pressure_points_[k];
      t->plog_ln_ptr[q] = l + pr.start_line_at_pressure_[k];
    }
    for (int k = 0; k < pr.total_arrhenius_lines_; ++k) {
      t->plog_lnA[l + k] = pr.log_e_afactor_[k];
      t->plog_sgn[l + k] = pr.sign_afactor_[k];
      t->plog_n[l + k] = pr.temperature_power_[k];
      t->plog_Ta[l + k] = pr.activation_temperature_[k];
    }
    l += pr.total_arrhenius_lines_;
  }
  t->plog_pt_ptr[rc->nPLogInterpolationStep] = q;
  t->plog_ln_ptr[npt] = l;
  return t;
}

void zrkref_krxn(void *h, double T, const double *C, double *Kf, double *Kr) {
  static_cast<mechanism *>(h)->getKrxnFromTC(T, C, Kf, Kr);
}

void zrkref_rates(void *h, double T, const double *C, double *net, double *cre, double *des,
                  double *rop) {
  static_cast<mechanism *>(h)->getReactionRates(T, C, net, cre, des, rop);
}

void zrkref_rates_limiter(void *h, double T, const double *C, const double *lim, double *net,
                          double *cre, double *des, double *rop) {
  static_cast<mechanism *>(h)->getReactionRatesLimiter(T, C, lim, net, cre, des, rop);
}

void zrkref_thermo(void *h, double T, double *cp_R, double *h_RT, double *g_RT) {
  mechanism *m = static_cast<mechanism *>(h);
  m->getCp_R_Enthalpy_RT(T, cp_R, h_RT);
  m->getNonDimGibbsFromT(T, g_RT);
}

static void rk_rates(void *ctx, double T, const double *C, const double *lim, double *net,
                     double *cre, double *des, double *rop) {
  static_cast<mechanism *>(ctx)->getReactionRatesLimiter(T, C, lim, net, cre, des, rop);
}
static void rk_u(void *ctx, double T, double *u) {
  static_cast<mechanism *>(ctx)->getIntEnergy_RT(T, u);
}
static double rk_cv(void *ctx, double T, const double *y, double *cv) {
  return static_cast<mechanism *>(ctx)->getMassCvFromTY(T, y, cv);
}
static double rk_dens(void *ctx, double T, double P, const double *y) {
  return static_cast<mechanism *>(ctx)->getDensityFromTPY(T, P, y);
}
static void rk_c(void *ctx, double v, const double *y, double *c) {
  static_cast<mechanism *>(ctx)->getCfromVY(v, y, c);
}

static void rk_h(void *ctx, double T, double *h) {
  static_cast<mechanism *>(ctx)->getEnthalpy_RT(T, h);
}
static double rk_cp(void *ctx, double T, const double *y, double *cp) {
  return static_cast<mechanism *>(ctx)->getMassCpFromTY(T, y, cp);
}
static double rk_mass_u(void *ctx, double T, const double *y) {
  return static_cast<mechanism *>(ctx)->getMassIntEnergyFromTY(T, y);
}
static double rk_mass_h(void *ctx, double T, const double *y) {
  return static_cast<mechanism *>(ctx)->getMassEnthalpyFromTY(T, y);
}
static double rk_pres(void *ctx, double T, double v, const double *y) {
  return static_cast<mechanism *>(ctx)->getPressureFromTVY(T, v, y);
}
static double rk_T_from_E(void *ctx, double E, const double *y, double Tg) {
  return static_cast<mechanism *>(ctx)->getTemperatureFromEY(E, y, Tg);
}
static double rk_T_from_H(void *ctx, double H, const double *y, double Tg) {
  return static_cast<mechanism *>(ctx)->getTemperatureFromHY(H, y, Tg);
}

void zrkref_kinetics(void *h, zo_kinetics *k) {
  k->ctx = h;
  k->rates_limiter = rk_rates;
  k->int_energy_RT = rk_u;
  k->mass_cv = rk_cv;
  k->density_TPY = rk_dens;
  k->c_from_vy = rk_c;
  k->enthalpy_RT = rk_h;
  k->mass_cp = rk_cp;
  k->mass_int_energy = rk_mass_u;
  k->mass_enthalpy = rk_mass_h;
  k->pressure_TVY = rk_pres;
  k->temp_from_EY = rk_T_from_E;
  k->temp_from_HY = rk_T_from_H;
}

// Mixture thermodynamics and reactor right-hand sides (zrk_oracle.h test
// hooks) on the reference library's own mechanism functions.
void zrkref_mix_thermo(void *h, int n, const double *T, const double *P, const double *Y,
                       const double *E, const double *H, double *out) {
  zo_kinetics k;
  zrkref_kinetics(h, &k);
  zo_mix_thermo(&k, static_cast<mechanism *>(h)->getNumSpecies(), n, T, P, Y, E, H, out);
}

int zrkref_reactor_rhs_batch(void *h, const zo_tables *t, int cp, int n, const double *T0,
                             const double *P0, const double *Y0, const double *dpdt,
                             const double *e_src, const double *y_src, const double *tm,
                             const double *y, double *ydot) {
  zo_kinetics k;
  zrkref_kinetics(h, &k);
  return zo_reactor_rhs_batch(t, &k, cp, n, T0, P0, Y0, dpdt, e_src, y_src, tm, y, ydot);
}

// Rates + plugin Jacobian over many states on the reference library, one
// mechanism object per thread (mechanism workspaces are not thread-safe).
int zrkref_batch_rates_jac(void **handles, int nthreads, const zo_tables *t,
                           const zo_jac_pattern *p, int nstates, const double *T,
                           const double *P, const double *Y, double Tref, double mmf,
                           double lim, double *wdot, double *jac, double *ydot) {
  std::vector<zo_kinetics> kins(nthreads);
  for (int i = 0; i < nthreads; ++i) zrkref_kinetics(handles[i], &kins[i]);
  return zo_batch_rates_jac(t, p, kins.data(), nthreads, nstates, T, P, Y, Tref, mmf, lim, wdot,
                            jac, ydot);
}

}  // extern "C"
