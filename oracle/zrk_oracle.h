/*
 * zrk_oracle.h -- CPU ORACLE (test infrastructure only, never shipped).
 *
 * A plain-C restatement of Zero-RK's batched stiff-reactor hot path, used as
 * the checker for the sm_100a kernels.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg load it.  Each function cites the reference
 * file:line it restates (paths relative to the Zero-RK checkout).
 *
 * Parity pinning: the rate/thermo/RHS functions are checked against the
 * reference's own zerork::mechanism library compiled from its sources by
 * oracle/Makefile (oracle/_ref), and against the closed-form known-answer
 * tests of tests/reactions/troe_gtest.cpp (6e-15 relative).
 */
#ifndef ZRK_ORACLE_H
#define ZRK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Falloff kinds: src/zerork/rate_const.h:13-16 (LINDEMANN, TROE_THREE_PARAMS,
 * TROE_FOUR_PARAMS, SRI). */
enum { ZO_FO_LINDEMANN = 0, ZO_FO_TROE3 = 1, ZO_FO_TROE4 = 2, ZO_FO_SRI = 3 };

/* Mechanism tables in the reference's own indexing:
 *  - species order = SPECIES section order (mechanism.cpp:117-138)
 *  - step order    = fwd, rev interleaved per reaction (info_net.cpp:65-97)
 *  - reactant/product lists expanded by integer stoichiometry
 *    (info_net.cpp:219-330)
 *  - Arrhenius parameters after unit conversion and the 1e-6 distinct-value
 *    merge (rate_const.cpp:266-332, :1093-1106), listed per step
 *  - reverse-from-Keq steps (rate_const.cpp:334-384)
 *  - third-body and falloff lists (rate_const.cpp:386-537), efficiencies in
 *    std::map (species-name) order, alpha = efficiency - 1.
 * fo_par holds 8 doubles per falloff reaction:
 *  [ln(Alow'), n_low, Ta_low, p3, p4, p5, p6, p7]
 *  Troe: p3=alpha, p4=T***, p5=T*, p6=T** (Troe4 only)
 *  SRI : p3=a, p4=b, p5=1/c (or -1), p6=d (1 if absent), p7=e (0 if absent) */
typedef struct zo_tables {
  int nsp, nrxn, nstep;
  int tot_reac, tot_prod;
  int n_arr, n_keq, n_tb, n_fo, n_tb_eff, n_fo_eff;
  int n_plog, n_plog_pt, n_plog_ln;
  double *mw;        /* [nsp] kg/kmol */
  double *thermo;    /* [nsp*16]: Tmid, 7 low, 7 high, pad */
  int *step_rxn;     /* [nstep] */
  int *step_dir;     /* [nstep] +1 fwd / -1 rev */
  int *reac_ptr;     /* [nstep+1] */
  int *reac_spc;     /* [tot_reac] */
  int *prod_ptr;     /* [nstep+1] */
  int *prod_spc;     /* [tot_prod] */
  int *arr_step;     /* [n_arr] ascending step index */
  double *arr_lnA, *arr_n, *arr_Ta;  /* [n_arr] */
  int *keq_step, *keq_fwd;           /* [n_keq] */
  double *keq_dn;                    /* [n_keq] nProd - nReac of fwd step */
  int *tb_fwd, *tb_rev, *tb_ptr, *tb_spc;  /* rev = -1 if irreversible */
  double *tb_alpha;
  int *fo_fwd, *fo_rev, *fo_type, *fo_spc, *fo_ptr, *fo_eff_spc;  /* fo_spc=-1 => M */
  double *fo_alpha, *fo_par;
  /* PLOG reactions (plog_reaction.cpp:8-132, rate_const.cpp:1146-1185): the
   * forward step, distinct pressures [plog_pt_ptr[j], plog_pt_ptr[j+1]) in Pa
   * (ascending) with their logs, and per pressure the Arrhenius lines
   * [plog_ln_ptr[q], plog_ln_ptr[q+1]): ln|A|, sign of A, n, Ta */
  int *plog_step, *plog_pt_ptr, *plog_ln_ptr;
  double *plog_p, *plog_lnp, *plog_lnA, *plog_sgn, *plog_n, *plog_Ta;
} zo_tables;

zo_tables *zo_tables_alloc(const int sizes[14]); /* nsp,nrxn,nstep,tot_reac,tot_prod,
                                                   n_arr,n_keq,n_tb,n_fo,n_tb_eff,n_fo_eff,
                                                   n_plog,n_plog_pt,n_plog_ln */
/* A PLOG reaction's rate coefficient at (T, P) (plog_reaction.cpp:187-300,
 * logarithmic interpolation between the bracketing pressures, the end
 * pressures' values outside them) */
double zo_plog_k(const zo_tables *t, int j, double T, double invT, double logT, double P);
void zo_tables_free(zo_tables *t);

/* Physical constants: src/zerork/constants.h:10-24 */
#define ZO_RU 8.314462618e3
#define ZO_PATM 1.01325e5

/* ---- thermo: src/zerork/nasa_poly.cpp:50-172 ---- */
void zo_cp_R(const zo_tables *t, double T, double *cp_R);
void zo_h_RT(const zo_tables *t, double T, double *h_RT);
void zo_g_RT(const zo_tables *t, double T, double *g_RT);

/* ---- rate coefficients: src/zerork/rate_const.cpp:539-582 (updateK) ---- */
void zo_rate_coefs(const zo_tables *t, double T, const double *C, double *K);

/* ---- rates: src/zerork/perf_net.cpp:190-274 (calcRatesFromTC_StepLimiter);
 * lim may be NULL for perf_net.cpp:126-188 (calcRatesFromTC). ---- */
void zo_rates(const zo_tables *t, double T, const double *C, const double *lim,
              double *net, double *cre, double *des, double *rop);

/* Kinetics provider: the reactor/Jacobian restatement calls mechanism-level
 * functions through this table so the same assembly code can run on top of
 * either this restatement or the reference library itself. */
typedef struct zo_kinetics {
  void *ctx;
  void (*rates_limiter)(void *ctx, double T, const double *C, const double *lim,
                        double *net, double *cre, double *des, double *rop);
  void (*int_energy_RT)(void *ctx, double T, double *u_RT);
  double (*mass_cv)(void *ctx, double T, const double *y, double *cv_spc);
  double (*density_TPY)(void *ctx, double T, double P, const double *y);
  void (*c_from_vy)(void *ctx, double v, const double *y, double *c);
  /* constant-pressure reactor and energy/pressure sources
   * (src/zerork/mechanism.cpp:292-547) */
  void (*enthalpy_RT)(void *ctx, double T, double *h_RT);
  double (*mass_cp)(void *ctx, double T, const double *y, double *cp_spc);
  double (*mass_int_energy)(void *ctx, double T, const double *y);
  double (*mass_enthalpy)(void *ctx, double T, const double *y);
  double (*pressure_TVY)(void *ctx, double T, double v, const double *y);
  double (*temp_from_EY)(void *ctx, double E, const double *y, double T_guess);
  double (*temp_from_HY)(void *ctx, double H, const double *y, double T_guess);
} zo_kinetics;

void zo_kinetics_oracle(const zo_tables *t, zo_kinetics *k);

/* Reactor state: constant volume (applications/cfd_plugin/
 * reactor_constant_volume_cpu.cpp:15-41 InitializeState) or constant
 * pressure (reactor_constant_pressure_cpu.cpp:15-41).  u_RT, cv_spc and
 * mean_cv hold the reactor's energy_, cx_mass_ and mean_cx_mass_: internal
 * energy and c_v for constant volume, enthalpy and c_p for constant
 * pressure. */
typedef struct zo_reactor {
  const zo_tables *t;
  zo_kinetics kin;
  int nsp, nstep;
  double inv_density, Tref, min_mass_frac;
  int cp;          /* 1: constant pressure (plugin option constant_volume = 0) */
  double dpdt;     /* pressure rate (Pa/s), ZERORK_FIELD_DPDT */
  double e_src;    /* energy source (J/kg/s), ZERORK_FIELD_E_SRC */
  double P0, T0;   /* pressure_ and initial_temperature_ */
  double E0;       /* initial_energy_: mass u (constant volume) or h (constant pressure) */
  double time;     /* time argument of the next evaluation, from the start of the call */
  double T_force;  /* > 0: evaluate at this temperature instead of the state's or the
                      energy source's (a finite-difference hook of the integrator) */
  double T_used;   /* temperature the last evaluation used */
  int fix_T;       /* 1: temperature not solved (solve_temperature_ false,
                      zerork_reactor_manager.cpp:1107-1113): the rates see T0
                      (or the energy source's temperature), Tdot = 0 */
  double *lim, *C, *net, *cre, *des, *rop, *u_RT, *cv_spc, mean_cv;
  double *tmp1, *tmp2, *tmp3;
  double *yscale;  /* [nsp+1] rounding scale of the last ydot: sum of |terms| */
  double *fscale;  /* [nsp+1] yscale of the caller's fy (set by the batch driver) */
  const double *y_src; /* [nsp] mass-fraction source terms (1/s) or NULL (ZERORK_FIELD_Y_SRC) */
} zo_reactor;

zo_reactor *zo_reactor_new(const zo_tables *t, const zo_kinetics *kin,
                           double Tref, double min_mass_frac, double step_limiter);
void zo_reactor_free(zo_reactor *r);
/* Density from (T, P, Y): sets inv_density. */
void zo_reactor_set_density(zo_reactor *r, double T, double P, const double *Y);
/* InitializeState at time 0 (reactor_constant_volume_cpu.cpp:15-41,
 * reactor_constant_pressure_cpu.cpp:15-41): density, initial energy and the
 * sources; r->cp selects the reactor. */
void zo_reactor_init_state(zo_reactor *r, double T, double P, const double *Y, double dpdt,
                           double e_src, const double *y_src);
/* GetState's pressure at time t for the end state (T, Y)
 * (reactor_constant_volume_cpu.cpp:59, reactor_constant_pressure_cpu.cpp:59-63). */
double zo_reactor_pressure(const zo_reactor *r, double t, double T, const double *Y);
/* GetState's temperature at time t: the state's T_state, or with fix_T the
 * temperature of the energy E0 + e_src t at composition Y
 * (reactor_constant_volume_cpu.cpp:51-56, reactor_constant_pressure_cpu.cpp:52-57). */
double zo_reactor_end_temperature(const zo_reactor *r, double t, const double *Y, double T_state);

/* ydot for y = [Y, T/Tref] at time r->time: GetTimeDerivative of
 * reactor_constant_volume_cpu.cpp:64-128 or reactor_constant_pressure_cpu.cpp:
 * 71-135.  Returns 1 if T <= 0. */
int zo_reactor_rhs(zo_reactor *r, const double *y, double *ydot);

/* Mixture thermodynamics through a kinetics provider (test hook), per state
 * s (Y reactor-major [n][nsp]): out[7s .. 7s+6] = density(T, P, Y),
 * pressure(T, 1/density, Y), mass u(T, Y), mass h(T, Y), mass c_p(T, Y),
 * T from (E[s], Y) and T from (H[s], Y), both with guess T[s]. */
void zo_mix_thermo(const zo_kinetics *k, int nsp, int n, const double *T, const double *P,
                   const double *Y, const double *E, const double *H, double *out);
/* GetTimeDerivative over states (test hook): reactor s initialised at
 * (T0, P0, Y0) with sources dpdt, e_src and y_src (each may be NULL), then
 * ydot at time tm[s] and state y[s] ([n][nsp+1] both).  cp selects the
 * constant-pressure reactor.  Returns the number of failed evaluations. */
int zo_reactor_rhs_batch(const zo_tables *t, const zo_kinetics *k, int cp, int n,
                         const double *T0, const double *P0, const double *Y0,
                         const double *dpdt, const double *e_src, const double *y_src,
                         const double *tm, const double *y, double *ydot);

/* Fixed Jacobian pattern: reactor_nvector_serial.cpp:122-281
 * (SetupSparseJacobianArrays), CSC over n = nsp+1 variables. */
typedef struct zo_jac_pattern {
  int n, nnz;
  int *col_ptr;   /* [n+1] */
  int *row_idx;   /* [nnz] */
  int *last_row;  /* [n]  index of row nsp in column j */
  int n_des, n_cre;
  int *des_conc, *des_step, *des_nz;  /* destruction terms */
  int *cre_conc, *cre_step, *cre_nz;  /* creation terms */
} zo_jac_pattern;

zo_jac_pattern *zo_jac_pattern_new(const zo_tables *t);
void zo_jac_pattern_free(zo_jac_pattern *p);

/* Jacobian values at y (fy = ydot(y)): reactor_nvector_serial.cpp:610-771
 * (SetupJacobianSparse).  If scale != NULL it receives, per nonzero, the sum
 * of magnitudes of the analytic terms (the natural rounding-error scale). */
int zo_jac_values(zo_reactor *r, const zo_jac_pattern *p, const double *y,
                  const double *fy, double *jac, double *scale);

/* Batched driver over independent (T, P, Y) states, reactor-major arrays.
 * Per state: inverse density from (T,P,Y); y = [Y, T/Tref]; fy = ydot(y);
 * wdot = net production rates at y; jac = Jacobian values at y.
 * kins[nthreads]: one provider per thread (providers are not thread-safe). */
int zo_batch_rates_jac(const zo_tables *t, const zo_jac_pattern *p,
                       const zo_kinetics *kins, int nthreads,
                       int nstates, const double *T, const double *P,
                       const double *Y, double Tref, double min_mass_frac,
                       double step_limiter, double *wdot, double *jac,
                       double *ydot);

/* As zo_batch_rates_jac, also returning rounding scales: wscale = create +
 * destroy per species (the magnitude net = create - destroy cancels from),
 * jscale = sum of magnitudes of the terms of each Jacobian entry (for the
 * forward-difference column: the term magnitudes of both right-hand sides
 * divided by the temperature step).  Serial. */
int zo_batch_rates_jac_scaled(const zo_tables *t, const zo_jac_pattern *p,
                              int nstates, const double *T, const double *P,
                              const double *Y, double Tref, double min_mass_frac,
                              double step_limiter, double *wdot, double *jac,
                              double *wscale, double *jscale);

#ifdef __cplusplus
}
#endif
#endif
