/*
 * zrk_oracle_bdf.h -- CPU ORACLE integrator (test infrastructure only).
 *
 * The reference integrates each reactor with SUNDIALS CVODE (BDF, Newton,
 * applications/cfd_plugin/solver_cvode.cpp:51-299).  SUNDIALS 5.8.0 is not
 * vendored in the reference (cmake/sundials5.CMakeLists.txt:8) and cannot be
 * fetched here, so this oracle restates a published variable-order BDF
 * instead: the quasi-constant step-size BDF of Shampine & Reichelt, "The
 * MATLAB ODE Suite", SIAM J. Sci. Comput. 18 (1997) (orders 1-5, modified
 * Newton iteration, order/step selection after order+1 equal steps), with
 * CVODE's option semantics from the plugin: rel_tol, abs_tol, max_steps,
 * max_dt, nonlinear_convergence_coeff (solver_cvode.cpp:66-88).  Newton
 * matrices are I - c J with J the reactor Jacobian of zrk_oracle.c
 * (SetupJacobianSparse semantics), factored densely with partial pivoting.
 * End states are therefore compared to the GPU integrator at the integration
 * tolerance, not step by step (CVODE's step sequence is unpinned).
 */
#ifndef ZRK_ORACLE_BDF_H
#define ZRK_ORACLE_BDF_H

#include "zrk_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zo_bdf_opts {
  double rtol, atol, max_dt, nlscoef;
  int max_steps;
  double Tref, min_mass_frac, step_limiter;
  int analytic; /* 1: SetupJacobianSparse values; 0: dense divided differences
                   (the plugin's analytic = 0, reactor_nvector_serial.cpp:360) */
  /* cvode_num_retries and the tolerance adjustments: after a failed attempt
   * the integration restarts from the last accepted state with atol *=
   * retry_atol, rtol *= retry_rtol, at most max_retries attempts in all
   * (solver_cvode.cpp:216-246) */
  int max_retries;
  double retry_atol, retry_rtol;
  /* delta_temperature_ignition: > 0 records the first time T reaches
   * T0 + dT_ign (ReactorNVectorSerial::RootFunction, :774-784), located by
   * linear interpolation between the accepted steps that bracket it */
  double dT_ign;
  /* constant_volume: 1 constant-volume reactor, 0 constant-pressure reactor
   * (zerork_reactor_manager.cpp:85, :913-917) */
  int constant_volume;
  /* stop_after_ignition (solver_cvode.cpp:259-263): with dT_ign > 0 the call
   * ends at the first crossing, its state interpolated linearly between the
   * two accepted steps around it */
  int stop_ign;
  /* abstol_dens (reactor_nvector_serial.cpp:107-119): the absolute tolerance
   * of species k is abs_tol / (rho / W_k * 1e-3), rho the initial density */
  int abstol_dens;
  /* 1: CVODE's per-step failure limits (7 error-test, 10 convergence
   * failures fail the attempt) and its order/step cut after the 3rd
   * error-test failure, as the plugin runs; 0: neither (tight-tolerance
   * reference runs, where the energy inversion's 1e-6 K stop is a noise
   * floor that makes repeated rejections normal) */
  int fail_caps;
} zo_bdf_opts;

typedef struct zo_bdf_stats {
  int nsteps, nrej, nnewt, njac, nlu, nrhs, status; /* status 0 ok, <0 failure */
  int retries;
} zo_bdf_stats;

void zo_bdf_default_opts(zo_bdf_opts *o);

/* Integrate one reactor (constant volume or constant pressure, o->
 * constant_volume) from (T, P, Y) for dt seconds: InitializeState /
 * Integrate / GetState of the cfd_plugin (reactor_constant_volume_cpu.cpp:
 * 15-61, reactor_constant_pressure_cpu.cpp:15-66, zerork_reactor_manager.cpp:
 * 1090-1146), with optional mass-fraction sources y_src [nsp] (or NULL), a
 * pressure rate dpdt (Pa/s) and an energy source e_src (J/kg/s).  fix_T = 1
 * integrates without solving the temperature (the plugin's
 * always_solve_temperature = 0 for a reactor whose previous temperature
 * delta is not positive).  On return T, P, Y hold the end state. */
int zo_reactor_solve(const zo_tables *t, const zo_jac_pattern *p, const zo_kinetics *kin,
                     const zo_bdf_opts *o, double dt, double *T, double *P, double *Y,
                     const double *y_src, double dpdt, double e_src, int fix_T, double *t_ign,
                     zo_bdf_stats *st);

/* Batch over reactors (reactor-major Y [n][nsp]) with nthreads OpenMP
 * threads, one reactor object per thread; stats may be NULL. */
int zo_reactor_solve_batch(const zo_tables *t, const zo_jac_pattern *p, const zo_bdf_opts *o,
                           int nthreads, int n, double dt, double *T, double *P, double *Y,
                           const double *y_src, const double *dpdt, const double *e_src,
                           const int *fix_T, double *t_ign, zo_bdf_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
