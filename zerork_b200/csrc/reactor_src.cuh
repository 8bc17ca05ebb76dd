// reactor_src.cuh -- reactor terms beyond the closed constant-volume system,
// shared by the CTA (dense) and warp (sparse) integrators:
//   * the constant-pressure reactor (plugin option constant_volume = 0,
//     reactor_constant_pressure_cpu.cpp:71-135): enthalpy and c_p in place
//     of internal energy and c_v, density from the current pressure;
//   * the pressure-rate source DPDT and the energy source E_SRC
//     (reactor_constant_volume_cpu.cpp:64-128 and the constant-pressure
//     file), including the temperature an energy source implies, found by
//     the Newton inversions T(E, Y) and T(H, Y) of
//     src/zerork/mechanism.cpp:477-547.
// Sums over species go through a reduction functor (block or warp sum) that
// hands every thread the same total, so all threads take the same branches.
#pragma once
#include <cuda_runtime.h>

#include "kinetics_dev.cuh"

namespace zrk {

// Sources and initial state of the reactor being integrated.
struct ReactorSrc {
  double dpdt = 0.0;  // pressure rate (Pa/s), ZERORK_FIELD_DPDT
  double esrc = 0.0;  // energy source (J/kg/s), ZERORK_FIELD_E_SRC
  double P0 = 0.0;    // pressure at the start of the call
  double E0 = 0.0;    // mass internal energy (constant volume) or enthalpy
                      // (constant pressure) at the start; set when esrc != 0
                      // or fixT
  bool ysrc = false;  // mass-fraction sources present: the constant-pressure
                      // reactor then keeps its initial density
  bool fixT = false;  // temperature not solved (always_solve_temperature = 0
                      // and a previous temperature delta <= 0,
                      // zerork_reactor_manager.cpp:1107-1113): the rates see
                      // T0 (or the energy source's temperature), Tdot = 0
  double T0 = 0.0;    // temperature at the start of the call
};

// NASA-7 c_p/R and h/RT, the arithmetic of nasa_cp_h_g without g.
__device__ __forceinline__ void nasa_cp_h(const double *__restrict__ c, double T, double *cp,
                                          double *h) {
  const double invT = 1.0 / T;
  const double m0 = T * 0.50000000000000000000;
  const double T2 = T * T, T3 = T * T2, T4 = T * T3;
  const double m1 = T2 * 0.33333333333333333333;
  const double m2 = T3 * 0.25000000000000000000;
  const double m3 = T4 * 0.20000000000000000000;
  const int o = (T < c[0]) ? 1 : 8;
  const double a1 = c[o], a2 = c[o + 1], a3 = c[o + 2], a4 = c[o + 3], a5 = c[o + 4],
               a6 = c[o + 5];
  *cp = a1 + T * (a2 + T * (a3 + T * (a4 + T * a5)));
  *h = a1 + a2 * m0 + a3 * m1 + a4 * m2 + a5 * m3 + a6 * invT;
}

// Mixture mass energy e = sum_k y_k e_k Ru T / W_k with e_k = h_k/RT
// (enthalpy) or h_k/RT - 1 (internal energy), and heat capacity
// cx = sum_k y_k (c_p,k/R - [!cpx]) Ru / W_k (mechanism.cpp:336-434).
// Threads own species k = i0, i0 + stride, ...
template <class Red>
__device__ void mix_energy(const DevMech &m, bool enthalpy, bool cpx, double T, const double *y,
                           bool clamp, double mmf, int i0, int stride, Red red, double &e,
                           double &cx) {
  double pe = 0.0, pc = 0.0;
  for (int k = i0; k < m.nsp; k += stride) {
    double yk = y[k];
    if (clamp) yk = clamp_mass_fraction(yk, mmf);
    double cpR, hRT;
    nasa_cp_h(m.thermo + 16 * k, T, &cpR, &hRT);
    pe += ((enthalpy ? hRT : hRT - 1.0) * (m.ru_inv_mw[k] * T)) * yk;
    pc += ((cpx ? cpR : cpR - 1.0) * m.ru_inv_mw[k]) * yk;
  }
  e = red(pe);
  cx = red(pc);
}

// T(E, Y) (enthalpy = false) or T(H, Y) (enthalpy = true): Newton on the
// mixture energy between 100 K and 5000 K from the guess T_guess, steps
// clipped to +-100 K, stopping below 1e-6 K or when a step no longer changes
// T, at most 400 iterations; linear extrapolation outside the range.  As in
// the reference, both iterations divide by the mixture c_v, and so does the
// extrapolation above 5000 K; only the enthalpy extrapolation below 100 K
// uses c_p.
template <class Red>
__device__ double temp_from_energy(const DevMech &m, bool enthalpy, double E, const double *y,
                                   bool clamp, double mmf, double T_guess, int i0, int stride,
                                   Red red) {
  const double Tmin = 100.0, Tmax = 5000.0;
  double Emin, cmin, Emax, cmax;
  mix_energy(m, enthalpy, enthalpy, Tmin, y, clamp, mmf, i0, stride, red, Emin, cmin);
  mix_energy(m, enthalpy, false, Tmax, y, clamp, mmf, i0, stride, red, Emax, cmax);
  if (E < Emin) return Tmin - (Emin - E) / cmin;
  if (E > Emax) return Tmax - (Emax - E) / cmax;
  double T = T_guess;
  if (T < Tmin || T > Tmax) T = Tmin + (Tmax - Tmin) / (Emax - Emin) * (E - Emin);
  for (int i = 0; i < 400; ++i) {
    double Ei, ci;
    mix_energy(m, enthalpy, false, T, y, clamp, mmf, i0, stride, red, Ei, ci);
    const double dT = fmin(fmax((E - Ei) / ci, -100.0), 100.0);
    if (fabs(dT) < 1.0e-6 || T + dT == T) break;
    T += dT;
  }
  return T;
}

// Temperature and inverse density of one right-hand-side evaluation at time
// t from the start of the call.  T enters as the state's temperature
// (clamped at 1e4 K); v0 is the inverse density at the start.
//   constant pressure: v from P0 + dpdt t unless mass sources are set, then
//                      T from the enthalpy H0 + esrc t when esrc != 0;
//   constant volume:   T from the internal energy E0 + esrc t when esrc != 0,
//                      then v from the pressure of (T, v0) plus dpdt t when
//                      dpdt != 0.
// T_force > 0 replaces the energy-source temperature (the integrator's
// finite difference in that temperature).
template <class Red>
__device__ void source_T_v(const DevMech &m, bool cp, const ReactorSrc &src, double t,
                           const double *y, bool clamp, double mmf, double v0, double T_force,
                           int i0, int stride, Red red, double &T, double &v) {
  v = v0;
  auto mw_mix = [&]() {
    double a = 0.0;
    for (int k = i0; k < m.nsp; k += stride) {
      double yk = y[k];
      if (clamp) yk = clamp_mass_fraction(yk, mmf);
      a += yk * m.inv_mw[k];
    }
    return 1.0 / red(a);
  };
  if (cp) {
    if (!src.ysrc) {
      const double mw = mw_mix();
      v = 1.0 / ((src.P0 + src.dpdt * t) * mw / (kRuD * T));
    }
    if (T_force > 0.0)
      T = T_force;
    else if (src.esrc != 0.0)
      T = temp_from_energy(m, true, src.E0 + src.esrc * t, y, clamp, mmf, T, i0, stride, red);
  } else {
    if (T_force > 0.0)
      T = T_force;
    else if (src.esrc != 0.0)
      T = temp_from_energy(m, false, src.E0 + src.esrc * t, y, clamp, mmf, T, i0, stride, red);
    if (src.dpdt != 0.0) {
      const double mw = mw_mix();
      const double P = kRuD * T / (v0 * mw) + src.dpdt * t;
      v = 1.0 / (P * mw / (kRuD * T));
    }
  }
}

// GetState's temperature at the end time t_end for the end composition y:
// the state's T_state, or, when the temperature was not solved, the
// temperature of the energy E0 + esrc t_end (reactor_constant_volume_cpu.cpp:
// 51-56, reactor_constant_pressure_cpu.cpp:52-57).
template <class Red>
__device__ double end_temperature(const DevMech &m, bool cp, const ReactorSrc &src, double t_end,
                                  const double *y, double T_state, int i0, int stride, Red red) {
  if (!src.fixT) return T_state;
  return temp_from_energy(m, cp, src.E0 + src.esrc * t_end, y, false, 0.0, src.T0, i0, stride, red);
}

// GetState's pressure at the end time t_end for the end state (T, mixture
// molecular weight mw) (reactor_constant_volume_cpu.cpp:59,
// reactor_constant_pressure_cpu.cpp:59-63).
__device__ __forceinline__ double end_pressure(bool cp, const ReactorSrc &src, double t_end,
                                               double T, double mw, double v0) {
  if (cp && !src.ysrc) return src.P0 + src.dpdt * t_end;
  const double P = kRuD * T / (v0 * mw);
  return (cp || src.dpdt == 0.0) ? P : P + src.dpdt * t_end;
}

}  // namespace zrk
