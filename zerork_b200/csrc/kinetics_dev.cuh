// kinetics_dev.cuh -- device helpers shared by the rate and integrator
// kernels: NASA-7 thermo (src/zerork/nasa_poly.cpp:50-172), one reaction's
// two steps (src/zerork/rate_const.cpp:539-582 and perf_net.cpp:190-274),
// and the Jacobian's mass-fraction clamp (reactor_nvector_serial.cpp:629-640).
#pragma once
#include <cuda_runtime.h>

#include "devmech.h"

namespace zrk {

constexpr double kRuD = 8.314462618e3;  // src/zerork/constants.h:10
constexpr double kPatmD = 1.01325e5;    // src/zerork/constants.h:12

// A mechanism table as the kernel reads it: its copy in the CTA's shared
// memory when the kernel staged the hot tables (tab = the copy of the block
// that starts at the global base), the global table itself for tab = null.
// The staged address is formed from the shared-memory pointer, not by
// offsetting the global one: a pointer derived from a kernel parameter may
// be compiled as a global-space access, which a shared address must not
// reach.  With tab a compile-time null the select folds away.
template <class T>
__device__ __forceinline__ const T *rb(const T *p, const char *tab, const unsigned char *gbase) {
  return tab ? reinterpret_cast<const T *>(
                   tab + (reinterpret_cast<const char *>(p) - reinterpret_cast<const char *>(gbase)))
             : p;
}

// NASA-7 polynomials (src/zerork/nasa_poly.cpp:50-172), one species, one T.
__device__ __forceinline__ void nasa_cp_h_g(const double *__restrict__ c, double T, double logT,
                                            double *cp, double *h, double *g) {
  const double invT = 1.0 / T;
  const double m0 = T * 0.50000000000000000000;
  const double T2 = T * T, T3 = T * T2, T4 = T * T3;
  const double m1 = T2 * 0.33333333333333333333;
  const double m2 = T3 * 0.25000000000000000000;
  const double m3 = T4 * 0.20000000000000000000;
  const double g0 = 1.0 - logT;
  const double g1 = T * -0.50000000000000000000;
  const double g2 = T2 * -0.16666666666666666667;
  const double g3 = T3 * -0.08333333333333333333;
  const double g4 = T4 * -0.05000000000000000000;
  const int o = (T < c[0]) ? 1 : 8;
  const double a1 = c[o], a2 = c[o + 1], a3 = c[o + 2], a4 = c[o + 3], a5 = c[o + 4],
               a6 = c[o + 5], a7 = c[o + 6];
  *cp = a1 + T * (a2 + T * (a3 + T * (a4 + T * a5)));
  *h = a1 + a2 * m0 + a3 * m1 + a4 * m2 + a5 * m3 + a6 * invT;
  *g = a1 * g0 + a2 * g1 + a3 * g2 + a4 * g3 + a5 * g4 + a6 * invT - a7;
}

__device__ __forceinline__ double nasa_cp(const double *__restrict__ c, double T) {
  const int o = (T < c[0]) ? 1 : 8;
  return c[o] + T * (c[o + 1] + T * (c[o + 2] + T * (c[o + 3] + T * c[o + 4])));
}

// A PLOG reaction's forward rate coefficient at (T, P): the Arrhenius lines
// of each distinct pressure summed with the sign of their A, the end
// pressures' values outside [p_min, p_max] and logarithmic interpolation
// between the bracketing pressures inside; zero for T or P <= 0 or a
// non-positive bracketing value (src/zerork/plog_reaction.cpp:166-300,
// without extrapolation as rate_const.cpp:1174-1182 builds them).
__device__ __forceinline__ double plog_at(const DevMech &m, int q, double invT, double logT,
                                          const char *tab = nullptr) {
  const int *lp = rb(m.plog_ln_ptr, tab, m.base);
  const double *sg = rb(m.plog_sgn, tab, m.base), *la = rb(m.plog_lnA, tab, m.base), *ln = rb(m.plog_n, tab, m.base),
               *lt = rb(m.plog_Ta, tab, m.base);
  double k = 0.0;
  for (int l = lp[q]; l < lp[q + 1]; ++l) k += sg[l] * exp(la[l] + logT * ln[l] - invT * lt[l]);
  return k;
}

static __device__ __forceinline__ double plog_rate(const DevMech &m, int j, double T, double invT, double logT,
                                         double P, const char *tab = nullptr) {
  const int *pp = rb(m.plog_pt_ptr, tab, m.base);
  const double *pv = rb(m.plog_p, tab, m.base), *lnp = rb(m.plog_lnp, tab, m.base);
  const int q0 = pp[j], q1 = pp[j + 1];
  if (T <= 0.0 || P <= 0.0) return 0.0;
  if (q1 - q0 == 1 || P <= pv[q0]) return plog_at(m, q0, invT, logT, tab);
  if (P >= pv[q1 - 1]) return plog_at(m, q1 - 1, invT, logT, tab);
  int r = q0;
  while (r + 1 < q1 - 1 && !(pv[r] <= P && P < pv[r + 1])) ++r;
  const double k1 = plog_at(m, r, invT, logT, tab);
  if (k1 <= 0.0) return 0.0;
  const double k2 = plog_at(m, r + 1, invT, logT, tab);
  if (k2 <= 0.0) return 0.0;
  const double e = log(k2 / k1) / (lnp[r + 1] - lnp[r]);
  return k1 * pow(P / pv[r], e);
}

// A reaction record read as six independent 16-byte loads: one memory round
// trip instead of a chain of dependent field loads (generic loads: the
// record may sit in a staged shared-memory copy).
__device__ __forceinline__ RxnRec load_rxn(const RxnRec *p) {
  static_assert(sizeof(RxnRec) == 96, "RxnRec layout");
  const int4 *src = reinterpret_cast<const int4 *>(p);
  int4 b[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) b[i] = src[i];
  RxnRec R;
  memcpy(&R, b, sizeof(R));
  return R;
}

// One reaction (both steps) for the V states a thread owns (states
// q + k*GS of the tile): rate constants, third body, falloff, step limiter
// (one scalar for all steps, or one per step when lim_step is given) and
// concentration products.  The V independent chains give the scheduler
// instruction-level parallelism across states.
template <int TS, int V>
__device__ __forceinline__ void reaction_item(const DevMech &m, const RxnRec &R, int q,
                                              const double *__restrict__ sC,
                                              const double *__restrict__ sG, double *sROP,
                                              const double *T, const double *logT,
                                              const double *invT, const double *lprt,
                                              const double *Csum, double lim,
                                              const double *lim_step = nullptr, const char *tab = nullptr) {
  constexpr int GS = TS / V;
  double kf[V], kr[V];
  if (R.flags & kPlog) {  // at the pressure of the concentrations, Csum Ru T (rate_const.cpp:548-567)
#pragma unroll
    for (int k = 0; k < V; ++k) kf[k] = plog_rate(m, R.aux, T[k], invT[k], logT[k], Csum[k] * kRuD * T[k], tab);
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) kf[k] = exp(R.lnA + R.n * logT[k] - R.Ta * invT[k]);
  }
  if (R.flags & kRevArr) {
#pragma unroll
    for (int k = 0; k < V; ++k) kr[k] = exp(R.lnA_r + R.n_r * logT[k] - R.Ta_r * invT[k]);
  } else if (R.flags & kRevKeq) {
    double s[V];
#pragma unroll
    for (int k = 0; k < V; ++k) s[k] = 0.0;
    for (int i = 0; i < R.np; ++i) {
      const double *gp = sG + R.p[i] * TS + q;
#pragma unroll
      for (int k = 0; k < V; ++k) s[k] += gp[k * GS];
    }
    for (int i = 0; i < R.nr; ++i) {
      const double *gr = sG + R.r[i] * TS + q;
#pragma unroll
      for (int k = 0; k < V; ++k) s[k] -= gr[k * GS];
    }
#pragma unroll
    for (int k = 0; k < V; ++k) kr[k] = exp(s[k] - R.lnA_r * lprt[k]) * kf[k];
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) kr[k] = 0.0;
  }
  if (R.flags & kThirdBody) {
    double Cm[V];
#pragma unroll
    for (int k = 0; k < V; ++k) Cm[k] = Csum[k];
    // efficiencies four at a time: the table loads are independent of the
    // sums, which keep the list order
    const int e0 = rb(m.tb_ptr, tab, m.base)[R.aux], e1 = rb(m.tb_ptr, tab, m.base)[R.aux + 1];
    int e = e0;
    for (; e + 3 < e1; e += 4) {
      const double a0 = rb(m.tb_alpha, tab, m.base)[e], a1 = rb(m.tb_alpha, tab, m.base)[e + 1], a2 = rb(m.tb_alpha, tab, m.base)[e + 2],
                   a3 = rb(m.tb_alpha, tab, m.base)[e + 3];
      const double *c0 = sC + rb(m.tb_spc, tab, m.base)[e] * TS + q, *c1 = sC + rb(m.tb_spc, tab, m.base)[e + 1] * TS + q,
                   *c2 = sC + rb(m.tb_spc, tab, m.base)[e + 2] * TS + q, *c3 = sC + rb(m.tb_spc, tab, m.base)[e + 3] * TS + q;
#pragma unroll
      for (int k = 0; k < V; ++k) {
        Cm[k] += c0[k * GS] * a0;
        Cm[k] += c1[k * GS] * a1;
        Cm[k] += c2[k * GS] * a2;
        Cm[k] += c3[k * GS] * a3;
      }
    }
    for (; e < e1; ++e) {
      const double a = rb(m.tb_alpha, tab, m.base)[e];
      const double *cp = sC + rb(m.tb_spc, tab, m.base)[e] * TS + q;
#pragma unroll
      for (int k = 0; k < V; ++k) Cm[k] += cp[k * GS] * a;
    }
#pragma unroll
    for (int k = 0; k < V; ++k) {
      kf[k] *= Cm[k];
      kr[k] *= Cm[k];
    }
  }
  if (R.flags & kFalloff) {
    const int f = R.aux;
    const double *p = rb(m.fo_par, tab, m.base) + 8 * f;
    const int fs = rb(m.fo_spc, tab, m.base)[f];
    const int ty = rb(m.fo_type, tab, m.base)[f];
    double Cm[V];
    if (fs >= 0) {
#pragma unroll
      for (int k = 0; k < V; ++k) Cm[k] = sC[fs * TS + q + k * GS];
    } else {
#pragma unroll
      for (int k = 0; k < V; ++k) Cm[k] = Csum[k];
      const int e0 = rb(m.fo_ptr, tab, m.base)[f], e1 = rb(m.fo_ptr, tab, m.base)[f + 1];
      int e = e0;
      for (; e + 3 < e1; e += 4) {
        const double a0 = rb(m.fo_alpha, tab, m.base)[e], a1 = rb(m.fo_alpha, tab, m.base)[e + 1], a2 = rb(m.fo_alpha, tab, m.base)[e + 2],
                     a3 = rb(m.fo_alpha, tab, m.base)[e + 3];
        const double *c0 = sC + rb(m.fo_spc_eff, tab, m.base)[e] * TS + q, *c1 = sC + rb(m.fo_spc_eff, tab, m.base)[e + 1] * TS + q,
                     *c2 = sC + rb(m.fo_spc_eff, tab, m.base)[e + 2] * TS + q, *c3 = sC + rb(m.fo_spc_eff, tab, m.base)[e + 3] * TS + q;
#pragma unroll
        for (int k = 0; k < V; ++k) {
          Cm[k] += c0[k * GS] * a0;
          Cm[k] += c1[k * GS] * a1;
          Cm[k] += c2[k * GS] * a2;
          Cm[k] += c3[k * GS] * a3;
        }
      }
      for (; e < e1; ++e) {
        const double a = rb(m.fo_alpha, tab, m.base)[e];
        const double *cp = sC + rb(m.fo_spc_eff, tab, m.base)[e] * TS + q;
#pragma unroll
        for (int k = 0; k < V; ++k) Cm[k] += cp[k * GS] * a;
      }
    }
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const double Klow = exp(p[0] + p[1] * logT[k] - p[2] * invT[k]);
      double Pr = Klow * Cm[k] / kf[k];
      if (Pr < 1.0e-300) Pr = 1.0e-300;
      double lPr = log10(Pr);
      double fT = 1.0;
      if (ty == kTroe3 || ty == kTroe4) {
        double Fc = 0.0;
        if (p[4] != 0) Fc += (1.0 - p[3]) * exp(-T[k] / p[4]);
        if (p[5] != 0) Fc += p[3] * exp(-T[k] / p[5]);
        if (ty == kTroe4) Fc += exp(-p[6] * invT[k]);
        if (Fc < 1.0e-300) Fc = 1.0e-300;
        fT = log10(Fc);
        const double nT = 0.75 - 1.27 * fT;
        lPr -= (0.4 + 0.67 * fT);
        lPr = lPr / (nT - 0.14 * lPr);
        lPr *= lPr;
        fT /= (1.0 + lPr);
        fT = exp10(fT);
      } else if (ty == kSRI) {
        const double xp = 1.0 / (1.0 + lPr * lPr);
        fT = p[3] * exp(-p[4] * invT[k]);
        if (p[5] > 0) fT += exp(-T[k] * p[5]);
        fT = pow(fT, xp);
        fT *= p[6];
        fT *= pow(T[k], p[7]);
      }
      const double Pc = fT * Pr / (1.0 + Pr);
      kf[k] *= Pc;
      kr[k] *= Pc;
    }
  }
  if (lim_step) {  // one limit per step (perf_net.cpp:213-224)
    const double lf = lim_step[R.fwd];
    if (0.0 < lf && lf < 1.0e300) {
#pragma unroll
      for (int k = 0; k < V; ++k) kf[k] *= lf / (lf + kf[k]);
    }
    if (R.rev >= 0) {
      const double lr = lim_step[R.rev];
      if (0.0 < lr && lr < 1.0e300) {
#pragma unroll
        for (int k = 0; k < V; ++k) kr[k] *= lr / (lr + kr[k]);
      }
    }
  } else if (0.0 < lim && lim < 1.0e300) {  // the plugin's step_limiter option
#pragma unroll
    for (int k = 0; k < V; ++k) {
      kf[k] *= lim / (lim + kf[k]);
      if (R.rev >= 0) kr[k] *= lim / (lim + kr[k]);
    }
  }
  for (int i = 0; i < R.nr; ++i) {
    const double *cp = sC + R.r[i] * TS + q;
#pragma unroll
    for (int k = 0; k < V; ++k) kf[k] *= cp[k * GS];
  }
#pragma unroll
  for (int k = 0; k < V; ++k) sROP[R.fwd * TS + q + k * GS] = kf[k];
  if (R.rev >= 0) {
    for (int i = 0; i < R.np; ++i) {
      const double *cp = sC + R.p[i] * TS + q;
#pragma unroll
      for (int k = 0; k < V; ++k) kr[k] *= cp[k * GS];
    }
#pragma unroll
    for (int k = 0; k < V; ++k) sROP[R.rev * TS + q + k * GS] = kr[k];
  }
}

__device__ __forceinline__ double clamp_mass_fraction(double y, double mmf) {
  if (fabs(y) < mmf) return (y < 0.0) ? -mmf : mmf;
  return y;
}


}  // namespace zrk
