// kinetics.cu -- fused FP64 net production rates + sparse analytic Jacobian
// for sm_100a.
//
// One CTA works on a tile of TS independent states at a time.  A "group" of
// TS consecutive threads owns one work item (species, reaction or Jacobian
// column) for all TS states of the tile, so every table read is a warp-uniform
// broadcast and every state read/write is a coalesced TS-wide row of the
// species-major (SoA) arrays  x[item * ld + state].  Intermediate per-state
// vectors (concentrations, g/RT, u/RT, rates of progress) live in a workspace
// of rows of TS doubles, placed in shared memory when it fits and in a global
// scratch slice per CTA otherwise.
//
// Semantics follow the reference operation for operation:
//   * rate constants   : src/zerork/rate_const.cpp:539-582 (Arrhenius :669-687,
//                        Keq :690-731, third body :862-888, falloff :890-1012)
//   * rates            : src/zerork/perf_net.cpp:190-274 (step limiter, ROP,
//                        destruction/creation in ascending step order)
//   * reactor RHS      : applications/cfd_plugin/reactor_constant_volume_cpu.cpp:64-128
//   * Jacobian values  : applications/cfd_plugin/reactor_nvector_serial.cpp:610-771
//                        (clamped analytic part, temperature row, forward-
//                        difference temperature column, dC->dY conversion).
#include <cuda_runtime.h>

#include <cstdio>

#include "devmech.h"
#include "kinetics.h"

namespace zrk {

namespace {

constexpr double kRu = 8.314462618e3;
constexpr double kPatm = 1.01325e5;

enum Scal {
  S_T, S_P, S_YS, S_V, S_TR, S_LOGT, S_INVT, S_LPRT, S_CSUM, S_CV, S_TDOT, S_CVC, S_TDOTC,
  S_YSP, S_MULT, S_CVP, S_TDOTP, kNScal
};

struct Layout {
  int rC, rU, rX, rG, rROP, rPart, rScal, rows;
};

__host__ __device__ inline Layout make_layout(int S, int N, int NG) {
  Layout L;
  L.rC = 0;
  L.rU = S;
  L.rX = 2 * S;
  L.rG = 3 * S;
  L.rROP = 4 * S;
  L.rPart = 4 * S + N;
  L.rScal = L.rPart + 3 * NG;
  L.rows = L.rScal + kNScal;
  return L;
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

// One reaction (both steps) for one state: rate constants, third body,
// falloff, step limiter and concentration products.
template <int TS>
__device__ __forceinline__ void reaction_item(const DevMech &m, const RxnRec &R, int sl,
                                              const double *__restrict__ sC,
                                              const double *__restrict__ sG, double *sROP,
                                              double T, double logT, double invT, double lprt,
                                              double Csum, double lim) {
  double kf = exp(R.lnA + R.n * logT - R.Ta * invT);
  double kr = 0.0;
  if (R.flags & kRevArr) {
    kr = exp(R.lnA_r + R.n_r * logT - R.Ta_r * invT);
  } else if (R.flags & kRevKeq) {
    double s = 0.0;
    for (int k = 0; k < R.np; ++k) s += sG[R.p[k] * TS + sl];
    for (int k = 0; k < R.nr; ++k) s -= sG[R.r[k] * TS + sl];
    kr = exp(s - R.lnA_r * lprt) * kf;
  }
  if (R.flags & kThirdBody) {
    double Cm = Csum;
    for (int e = m.tb_ptr[R.aux]; e < m.tb_ptr[R.aux + 1]; ++e)
      Cm += sC[m.tb_spc[e] * TS + sl] * m.tb_alpha[e];
    kf *= Cm;
    kr *= Cm;
  }
  if (R.flags & kFalloff) {
    const int f = R.aux;
    const double *p = m.fo_par + 8 * f;
    const double Klow = exp(p[0] + p[1] * logT - p[2] * invT);
    double Cm;
    const int fs = m.fo_spc[f];
    if (fs >= 0) {
      Cm = sC[fs * TS + sl];
    } else {
      Cm = Csum;
      for (int e = m.fo_ptr[f]; e < m.fo_ptr[f + 1]; ++e)
        Cm += sC[m.fo_spc_eff[e] * TS + sl] * m.fo_alpha[e];
    }
    double Pr = Klow * Cm / kf;
    if (Pr < 1.0e-300) Pr = 1.0e-300;
    double lPr = log10(Pr);
    double fT = 1.0;
    const int ty = m.fo_type[f];
    if (ty == kTroe3 || ty == kTroe4) {
      double Fc = 0.0;
      if (p[4] != 0) Fc += (1.0 - p[3]) * exp(-T / p[4]);
      if (p[5] != 0) Fc += p[3] * exp(-T / p[5]);
      if (ty == kTroe4) Fc += exp(-p[6] * invT);
      if (Fc < 1.0e-300) Fc = 1.0e-300;
      fT = log10(Fc);
      const double nT = 0.75 - 1.27 * fT;
      lPr -= (0.4 + 0.67 * fT);
      lPr = lPr / (nT - 0.14 * lPr);
      lPr *= lPr;
      fT /= (1.0 + lPr);
      fT = pow(10.0, fT);
    } else if (ty == kSRI) {
      const double xp = 1.0 / (1.0 + lPr * lPr);
      fT = p[3] * exp(-p[4] * invT);
      if (p[5] > 0) fT += exp(-T * p[5]);
      fT = pow(fT, xp);
      fT *= p[6];
      fT *= pow(T, p[7]);
    }
    const double Pc = fT * Pr / (1.0 + Pr);
    kf *= Pc;
    kr *= Pc;
  }
  if (0.0 < lim && lim < 1.0e300) {
    kf *= lim / (lim + kf);
    if (R.rev >= 0) kr *= lim / (lim + kr);
  }
  for (int k = 0; k < R.nr; ++k) kf *= sC[R.r[k] * TS + sl];
  sROP[R.fwd * TS + sl] = kf;
  if (R.rev >= 0) {
    for (int k = 0; k < R.np; ++k) kr *= sC[R.p[k] * TS + sl];
    sROP[R.rev * TS + sl] = kr;
  }
}

__device__ __forceinline__ double clampy(double y, double mmf) {
  if (fabs(y) < mmf) return (y < 0.0) ? -mmf : mmf;
  return y;
}

template <int TS>
__global__ void __launch_bounds__(512, 1) rates_jac_kernel(
    DevMech m, int n, int ld, const double *__restrict__ Tin, const double *__restrict__ Pin,
    const double *__restrict__ Y, double *__restrict__ wdot, double *__restrict__ jac,
    double *__restrict__ ydot, KinParams kp, double *__restrict__ gscratch, int ws_doubles) {
  extern __shared__ double smem_dyn[];
  const int S = m.nsp, N = m.nstep;
  const int NG = blockDim.x / TS;
  const int g = threadIdx.x / TS;
  const int sl = threadIdx.x % TS;
  const Layout L = make_layout(S, N, NG);
  double *ws = gscratch ? gscratch + (size_t)blockIdx.x * ws_doubles : smem_dyn;
  double *sC = ws + L.rC * TS, *sU = ws + L.rU * TS, *sX = ws + L.rX * TS, *sG = ws + L.rG * TS;
  double *sROP = ws + L.rROP * TS, *sPart = ws + L.rPart * TS, *sc = ws + L.rScal * TS;
#define SCAL(k) sc[(k) * TS + sl]
#define PART(a, grp) sPart[((a) * NG + (grp)) * TS + sl]
  const int ntiles = (n + TS - 1) / TS;
  const double dummy_y = 1.0 / S;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int st = tile * TS + sl;
    const bool valid = st < n;
    // ---- per-state inputs and mixture molecular weight
    double pa = 0.0;
    for (int s = g; s < S; s += NG) {
      const double y = valid ? Y[(size_t)s * ld + st] : dummy_y;
      pa += y * m.inv_mw[s];
    }
    PART(0, g) = pa;
    if (g == 0) {
      const double T = valid ? Tin[st] : 1000.0;
      const double P = valid ? Pin[st] : kPatm;
      SCAL(S_T) = T;
      SCAL(S_P) = P;
      SCAL(S_YS) = T / kp.Tref;
    }
    __syncthreads();
    if (g == 0) {
      double sum = 0.0;
      for (int q = 0; q < NG; ++q) sum += PART(0, q);
      const double T = SCAL(S_T);
      const double mwmix = 1.0 / sum;
      const double rho = SCAL(S_P) * mwmix / (kRu * T);
      SCAL(S_V) = 1.0 / rho;
      double Tr = SCAL(S_YS) * kp.Tref;
      if (Tr > 1.0e4) Tr = 1.0e4;
      SCAL(S_TR) = Tr;
      SCAL(S_LOGT) = log(Tr);
      SCAL(S_INVT) = 1.0 / Tr;
      SCAL(S_LPRT) = log(kPatm / (kRu * Tr));
    }
    __syncthreads();
    // ---- species pass at T: C, g/RT, u/RT, partial sums
    {
      const double v = SCAL(S_V), dens = 1.0 / v, Tr = SCAL(S_TR), logT = SCAL(S_LOGT);
      double pc = 0.0, pcv = 0.0;
      int need = 0;
      for (int s = g; s < S; s += NG) {
        const double y = valid ? Y[(size_t)s * ld + st] : dummy_y;
        const double c = dens * m.inv_mw[s] * y;
        sC[s * TS + sl] = c;
        double cp, h, gg;
        nasa_cp_h_g(m.thermo + 16 * s, Tr, logT, &cp, &h, &gg);
        sG[s * TS + sl] = gg;
        sU[s * TS + sl] = h - 1.0;
        const double cvs = (cp - 1.0) * m.ru_inv_mw[s];
        pc += c;
        pcv += cvs * y;
        need |= (fabs(y) < kp.mmf);
      }
      PART(0, g) = pc;
      PART(1, g) = pcv;
      need = __syncthreads_or(need);
      if (g == 0) {
        double cs = 0.0, cv = 0.0;
        for (int q = 0; q < NG; ++q) {
          cs += PART(0, q);
          cv += PART(1, q);
        }
        SCAL(S_CSUM) = cs;
        SCAL(S_CV) = cv;
      }
      __syncthreads();
      // ---- reactions at T
      {
        const double lprt = SCAL(S_LPRT), invT = SCAL(S_INVT), Csum = SCAL(S_CSUM);
        for (int r = g; r < m.nrxn; r += NG)
          reaction_item<TS>(m, m.rxn[r], sl, sC, sG, sROP, Tr, logT, invT, lprt, Csum, kp.lim);
      }
      __syncthreads();
      // ---- net production rates, energy sum
      double pe = 0.0;
      for (int s = g; s < S; s += NG) {
        double des = 0.0, cre = 0.0;
        for (int k = m.sd_ptr[s]; k < m.sd_ptr[s + 1]; ++k) des += sROP[m.sd_step[k] * TS + sl];
        for (int k = m.sc_ptr[s]; k < m.sc_ptr[s + 1]; ++k) cre += sROP[m.sc_step[k] * TS + sl];
        const double net = cre - des;
        if (valid) {
          wdot[(size_t)s * ld + st] = net;
          if (ydot) ydot[(size_t)s * ld + st] = net * m.mw[s] * v;
        }
        pe += sU[s * TS + sl] * net * v;
      }
      PART(0, g) = pe;
      __syncthreads();
      if (g == 0) {
        double es = 0.0;
        for (int q = 0; q < NG; ++q) es += PART(0, q);
        const double Td = -es * kRu * SCAL(S_YS) / SCAL(S_CV) + 0.0;
        SCAL(S_TDOT) = Td;
        SCAL(S_TDOTC) = Td;
        SCAL(S_CVC) = SCAL(S_CV);
        if (valid && ydot) ydot[(size_t)S * ld + st] = Td;
      }
      __syncthreads();
      if (jac == nullptr) continue;
      // ---- clamped state (reactor_nvector_serial.cpp:629-640), only if needed
      if (need) {
        double pcv2 = 0.0;
        for (int s = g; s < S; s += NG) {
          const double y = valid ? Y[(size_t)s * ld + st] : dummy_y;
          const double yc = clampy(y, kp.mmf);
          sX[s * TS + sl] = dens * m.inv_mw[s] * yc;
          const double cvs = (nasa_cp(m.thermo + 16 * s, Tr) - 1.0) * m.ru_inv_mw[s];
          pcv2 += cvs * yc;
        }
        PART(1, g) = pcv2;
        double pc2 = 0.0;
        for (int s = g; s < S; s += NG) pc2 += sX[s * TS + sl];
        PART(0, g) = pc2;
        __syncthreads();
        if (g == 0) {
          double cs = 0.0, cv = 0.0;
          for (int q = 0; q < NG; ++q) {
            cs += PART(0, q);
            cv += PART(1, q);
          }
          SCAL(S_CSUM) = cs;
          SCAL(S_CVC) = cv;
        }
        __syncthreads();
        {
          const double lprt = SCAL(S_LPRT), invT = SCAL(S_INVT), Csum = SCAL(S_CSUM);
          for (int r = g; r < m.nrxn; r += NG)
            reaction_item<TS>(m, m.rxn[r], sl, sX, sG, sROP, Tr, logT, invT, lprt, Csum, kp.lim);
        }
        __syncthreads();
        double pe2 = 0.0;
        for (int s = g; s < S; s += NG) {
          double des = 0.0, cre = 0.0;
          for (int k = m.sd_ptr[s]; k < m.sd_ptr[s + 1]; ++k) des += sROP[m.sd_step[k] * TS + sl];
          for (int k = m.sc_ptr[s]; k < m.sc_ptr[s + 1]; ++k) cre += sROP[m.sc_step[k] * TS + sl];
          pe2 += sU[s * TS + sl] * (cre - des) * v;
        }
        PART(0, g) = pe2;
        __syncthreads();
        if (g == 0) {
          double es = 0.0;
          for (int q = 0; q < NG; ++q) es += PART(0, q);
          SCAL(S_TDOTC) = -es * kRu * SCAL(S_YS) / SCAL(S_CVC) + 0.0;
        }
        __syncthreads();
      }
      // ---- analytic Jacobian columns + temperature row
      {
        const double RuTemp = kRu * SCAL(S_YS);
        const double TdC = SCAL(S_TDOTC);
        const double multFact = -1.0 / SCAL(S_CVC);
        for (int j = g; j < S; j += NG) {
          const double y = valid ? Y[(size_t)j * ld + st] : dummy_y;
          const double t2 = m.mw[j] / clampy(y, kp.mmf) * v;
          const int k0 = m.col_ptr[j], k1 = m.col_ptr[j + 1] - 1;
          const double cvj = (nasa_cp(m.thermo + 16 * j, Tr) - 1.0) * m.ru_inv_mw[j];
          const double wcol = m.inv_mw[j];
          double trow = 0.0;
          for (int k = k0; k < k1; ++k) {
            const int row = m.row_idx[k];
            double val = 0.0;
            for (int q = m.nzd_ptr[k]; q < m.nzd_ptr[k + 1]; ++q) val -= sROP[m.nzd_step[q] * TS + sl] * t2;
            for (int q = m.nzc_ptr[k]; q < m.nzc_ptr[k + 1]; ++q) val += sROP[m.nzc_step[q] * TS + sl] * t2;
            trow += val * sU[row * TS + sl];
            if (valid) jac[(size_t)k * ld + st] = val * (m.mw[row] * wcol);
          }
          double tr = trow * RuTemp;
          tr += TdC * cvj * m.mw[j];
          tr *= wcol * multFact;
          if (valid) jac[(size_t)k1 * ld + st] = tr;
        }
      }
      __syncthreads();
    }
    if (jac == nullptr) continue;
    // ---- temperature-perturbed RHS for the forward-difference column
    if (g == 0) {
      const double yS = SCAL(S_YS);
      const double ySp = yS + yS * kp.sqrt_ur;
      const double dT = ySp - yS;
      SCAL(S_YSP) = ySp;
      SCAL(S_MULT) = 1.0 / dT;
      double Tp = ySp * kp.Tref;
      if (Tp > 1.0e4) Tp = 1.0e4;
      SCAL(S_TR) = Tp;
      SCAL(S_LOGT) = log(Tp);
      SCAL(S_INVT) = 1.0 / Tp;
      SCAL(S_LPRT) = log(kPatm / (kRu * Tp));
    }
    __syncthreads();
    {
      const double Tp = SCAL(S_TR), logTp = SCAL(S_LOGT), v = SCAL(S_V);
      double pcv = 0.0, pc = 0.0;
      for (int s = g; s < S; s += NG) {
        const double y = valid ? Y[(size_t)s * ld + st] : dummy_y;
        double cp, h, gg;
        nasa_cp_h_g(m.thermo + 16 * s, Tp, logTp, &cp, &h, &gg);
        sG[s * TS + sl] = gg;
        sU[s * TS + sl] = h - 1.0;
        pcv += ((cp - 1.0) * m.ru_inv_mw[s]) * y;
        pc += sC[s * TS + sl];
      }
      PART(0, g) = pc;
      PART(1, g) = pcv;
      __syncthreads();
      if (g == 0) {
        double cs = 0.0, cv = 0.0;
        for (int q = 0; q < NG; ++q) {
          cs += PART(0, q);
          cv += PART(1, q);
        }
        SCAL(S_CSUM) = cs;
        SCAL(S_CVP) = cv;
      }
      __syncthreads();
      {
        const double lprt = SCAL(S_LPRT), invT = SCAL(S_INVT), Csum = SCAL(S_CSUM);
        for (int r = g; r < m.nrxn; r += NG)
          reaction_item<TS>(m, m.rxn[r], sl, sC, sG, sROP, Tp, logTp, invT, lprt, Csum, kp.lim);
      }
      __syncthreads();
      double pe = 0.0;
      for (int s = g; s < S; s += NG) {
        double des = 0.0, cre = 0.0;
        for (int k = m.sd_ptr[s]; k < m.sd_ptr[s + 1]; ++k) des += sROP[m.sd_step[k] * TS + sl];
        for (int k = m.sc_ptr[s]; k < m.sc_ptr[s + 1]; ++k) cre += sROP[m.sc_step[k] * TS + sl];
        const double net = cre - des;
        sX[s * TS + sl] = net;
        pe += sU[s * TS + sl] * net * v;
      }
      PART(0, g) = pe;
      __syncthreads();
      if (g == 0) {
        double es = 0.0;
        for (int q = 0; q < NG; ++q) es += PART(0, q);
        SCAL(S_TDOTP) = -es * kRu * SCAL(S_YSP) / SCAL(S_CVP) + 0.0;
      }
      __syncthreads();
      const double mult = SCAL(S_MULT);
      const int k0 = m.col_ptr[S], k1 = m.col_ptr[S + 1];
      for (int k = k0 + g; k < k1; k += NG) {
        const int row = m.row_idx[k];
        double d;
        if (row < S) {
          const double f1 = sX[row * TS + sl] * m.mw[row] * v;
          const double f0 = (valid ? wdot[(size_t)row * ld + st] : 0.0) * m.mw[row] * v;
          d = (f1 - f0) * mult;
        } else {
          d = (SCAL(S_TDOTP) - SCAL(S_TDOT)) * mult;
        }
        if (valid) jac[(size_t)k * ld + st] = d;
      }
      __syncthreads();
    }
  }
#undef SCAL
#undef PART
}

template <int TS>
cudaError_t launch_ts(const DevMech &m, const RatesJacArgs &a, const KinParams &kp,
                      const LaunchCfg &cfg, cudaStream_t stream) {
  const int threads = cfg.warps * 32;
  const int NG = threads / TS;
  const Layout L = make_layout(m.nsp, m.nstep, NG);
  const size_t ws_bytes = (size_t)L.rows * TS * sizeof(double);
  const int ntiles = (a.n + TS - 1) / TS;
  if (ntiles == 0) return cudaSuccess;
  if (!cfg.global_ws) {
    cudaError_t e = cudaFuncSetAttribute(rates_jac_kernel<TS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ws_bytes);
    if (e != cudaSuccess) return e;
    rates_jac_kernel<TS><<<ntiles, threads, ws_bytes, stream>>>(
        m, a.n, a.ld, a.T, a.P, a.Y, a.wdot, a.jac, a.ydot, kp, nullptr, 0);
  } else {
    int grid = cfg.grid > 0 ? cfg.grid : ntiles;
    if (grid > ntiles) grid = ntiles;
    if ((size_t)grid * ws_bytes > a.scratch_bytes) return cudaErrorInvalidValue;
    rates_jac_kernel<TS><<<grid, threads, 0, stream>>>(m, a.n, a.ld, a.T, a.P, a.Y, a.wdot, a.jac,
                                                      a.ydot, kp, a.scratch,
                                                      (int)(ws_bytes / sizeof(double)));
  }
  return cudaGetLastError();
}

}  // namespace

size_t rates_jac_ws_bytes(const DevMech &m, const LaunchCfg &cfg) {
  const int NG = cfg.warps * 32 / cfg.ts;
  const Layout L = make_layout(m.nsp, m.nstep, NG);
  return (size_t)L.rows * cfg.ts * sizeof(double);
}

cudaError_t launch_rates_jac(const DevMech &m, const RatesJacArgs &a, const KinParams &kp,
                             const LaunchCfg &cfg, cudaStream_t stream) {
  switch (cfg.ts) {
    case 8: return launch_ts<8>(m, a, kp, cfg, stream);
    case 16: return launch_ts<16>(m, a, kp, cfg, stream);
    case 32: return launch_ts<32>(m, a, kp, cfg, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace zrk
