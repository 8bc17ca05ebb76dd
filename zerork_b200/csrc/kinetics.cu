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

#include <algorithm>
#include <cstdio>

#include "devmech.h"
#include "kinetics.h"
#include "kinetics_dev.cuh"

namespace zrk {

namespace {

constexpr double kRu = kRuD;
constexpr double kPatm = kPatmD;

struct Layout {
  int rC, rU, rROP, rG, rPart, rStash, rows;
};

// Workspace rows of TS doubles: concentrations, u/RT (later the perturbed
// net rates), rates of progress, g/RT, two buffers of per-warp partial sums
// (NW = warps) and two rows that keep the temperature derivative and heat
// capacity of the clamped state through the Jacobian phase.  The g/RT and
// partial rows are contiguous: in the Jacobian phase they hold the
// per-(group, column) temperature-row partials.  Kept small so the shared
// memory carve-out leaves L1 room for the mechanism tables.
__host__ __device__ inline Layout make_layout(int S, int N, int NW) {
  Layout L;
  L.rC = 0;
  L.rU = S;
  L.rROP = 2 * S;
  L.rG = 2 * S + N;
  L.rPart = 3 * S + N;
  L.rStash = L.rPart + 2 * NW;
  L.rows = L.rStash + 2;
  return L;
}

// Sum over the groups of a warp (lanes q, q+GS, ...) with shuffles; lanes
// q < GS of each warp then hold the warp's partial for their states.
template <int GS>
__device__ __forceinline__ double warp_group_sum(double v) {
#pragma unroll
  for (int o = GS; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Gather-sum of rates of progress over an index list, V states.
template <int TS, int V>
__device__ __forceinline__ void gather_rop(const double *__restrict__ sROP, const int *__restrict__ list,
                                           int b, int e, int q, double *acc) {
  constexpr int GS = TS / V;
  for (int i = b; i < e; ++i) {
    const double *rp = sROP + list[i] * TS + q;
#pragma unroll
    for (int k = 0; k < V; ++k) acc[k] += rp[k * GS];
  }
}

template <int TS, int V, int MAXT, bool STAGE, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) rates_jac_kernel(
    DevMech m, int n, int ld, const double *__restrict__ Tin, const double *__restrict__ Pin,
    const double *__restrict__ Y, double *__restrict__ wdot, double *__restrict__ jac,
    double *__restrict__ ydot, KinParams kp, double *__restrict__ gscratch, int ws_doubles,
    int stage_bytes) {
  constexpr int GS = TS / V;
  extern __shared__ double smem_dyn[];
  const int S = m.nsp, N = m.nstep;
  const int NW = blockDim.x >> 5;
  const int NG = blockDim.x / GS;
  const int g = threadIdx.x / GS;
  const int q = threadIdx.x % GS;
  const int w = threadIdx.x >> 5;
  const bool wlead = (threadIdx.x & 31) < GS;  // holds the warp partial
  const Layout L = make_layout(S, N, NW);
  double *ws = gscratch ? gscratch + (size_t)blockIdx.x * ws_doubles : smem_dyn;
  // STAGE: the mechanism's hot tables (stage_bytes of them) copied into
  // shared memory after the workspace; every table read below goes to the
  // copy (tab) instead of global memory
  const char *tab = nullptr;
  if constexpr (STAGE) {
    int4 *dst = reinterpret_cast<int4 *>(smem_dyn + (gscratch ? 0 : ws_doubles));
    const int4 *src = reinterpret_cast<const int4 *>(m.base);
    for (int i = threadIdx.x; i < stage_bytes / 16; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    tab = reinterpret_cast<const char *>(dst);
  }
#define TB(f) rb(m.f, tab, m.base)
  double *sC = ws + L.rC * TS, *sU = ws + L.rU * TS, *sG = ws + L.rG * TS;
  double *sROP = ws + L.rROP * TS, *sPart = ws + L.rPart * TS, *sStash = ws + L.rStash * TS;
#define PT(a, ww, k) sPart[((a) * NW + (ww)) * TS + q + (k) * GS]
#define FORV _Pragma("unroll") for (int k = 0; k < V; ++k)
// Items of a cost-sorted work list in snake order: round r gives group g the
// item at r*NG + g (r even) or r*NG + NG-1-g (r odd), so the costliest items
// spread over the groups and every group's total is close to the mean.
#define SNAKE(var, list, count)                                      \
  for (int snake_r = 0, var = 0; snake_r * NG < (count); ++snake_r)  \
    if (const int snake_p = snake_r * NG + ((snake_r & 1) ? NG - 1 - g : g); \
        snake_p < (count) && ((var = (list)[snake_p]), true))
// All reactions: the cost-sorted records (devmech.h rxn_by_cost) in snake
// order over the groups.
#define RXN_PASS(CONC, CSUM)                                                          \
  for (int rr_ = 0; rr_ * NG < m.nrxn; ++rr_) {                                      \
    const int rp_ = rr_ * NG + ((rr_ & 1) ? NG - 1 - g : g);                         \
    if (rp_ < m.nrxn)                                                                \
      reaction_item<TS, V>(m, load_rxn(TB(rxn_by_cost) + rp_), q, CONC, sG, sROP, Tr, logT, invT, \
                           lprt, CSUM, kp.lim, nullptr, tab);                                      \
  }
  const int ntiles = (n + TS - 1) / TS;
  const double dummy_y = 1.0 / S;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int st[V];
    bool valid[V];
    FORV {
      st[k] = tile * TS + q + k * GS;
      valid[k] = st[k] < n;
    }
    auto yload = [&](int s, int k) -> double {
      return valid[k] ? Y[(size_t)s * ld + st[k]] : dummy_y;
    };
    // ---- mixture molecular weight partials
    {
      double pa[V];
      FORV pa[k] = 0.0;
      for (int s = g; s < S; s += NG) {
        const double iw = TB(inv_mw)[s];
        FORV pa[k] += yload(s, k) * iw;
      }
      FORV pa[k] = warp_group_sum<GS>(pa[k]);
      if (wlead) FORV PT(0, w, k) = pa[k];
    }
    __syncthreads();
    // every thread reduces the warp partials of its own states (same order
    // everywhere, so the values agree) instead of a barrier-fenced one-group
    // phase
    double v[V], Tr[V], logT[V], invT[V], lprt[V], Csum[V], yS[V], cv[V], cvc[V];
    FORV {
      double sum = 0.0;
      for (int ww = 0; ww < NW; ++ww) sum += PT(0, ww, k);
      const double T = valid[k] ? Tin[st[k]] : 1000.0;
      const double P = valid[k] ? Pin[st[k]] : kPatm;
      yS[k] = T / kp.Tref;
      const double mwmix = 1.0 / sum;
      const double rho = P * mwmix / (kRu * T);
      v[k] = 1.0 / rho;
      double t = yS[k] * kp.Tref;
      if (t > 1.0e4) t = 1.0e4;
      Tr[k] = t;
      logT[k] = log(t);
      invT[k] = 1.0 / t;
      lprt[k] = log(kPatm / (kRu * t));
    }
    __syncthreads();  // the species pass reuses the partial rows
    // ---- species pass at T: C, g/RT, u/RT, partial sums
    int need = 0;
    {
      double pc[V], pcv[V];
      FORV pc[k] = pcv[k] = 0.0;
      for (int s = g; s < S; s += NG) {
        const double *th = TB(thermo) + 16 * s;
        const double iw = TB(inv_mw)[s], riw = TB(ru_inv_mw)[s];
        FORV {
          const double y = yload(s, k);
          const double c = (1.0 / v[k]) * iw * y;
          sC[s * TS + q + k * GS] = c;
          double cp, h, gg;
          nasa_cp_h_g(th, Tr[k], logT[k], &cp, &h, &gg);
          sG[s * TS + q + k * GS] = gg;
          sU[s * TS + q + k * GS] = h - 1.0;
          pc[k] += c;
          pcv[k] += ((cp - 1.0) * riw) * y;
          need |= (fabs(y) < kp.mmf);
        }
      }
      FORV {
        pc[k] = warp_group_sum<GS>(pc[k]);
        pcv[k] = warp_group_sum<GS>(pcv[k]);
      }
      if (wlead) FORV {
        PT(0, w, k) = pc[k];
        PT(1, w, k) = pcv[k];
      }
    }
    need = __syncthreads_or(need);
    FORV {
      double cs = 0.0, c2 = 0.0;
      for (int ww = 0; ww < NW; ++ww) {
        cs += PT(0, ww, k);
        c2 += PT(1, ww, k);
      }
      Csum[k] = cs;
      cv[k] = c2;
      cvc[k] = c2;
    }
    // ---- reactions at T
    RXN_PASS(sC, Csum)
    __syncthreads();
    // ---- net production rates, energy partial
    {
      double pe[V];
      FORV pe[k] = 0.0;
      SNAKE(s, TB(spc_order), S) {
        double des[V], cre[V];
        FORV des[k] = cre[k] = 0.0;
        gather_rop<TS, V>(sROP, TB(sd_step), TB(sd_ptr)[s], TB(sd_ptr)[s + 1], q, des);
        gather_rop<TS, V>(sROP, TB(sc_step), TB(sc_ptr)[s], TB(sc_ptr)[s + 1], q, cre);
        const double mws = TB(mw)[s];
        FORV {
          const double net = cre[k] - des[k];
          if (valid[k]) {
            wdot[(size_t)s * ld + st[k]] = net;
            if (ydot) ydot[(size_t)s * ld + st[k]] = net * mws * v[k];
          }
          pe[k] += sU[s * TS + q + k * GS] * net * v[k];
        }
      }
      FORV pe[k] = warp_group_sum<GS>(pe[k]);
      if (wlead) FORV PT(0, w, k) = pe[k];
    }
    __syncthreads();
    double td[V], tdc[V];
    FORV {
      double es = 0.0;
      for (int ww = 0; ww < NW; ++ww) es += PT(0, ww, k);
      td[k] = -es * kRu * yS[k] / cv[k] + 0.0;
      tdc[k] = td[k];
      if (g == 0 && valid[k] && ydot) ydot[(size_t)S * ld + st[k]] = td[k];
    }
    if (jac == nullptr) {
      __syncthreads();  // the next tile reuses the workspace
      continue;
    }
    // ---- clamped state (reactor_nvector_serial.cpp:629-640), only if needed:
    // the clamped concentrations take the C rows for this pass and the
    // unclamped ones are written back after it
    if (need) {
      __syncthreads();  // the energy partials above may still be read
      {
        double pc[V], pcv[V];
        FORV pc[k] = pcv[k] = 0.0;
        for (int s = g; s < S; s += NG) {
          const double *th = TB(thermo) + 16 * s;
          const double iw = TB(inv_mw)[s], riw = TB(ru_inv_mw)[s];
          FORV {
            const double yc = clamp_mass_fraction(yload(s, k), kp.mmf);
            const double c = (1.0 / v[k]) * iw * yc;
            sC[s * TS + q + k * GS] = c;
            pc[k] += c;
            pcv[k] += ((nasa_cp(th, Tr[k]) - 1.0) * riw) * yc;
          }
        }
        FORV {
          pc[k] = warp_group_sum<GS>(pc[k]);
          pcv[k] = warp_group_sum<GS>(pcv[k]);
        }
        if (wlead) FORV {
          PT(0, w, k) = pc[k];
          PT(1, w, k) = pcv[k];
        }
      }
      __syncthreads();
      {
        double Cc[V];
        FORV {
          double cs = 0.0, c2 = 0.0;
          for (int ww = 0; ww < NW; ++ww) {
            cs += PT(0, ww, k);
            c2 += PT(1, ww, k);
          }
          Cc[k] = cs;
          cvc[k] = c2;
        }
        RXN_PASS(sC, Cc)
      }
      __syncthreads();  // also fences the reads of PT(0), PT(1) above
      {
        double pe[V];
        FORV pe[k] = 0.0;
        SNAKE(s, TB(spc_order), S) {
          double des[V], cre[V];
          FORV des[k] = cre[k] = 0.0;
          gather_rop<TS, V>(sROP, TB(sd_step), TB(sd_ptr)[s], TB(sd_ptr)[s + 1], q, des);
          gather_rop<TS, V>(sROP, TB(sc_step), TB(sc_ptr)[s], TB(sc_ptr)[s + 1], q, cre);
          FORV pe[k] += sU[s * TS + q + k * GS] * (cre[k] - des[k]) * v[k];
        }
        FORV pe[k] = warp_group_sum<GS>(pe[k]);
        if (wlead) FORV PT(0, w, k) = pe[k];
        for (int s = g; s < S; s += NG) {  // the unclamped concentrations again
          const double iw = TB(inv_mw)[s];
          FORV sC[s * TS + q + k * GS] = (1.0 / v[k]) * iw * yload(s, k);
        }
      }
      __syncthreads();
      FORV {
        double es = 0.0;
        for (int ww = 0; ww < NW; ++ww) es += PT(0, ww, k);
        tdc[k] = -es * kRu * yS[k] / cvc[k] + 0.0;
      }
    }
    // ---- analytic Jacobian: the species-column entries (the flat item list of
    // devmech.h) in equal work shares over the groups, the temperature row of
    // each column from per-(group, column) partial sums kept in the g/RT and
    // partial rows (free in this phase: S + NGj - 1 <= S + 2 NW slots of TS
    // doubles)
    __syncthreads();  // the energy partials are read before the slots reuse them
    {
      int NGj = NG < S + 1 ? NG : S + 1;
      if (NGj > 2 * NW + 1) NGj = 2 * NW + 1;
      const int total = TB(jcost)[m.nj];
      double *sTP = sG;
      auto group_of = [&](int f) { return (int)(((long long)TB(jcost)[f] * NGj) / total); };
      // the temperature derivative and heat capacity of the (clamped) state
      // wait in partial rows for the temperature-row pass (fewer live registers)
      if (g == 0) FORV {
        sStash[q + k * GS] = tdc[k];
        sStash[TS + q + k * GS] = cvc[k];
      }
      if (g < NGj) {
        auto first_of = [&](int gg) {  // first item f with group_of(f) >= gg
          const long long thr = (long long)gg * total;
          int lo = 0, hi = m.nj;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((long long)TB(jcost)[mid] * NGj >= thr) hi = mid;
            else lo = mid + 1;
          }
          return lo;
        };
        const int f0 = first_of(g), f1 = first_of(g + 1);
        if (f0 < f1) {
          int j = 0, hi = S;  // the column holding f0: jf_ptr[j] <= f0 < jf_ptr[j+1]
          while (j < hi) {
            const int mid = (j + hi + 1) >> 1;
            if (TB(jf_ptr)[mid] <= f0) j = mid;
            else hi = mid - 1;
          }
          int jend = TB(jf_ptr)[j + 1];
          int t = TB(jt_ptr)[f0];
          double t2[V], trow[V], wcol = TB(inv_mw)[j];
          FORV {
            t2[k] = TB(mw)[j] / clamp_mass_fraction(yload(j, k), kp.mmf) * v[k];
            trow[k] = 0.0;
          }
          int2 wn = TB(jw)[f0];
          for (int f = f0; f < f1; ++f) {
            const int2 w = wn;
            if (f + 1 < f1) wn = TB(jw)[f + 1];  // the next item's record in flight during this one
            while (f == jend) {  // column j ends inside this share
              FORV sTP[(j + g) * TS + q + k * GS] = trow[k];
              ++j;
              jend = TB(jf_ptr)[j + 1];
              wcol = TB(inv_mw)[j];
              FORV {
                t2[k] = TB(mw)[j] / clamp_mass_fraction(yload(j, k), kp.mmf) * v[k];
                trow[k] = 0.0;
              }
            }
            const int row = w.x, nd = w.y & 0xffff, nc = w.y >> 16;
            double des[V], cre[V];
            FORV des[k] = cre[k] = 0.0;
            for (int e = 0; e < nd; ++e) {
              const double *rp = sROP + TB(jt)[t + e] * TS + q;
              FORV des[k] += rp[k * GS];
            }
            t += nd;
            for (int e = 0; e < nc; ++e) {
              const double *rp = sROP + TB(jt)[t + e] * TS + q;
              FORV cre[k] += rp[k * GS];
            }
            t += nc;
            const double conv = TB(mw)[row] * wcol;
            FORV {
              // destruction terms first, then creation (SetupJacobianSparse order)
              const double val = (0.0 - des[k] * t2[k]) + cre[k] * t2[k];
              trow[k] += val * sU[row * TS + q + k * GS];
              if (valid[k]) jac[(size_t)(f + j) * ld + st[k]] = val * conv;
            }
          }
          FORV sTP[(j + g) * TS + q + k * GS] = trow[k];
        } else if (f0 < m.nj) {
          // an empty share inside a column (one item's work spans several
          // shares): its slot of that column holds a zero partial
          int j = 0, hi = S;
          while (j < hi) {
            const int mid = (j + hi + 1) >> 1;
            if (TB(jf_ptr)[mid] <= f0) j = mid;
            else hi = mid - 1;
          }
          FORV sTP[(j + g) * TS + q + k * GS] = 0.0;
        }
      }
      __syncthreads();
      // temperature row of column j: the partials of groups group_of(first
      // item) .. group_of(last item), in group order
      for (int j = g; j < S; j += NG) {
        const int g0 = group_of(TB(jf_ptr)[j]), g1 = group_of(TB(jf_ptr)[j + 1] - 1);
        double tp[V];
        FORV tp[k] = 0.0;
#pragma unroll 1
        for (int gg = g0; gg <= g1; ++gg) {
          const double *pp = sTP + (j + gg) * TS + q;
          FORV tp[k] += pp[k * GS];
        }
        const double *th = TB(thermo) + 16 * j;
        const size_t kk = (size_t)(TB(jf_ptr)[j + 1] + j) * ld;
        FORV {
          double Tk = yS[k] * kp.Tref;  // the clamped temperature of this state
          if (Tk > 1.0e4) Tk = 1.0e4;
          const double cvj = (nasa_cp(th, Tk) - 1.0) * TB(ru_inv_mw)[j];
          double tr = tp[k] * (kRu * yS[k]);
          tr += sStash[q + k * GS] * cvj * TB(mw)[j];
          tr *= TB(inv_mw)[j] * (-1.0 / sStash[TS + q + k * GS]);
          if (valid[k]) jac[kk + st[k]] = tr;
        }
      }
    }
    __syncthreads();
    // ---- temperature-perturbed RHS for the forward-difference column
    double ysp[V], mult[V];
    FORV {
      ysp[k] = yS[k] + yS[k] * kp.sqrt_ur;
      mult[k] = 1.0 / (ysp[k] - yS[k]);
      double Tp = ysp[k] * kp.Tref;
      if (Tp > 1.0e4) Tp = 1.0e4;
      Tr[k] = Tp;
      logT[k] = log(Tp);
      invT[k] = 1.0 / Tp;
      lprt[k] = log(kPatm / (kRu * Tp));
    }
    {
      double pcv[V];
      FORV pcv[k] = 0.0;
      for (int s = g; s < S; s += NG) {
        const double *th = TB(thermo) + 16 * s;
        const double riw = TB(ru_inv_mw)[s];
        FORV {
          double cp, h, gg;
          nasa_cp_h_g(th, Tr[k], logT[k], &cp, &h, &gg);
          sG[s * TS + q + k * GS] = gg;
          sU[s * TS + q + k * GS] = h - 1.0;
          pcv[k] += ((cp - 1.0) * riw) * yload(s, k);
        }
      }
      FORV pcv[k] = warp_group_sum<GS>(pcv[k]);
      if (wlead) FORV PT(1, w, k) = pcv[k];
    }
    __syncthreads();
    double cvp[V];
    FORV {
      double c2 = 0.0;
      for (int ww = 0; ww < NW; ++ww) c2 += PT(1, ww, k);
      cvp[k] = c2;
    }
    RXN_PASS(sC, Csum)
    __syncthreads();
    {
      double pe[V];
      FORV pe[k] = 0.0;
      SNAKE(s, TB(spc_order), S) {
        double des[V], cre[V];
        FORV des[k] = cre[k] = 0.0;
        gather_rop<TS, V>(sROP, TB(sd_step), TB(sd_ptr)[s], TB(sd_ptr)[s + 1], q, des);
        gather_rop<TS, V>(sROP, TB(sc_step), TB(sc_ptr)[s], TB(sc_ptr)[s + 1], q, cre);
        FORV {
          const double net = cre[k] - des[k];
          pe[k] += sU[s * TS + q + k * GS] * net * v[k];
          sU[s * TS + q + k * GS] = net;  // u/RT at T' is not needed again
        }
      }
      FORV pe[k] = warp_group_sum<GS>(pe[k]);
      if (wlead) FORV PT(0, w, k) = pe[k];
    }
    __syncthreads();
    {
      double tdp[V];
      FORV {
        double es = 0.0;
        for (int ww = 0; ww < NW; ++ww) es += PT(0, ww, k);
        tdp[k] = -es * kRu * ysp[k] / cvp[k] + 0.0;
      }
      const int k0 = TB(col_ptr)[S], k1 = TB(col_ptr)[S + 1];
      for (int kk = k0 + g; kk < k1; kk += NG) {
        const int row = TB(row_idx)[kk];
        FORV {
          double d;
          if (row < S) {
            const double mr = TB(mw)[row];
            const double f1 = sU[row * TS + q + k * GS] * mr * v[k];
            const double f0 = (valid[k] ? wdot[(size_t)row * ld + st[k]] : 0.0) * mr * v[k];
            d = (f1 - f0) * mult[k];
          } else {
            d = (tdp[k] - td[k]) * mult[k];
          }
          if (valid[k]) jac[(size_t)kk * ld + st[k]] = d;
        }
      }
    }
    __syncthreads();
  }
#undef PT
#undef TB
#undef FORV
#undef SNAKE
#undef RXN_PASS
}

template <int TS, int V, int MAXT, bool STAGE, int MINB>
cudaError_t launch_tvms(const DevMech &m, const RatesJacArgs &a, const KinParams &kp,
                        const LaunchCfg &cfg, cudaStream_t stream) {
  const int threads = cfg.warps * 32;
  const Layout L = make_layout(m.nsp, m.nstep, cfg.warps);
  const size_t ws_bytes = (size_t)L.rows * TS * sizeof(double);
  const int ntiles = (a.n + TS - 1) / TS;
  if (ntiles == 0) return cudaSuccess;
  const int stage_bytes = STAGE ? m.hot_bytes : 0;
  const size_t smem = (cfg.global_ws ? 0 : ws_bytes) + stage_bytes;
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(rates_jac_kernel<TS, V, MAXT, STAGE, MINB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // the smallest shared-memory carve-out that holds the workspace (and the
  // staged tables), so the rest of the SM's 256 KB stays L1
  const int pct = (int)((100 * MINB * (smem + 1024) + 228 * 1024 - 1) / (228 * 1024));
  e = cudaFuncSetAttribute(rates_jac_kernel<TS, V, MAXT, STAGE, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           pct < 100 ? pct : 100);
  if (e != cudaSuccess) return e;
  if (!cfg.global_ws) {
    // persistent CTAs when the tables are staged (one copy per CTA, not per tile)
    int grid = ntiles;
    if (STAGE) {
      int dev = 0, sms = 148, per_sm = 1;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rates_jac_kernel<TS, V, MAXT, STAGE, MINB>, threads, smem);
      grid = std::min(ntiles, sms * std::max(1, per_sm));
    }
    rates_jac_kernel<TS, V, MAXT, STAGE, MINB><<<grid, threads, smem, stream>>>(
        m, a.n, a.ld, a.T, a.P, a.Y, a.wdot, a.jac, a.ydot, kp, nullptr, (int)(ws_bytes / sizeof(double)),
        stage_bytes);
  } else {
    int grid = cfg.grid > 0 ? cfg.grid : ntiles;
    if (grid > ntiles) grid = ntiles;
    if ((size_t)grid * ws_bytes > a.scratch_bytes) return cudaErrorInvalidValue;
    rates_jac_kernel<TS, V, MAXT, STAGE, MINB><<<grid, threads, smem, stream>>>(m, a.n, a.ld, a.T, a.P, a.Y, a.wdot,
                                                            a.jac, a.ydot, kp, a.scratch,
                                                            (int)(ws_bytes / sizeof(double)), stage_bytes);
  }
  return cudaGetLastError();
}

// Staged tables only with tiles of at most 16 states (larger tiles leave no
// room for them beside the workspace).
template <int TS, int V, int MAXT>
cudaError_t launch_tvm(const DevMech &m, const RatesJacArgs &a, const KinParams &kp,
                       const LaunchCfg &cfg, cudaStream_t stream) {
  if constexpr (TS <= 16) {
    if (cfg.stage) return launch_tvms<TS, V, MAXT, true, 1>(m, a, kp, cfg, stream);
    if constexpr (MAXT == 256) {
      if (cfg.minb == 2) return launch_tvms<TS, V, MAXT, false, 2>(m, a, kp, cfg, stream);
    }
  } else {
    if (cfg.stage) return cudaErrorInvalidValue;
  }
  if (cfg.minb != 1) return cudaErrorInvalidValue;
  return launch_tvms<TS, V, MAXT, false, 1>(m, a, kp, cfg, stream);
}

// Up to 8 warps per CTA the kernel may use 255 registers per thread, up to
// 16 warps 128, and with 32 warps (one state per thread only) 64: twice the
// resident warps to hide latency with.
template <int TS, int V>
cudaError_t launch_tv(const DevMech &m, const RatesJacArgs &a, const KinParams &kp,
                      const LaunchCfg &cfg, cudaStream_t stream) {
  if (cfg.warps <= 8) return launch_tvm<TS, V, 256>(m, a, kp, cfg, stream);
  if (cfg.warps <= 16) return launch_tvm<TS, V, 512>(m, a, kp, cfg, stream);
  if constexpr (V == 1) return launch_tvm<TS, V, 1024>(m, a, kp, cfg, stream);
  return cudaErrorInvalidValue;
}

}  // namespace

size_t rates_jac_ws_bytes(const DevMech &m, const LaunchCfg &cfg) {
  const Layout L = make_layout(m.nsp, m.nstep, cfg.warps);
  return (size_t)L.rows * cfg.ts * sizeof(double);
}

size_t rates_jac_smem_bytes(const DevMech &m, const LaunchCfg &cfg) {
  return (cfg.global_ws ? 0 : rates_jac_ws_bytes(m, cfg)) + (cfg.stage ? (size_t)m.hot_bytes : 0);
}

bool rates_jac_mapping_ok(const LaunchCfg &c) {
  if (c.warps < 1 || c.warps > 32) return false;
  if (c.minb != 1 && (c.minb != 2 || c.warps > 8 || c.ts > 16 || c.stage)) return false;
  if (c.warps > 16 && c.v != 1) return false;  // 64 registers per thread: one state each
  switch (c.ts * 8 + c.v) {
    case 8 * 8 + 1: case 8 * 8 + 2: case 8 * 8 + 4:
    case 16 * 8 + 1: case 16 * 8 + 2: case 16 * 8 + 4:
    case 32 * 8 + 1: case 32 * 8 + 2: case 32 * 8 + 4:
      return true;
    default:
      return false;
  }
}

cudaError_t launch_rates_jac(const DevMech &m, const RatesJacArgs &a, const KinParams &kp,
                             const LaunchCfg &cfg, cudaStream_t stream) {
  switch (cfg.ts * 8 + cfg.v) {
    case 8 * 8 + 1: return launch_tv<8, 1>(m, a, kp, cfg, stream);
    case 8 * 8 + 2: return launch_tv<8, 2>(m, a, kp, cfg, stream);
    case 8 * 8 + 4: return launch_tv<8, 4>(m, a, kp, cfg, stream);
    case 16 * 8 + 1: return launch_tv<16, 1>(m, a, kp, cfg, stream);
    case 16 * 8 + 2: return launch_tv<16, 2>(m, a, kp, cfg, stream);
    case 16 * 8 + 4: return launch_tv<16, 4>(m, a, kp, cfg, stream);
    case 32 * 8 + 1: return launch_tv<32, 1>(m, a, kp, cfg, stream);
    case 32 * 8 + 2: return launch_tv<32, 2>(m, a, kp, cfg, stream);
    case 32 * 8 + 4: return launch_tv<32, 4>(m, a, kp, cfg, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace zrk
