// rates_tc.cu -- rates of progress and species production rates from
// temperature and concentrations, for many states at once: the computation
// behind zerork::mechanism::getReactionRates / getReactionRatesLimiter
// (src/zerork/mechanism.cpp:556-620, perf_net.cpp:126-274) and
// mechanism_cuda::getReactionRates(Limiter)_CUDA_mr_dev
// (src/zerork/mechanism_cuda.h:19-45).
//
// Same tiling as the fused rates + Jacobian kernel (kinetics.cu): a CTA works
// on tiles of TS states, a group of TS / V threads owns one work item
// (species or reaction) for all states of the tile, and states are the fast
// index of every array (x[item * ld + state]).  The temperature is used as
// given (no clamp: the reactor clamps before calling these entry points) and
// the pressure of PLOG reactions is the concentrations' Csum Ru T
// (rate_const.cpp:548-567).
#include <cuda_runtime.h>

#include "devmech.h"
#include "kinetics.h"
#include "kinetics_dev.cuh"

namespace zrk {
namespace {

template <int TS, int V, int MINB>
__global__ void __launch_bounds__(256, MINB) rates_tc_kernel(DevMech m, int n, int ld,
                                                      const double *__restrict__ Tin,
                                                      const double *__restrict__ Cin,
                                                      const double *__restrict__ lim_step,
                                                      double *__restrict__ net,
                                                      double *__restrict__ cre_out,
                                                      double *__restrict__ des_out,
                                                      double *__restrict__ rop_out) {
  constexpr int GS = TS / V;
  extern __shared__ double smem_dyn[];
  const int S = m.nsp, N = m.nstep;
  const int NW = blockDim.x >> 5, NG = blockDim.x / GS;
  const int g = threadIdx.x / GS, q = threadIdx.x % GS, w = threadIdx.x >> 5;
  const bool wlead = (threadIdx.x & 31) < GS;
  double *sC = smem_dyn, *sG = sC + S * TS, *sROP = sG + S * TS, *sPart = sROP + (size_t)N * TS;
#define FORV _Pragma("unroll") for (int k = 0; k < V; ++k)
  const int ntiles = (n + TS - 1) / TS;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int st[V];
    bool valid[V];
    double T[V], logT[V], invT[V], lprt[V], Csum[V];
    FORV {
      st[k] = tile * TS + q + k * GS;
      valid[k] = st[k] < n;
      T[k] = valid[k] ? Tin[st[k]] : 1000.0;
      logT[k] = log(T[k]);
      invT[k] = 1.0 / T[k];
      lprt[k] = log(kPatmD / (kRuD * T[k]));
    }
    // concentrations and g/RT; partial concentration sums per warp
    {
      double pc[V];
      FORV pc[k] = 0.0;
      for (int s = g; s < S; s += NG) {
        const double *th = m.thermo + 16 * s;
        FORV {
          const double c = valid[k] ? Cin[(size_t)s * ld + st[k]] : 0.0;
          sC[s * TS + q + k * GS] = c;
          double cp, h, gg;
          nasa_cp_h_g(th, T[k], logT[k], &cp, &h, &gg);
          sG[s * TS + q + k * GS] = gg;
          pc[k] += c;
        }
      }
#pragma unroll
      for (int o = GS; o < 32; o <<= 1) FORV pc[k] += __shfl_xor_sync(0xffffffffu, pc[k], o);
      if (wlead) FORV sPart[w * TS + q + k * GS] = pc[k];
    }
    __syncthreads();
    FORV {
      double cs = 0.0;
      for (int ww = 0; ww < NW; ++ww) cs += sPart[ww * TS + q + k * GS];
      Csum[k] = cs;
    }
    // reactions: both steps of each reaction, the cost-sorted records dealt
    // to the groups in snake order (round r gives group g the record at
    // r*NG + g, or r*NG + NG-1-g for odd r) so every group's work is close
    // to the mean
    for (int rr = 0; rr * NG < m.nrxn; ++rr) {
      const int rp = rr * NG + ((rr & 1) ? NG - 1 - g : g);
      if (rp < m.nrxn)
        reaction_item<TS, V>(m, load_rxn(m.rxn_by_cost + rp), q, sC, sG, sROP, T, logT, invT, lprt, Csum,
                             0.0, lim_step);
    }
    __syncthreads();
    // destruction and creation in ascending step order, net = create - destroy
    for (int s = g; s < S; s += NG) {
      double des[V], cre[V];
      FORV des[k] = cre[k] = 0.0;
      for (int i = m.sd_ptr[s]; i < m.sd_ptr[s + 1]; ++i) {
        const double *rp = sROP + m.sd_step[i] * TS + q;
        FORV des[k] += rp[k * GS];
      }
      for (int i = m.sc_ptr[s]; i < m.sc_ptr[s + 1]; ++i) {
        const double *rp = sROP + m.sc_step[i] * TS + q;
        FORV cre[k] += rp[k * GS];
      }
      FORV if (valid[k]) {
        const size_t o = (size_t)s * ld + st[k];
        if (net) net[o] = cre[k] - des[k];
        if (cre_out) cre_out[o] = cre[k];
        if (des_out) des_out[o] = des[k];
      }
    }
    if (rop_out)
      for (int j = g; j < N; j += NG) FORV if (valid[k]) rop_out[(size_t)j * ld + st[k]] = sROP[j * TS + q + k * GS];
    __syncthreads();  // the next tile reuses the workspace
  }
#undef FORV
}

template <int TS, int V, int MINB>
cudaError_t launch_tv(const DevMech &m, const RatesTCArgs &a, int threads, cudaStream_t stream) {
  const int NW = threads / 32;
  const size_t bytes = ((size_t)(2 * m.nsp + m.nstep) * TS + (size_t)NW * TS) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(rates_tc_kernel<TS, V, MINB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (a.n + TS - 1) / TS;
  const int grid = ntiles < 8 * sms ? ntiles : 8 * sms;
  rates_tc_kernel<TS, V, MINB><<<grid, threads, bytes, stream>>>(m, a.n, a.ld, a.T, a.C, a.lim_step,
                                                          a.net, a.create, a.destroy, a.rop);
  return cudaGetLastError();
}

}  // namespace

size_t rates_tc_smem_bytes(const DevMech &m, int ts, int threads) {
  return ((size_t)(2 * m.nsp + m.nstep) * ts + (size_t)(threads / 32) * ts) * sizeof(double);
}

cudaError_t launch_rates_tc(const DevMech &m, const RatesTCArgs &a, cudaStream_t stream) {
  if (a.n <= 0) return cudaSuccess;
  // two 8-warp CTAs per SM (16 resident warps, 128 registers each) with 16
  // states per tile where two workspaces fit in shared memory; else one CTA
  // per SM with the largest tile that fits
  const size_t kMax = 227 * 1024, kSm = 228 * 1024;
  if (2 * (rates_tc_smem_bytes(m, 16, 256) + 1024) <= kSm) return launch_tv<16, 2, 2>(m, a, 256, stream);
  if (rates_tc_smem_bytes(m, 32, 256) <= kMax) return launch_tv<32, 2, 1>(m, a, 256, stream);
  if (rates_tc_smem_bytes(m, 16, 256) <= kMax) return launch_tv<16, 1, 1>(m, a, 256, stream);
  if (rates_tc_smem_bytes(m, 8, 256) <= kMax) return launch_tv<8, 1, 1>(m, a, 256, stream);
  return cudaErrorInvalidValue;
}

}  // namespace zrk
