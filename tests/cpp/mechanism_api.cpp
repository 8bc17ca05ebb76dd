// mechanism_api.cpp -- drives the C++ mechanism surface of
// include/zerork_b200_mechanism.h the way reference callers use
// zerork::mechanism / zerork::mechanism_cuda, for tests/test_mechanism_api.py.
//
//   mechanism_api <mech> <therm> <states.bin> <out.bin>
//
// states.bin: int32 n, then n records of {T, P, Y[nsp]} (doubles).  For each
// state it writes {net, create, destroy [nsp], rop [nstep]} from
// getReactionRatesLimiter (limit 1e22 on every step), net from
// getNetReactionRates and from getReactionRates, u/RT [nsp] and mass c_v
// from the host helpers, then the same rates for all n states from
// mechanism_cuda::getReactionRatesLimiter_CUDA_mr_dev.  Exit code 2 with the
// library's message when the mechanism cannot be created (no CUDA device).
#include <cuda_runtime.h>

#include <cstdio>
#include <exception>
#include <vector>

#include "zerork_b200_mechanism.h"

int main(int argc, char **argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s mech therm states.bin out.bin\n", argv[0]);
    return 1;
  }
  try {
    zerork_b200::mechanism_cuda mech(argv[1], argv[2], "/dev/null", 0, 4096);
    const int ns = mech.getNumSpecies(), nst = mech.getNumSteps();
    FILE *in = std::fopen(argv[3], "rb");
    if (!in) return 1;
    int n = 0;
    if (std::fread(&n, sizeof(int), 1, in) != 1) return 1;
    std::vector<double> rec((size_t)n * (ns + 2));
    if (std::fread(rec.data(), sizeof(double), rec.size(), in) != rec.size()) return 1;
    std::fclose(in);
    FILE *out = std::fopen(argv[4], "wb");
    std::vector<double> C(ns), net(ns), cre(ns), des(ns), rop(nst), lim(nst, 1.0e22), u(ns), cv(ns);
    std::vector<double> Tall(n), Call((size_t)ns * n);
    for (int i = 0; i < n; ++i) {
      const double T = rec[(size_t)i * (ns + 2)], P = rec[(size_t)i * (ns + 2) + 1];
      const double *Y = &rec[(size_t)i * (ns + 2) + 2];
      const double v = 1.0 / mech.getDensityFromTPY(T, P, Y);
      mech.getCfromVY(v, Y, C.data());
      mech.getReactionRatesLimiter(T, C.data(), lim.data(), net.data(), cre.data(), des.data(), rop.data());
      std::fwrite(net.data(), sizeof(double), ns, out);
      std::fwrite(cre.data(), sizeof(double), ns, out);
      std::fwrite(des.data(), sizeof(double), ns, out);
      std::fwrite(rop.data(), sizeof(double), nst, out);
      mech.getNetReactionRates(T, C.data(), net.data());
      std::fwrite(net.data(), sizeof(double), ns, out);
      mech.getReactionRates(T, C.data(), net.data(), cre.data(), des.data(), rop.data());
      std::fwrite(net.data(), sizeof(double), ns, out);
      mech.getIntEnergy_RT(T, u.data());
      std::fwrite(u.data(), sizeof(double), ns, out);
      const double cvm = mech.getMassCvFromTY(T, Y, cv.data());
      std::fwrite(&cvm, sizeof(double), 1, out);
      Tall[i] = T;
      for (int j = 0; j < ns; ++j) Call[(size_t)j * n + i] = C[j];
    }
    // the multi-reactor device entry on the same states
    double *dT, *dC, *dL, *dN, *dCr, *dDe, *dR;
    cudaMalloc(&dT, n * sizeof(double));
    cudaMalloc(&dC, (size_t)ns * n * sizeof(double));
    cudaMalloc(&dL, nst * sizeof(double));
    cudaMalloc(&dN, (size_t)ns * n * sizeof(double));
    cudaMalloc(&dCr, (size_t)ns * n * sizeof(double));
    cudaMalloc(&dDe, (size_t)ns * n * sizeof(double));
    cudaMalloc(&dR, (size_t)nst * n * sizeof(double));
    cudaMemcpy(dT, Tall.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dC, Call.data(), (size_t)ns * n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(dL, lim.data(), nst * sizeof(double), cudaMemcpyHostToDevice);
    mech.getReactionRatesLimiter_CUDA_mr_dev(n, dT, dC, dL, dN, dCr, dDe, dR);
    std::vector<double> h((size_t)(3 * ns + nst) * n);
    cudaMemcpy(h.data(), dN, (size_t)ns * n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(h.data() + (size_t)ns * n, dCr, (size_t)ns * n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(h.data() + (size_t)2 * ns * n, dDe, (size_t)ns * n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(h.data() + (size_t)3 * ns * n, dR, (size_t)nst * n * sizeof(double), cudaMemcpyDeviceToHost);
    std::fwrite(h.data(), sizeof(double), h.size(), out);
    std::fclose(out);
    for (double *p : {dT, dC, dL, dN, dCr, dDe, dR}) cudaFree(p);
    if (cudaGetLastError() != cudaSuccess) return 3;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 2;
  }
  return 0;
}
