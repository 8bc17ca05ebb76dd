// ref_cuda_shim.cu -- ORACLE test infrastructure: a C interface over the
// reference's own GPU mechanism (zerork::mechanism_cuda, src/zerork/
// mechanism_cuda.h:9-45), compiled unmodified from the reference sources for
// sm_100a by oracle/Makefile (target ref-cuda) into oracle/_ref.  Used only
// to time the reference GPU rate path beside this repository's kernels
// (bench.py's reference_gpu block); nothing in the product links it.
#include <cstdio>
#include <exception>

#include "zerork/mechanism_cuda.h"

extern "C" {

void *zrkref_cuda_load(const char *mech, const char *therm, const char *log, int n_max) {
  try {
    return new zerork::mechanism_cuda(mech, therm, log, 0, n_max);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "zrkref_cuda_load: %s\n", e.what());
    return nullptr;
  }
}

void zrkref_cuda_free(void *h) { delete static_cast<zerork::mechanism_cuda *>(h); }

int zrkref_cuda_n_max(void *h) { return static_cast<zerork::mechanism_cuda *>(h)->nReactorsMax(); }

// getReactionRates_CUDA_mr_dev on device arrays (species-major, n leading)
void zrkref_cuda_rates(void *h, int n, const double *T_dev, const double *C_dev, double *net,
                       double *cre, double *des, double *rop) {
  static_cast<zerork::mechanism_cuda *>(h)->getReactionRates_CUDA_mr_dev(n, T_dev, C_dev, net, cre,
                                                                        des, rop);
}

}  // extern "C"
