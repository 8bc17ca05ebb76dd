// integrator_dense_nc1.cu -- dense-block integrator kernels for 1 <= nsp + 1 <= 32.
#include "integrator_dense.cuh"

namespace zrk {

cudaError_t launch_integrate_dense_nc1(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                        int threads, int ctas, int spill, size_t smem, int lda,
                                        cudaStream_t stream) {
  return o.lu_fp32 ? launch_dense<float, 1>(m, o, a, threads, ctas, spill, smem, lda, stream)
                   : launch_dense<double, 1>(m, o, a, threads, ctas, spill, smem, lda, stream);
}

}  // namespace zrk
