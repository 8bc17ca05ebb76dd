// integrator_dense_nc7.cu -- dense-block integrator kernels for 193 <= nsp + 1 <= 224.
#include "integrator_dense.cuh"

namespace zrk {

cudaError_t launch_integrate_dense_nc7(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                        int threads, int ctas, int spill, size_t smem, int lda,
                                        cudaStream_t stream) {
  return o.lu_fp32 ? launch_dense<float, 7>(m, o, a, threads, ctas, spill, smem, lda, stream)
                   : launch_dense<double, 7>(m, o, a, threads, ctas, spill, smem, lda, stream);
}

}  // namespace zrk
