// integrator_dense_nc6.cu -- dense-block integrator kernels for 161 <= nsp + 1 <= 192.
#include "integrator_dense.cuh"

namespace zrk {

cudaError_t launch_integrate_dense_nc6(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                        int threads, int ctas, int spill, size_t smem, int lda,
                                        cudaStream_t stream) {
  return o.lu_fp32 ? launch_dense<float, 6>(m, o, a, threads, ctas, spill, smem, lda, stream)
                   : launch_dense<double, 6>(m, o, a, threads, ctas, spill, smem, lda, stream);
}

}  // namespace zrk
