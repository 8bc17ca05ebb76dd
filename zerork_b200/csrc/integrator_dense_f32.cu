// integrator_dense_f32.cu -- dense-block integrator kernel with a float Newton factor.
#include "integrator_dense.cuh"

namespace zrk {

cudaError_t launch_integrate_dense_f32(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                       int threads, int ctas, int spill, size_t smem, int lda,
                                       cudaStream_t stream) {
  return launch_dense<float>(m, o, a, threads, ctas, spill, smem, lda, stream);
}

}  // namespace zrk
