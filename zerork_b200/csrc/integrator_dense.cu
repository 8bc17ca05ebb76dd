// integrator_dense.cu -- host side of the dense-block integrator: shared
// memory layout and the launch dispatch over the factor type.
#include "integrator_dense.cuh"

namespace zrk {

size_t dense_smem_bytes(const DevMech &m, bool fp32, int *lda_out, int spill) {
  const int n = m.nsp + 1;
  const int lda = (n % 2 == 1) ? n : n + 1;  // odd row stride: conflict-free column walks
  if (lda_out) *lda_out = lda;
  size_t d = 128 + 3 * (size_t)m.nsp + 12 * (size_t)n + ((n + 1) / 2 + 1) + kPredBuf;
  if (fp32) d += (kMaxl + 3) * (size_t)n;
  if (!(spill & 1)) d += m.nstep;
  if (!(spill & 2)) d += (kMaxOrder + 3) * (size_t)n;
  if (spill & 4) d += m.nnz;  // reactor Jacobian in shared memory
  size_t bytes = d * sizeof(double) + (size_t)n * lda * (fp32 ? sizeof(float) : sizeof(double));
  return ((bytes + 15) / 16) * 16;
}

size_t dense_spill_doubles(const DevMech &m) {
  // rates of progress, BDF differences, energy-source coupling vectors
  return (size_t)m.nstep + (kMaxOrder + 6) * (size_t)(m.nsp + 1);
}


cudaError_t launch_integrate_dense(const DevMech &m, const IntegOpts &o, const IntegArgs &a,
                                   int threads, int ctas, int spill, cudaStream_t stream) {
  int lda = 0;
  const size_t smem = dense_smem_bytes(m, o.lu_fp32 != 0, &lda, spill);
  const int n = m.nsp + 1;
  if (n > kDenseMaxN) return cudaErrorInvalidValue;
  return o.lu_fp32 ? launch_integrate_dense_f32(m, o, a, threads, ctas, spill, smem, lda, stream)
                   : launch_integrate_dense_f64(m, o, a, threads, ctas, spill, smem, lda, stream);
}

}  // namespace zrk
