// integrator_dense.cu -- host side of the dense-block integrator: shared
// memory layout and the launch dispatch over the register-chunk count.
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
  // register chunks of 32 columns per lane in the inversion: ceil(n / 32)
  const int nc = (n + 31) / 32;
  switch (nc) {
    case 1: return launch_integrate_dense_nc1(m, o, a, threads, ctas, spill, smem, lda, stream);
    case 2: return launch_integrate_dense_nc2(m, o, a, threads, ctas, spill, smem, lda, stream);
    case 3: return launch_integrate_dense_nc3(m, o, a, threads, ctas, spill, smem, lda, stream);
    case 4: return launch_integrate_dense_nc4(m, o, a, threads, ctas, spill, smem, lda, stream);
    case 5: return launch_integrate_dense_nc5(m, o, a, threads, ctas, spill, smem, lda, stream);
    case 6: return launch_integrate_dense_nc6(m, o, a, threads, ctas, spill, smem, lda, stream);
    case 7: return launch_integrate_dense_nc7(m, o, a, threads, ctas, spill, smem, lda, stream);
    case 8: return launch_integrate_dense_nc8(m, o, a, threads, ctas, spill, smem, lda, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace zrk
