// mlp.cu -- the learned BDF predictor network: a multilayer perceptron with
// SiLU hidden layers, BF16 weights and activations, FP32 accumulation, FP32
// master weights and Adam moments, trained and evaluated by the kernels in
// this file (no library GEMM).
//
// Layouts (row-major, every dimension padded to a multiple of 16):
//   X_l [batch x K_l] bf16 (layer input), W_l [K_l x N_l] bf16, b_l [N_l] f32,
//   Z_l [batch x N_l] f32 (pre-activation, kept for the backward pass).
// The matrix products run on the tensor cores through 16x16x16 BF16
// fragments with FP32 accumulators; a CTA of 4 warps owns a 64 x 64 tile of
// the output, each warp 32 x 32.  Transposed operands (X^T dZ for the weight
// gradient, dZ W^T for the input gradient) are read in place through
// column-major fragments.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/zerork_b200.h"
#include "../../include/zerork_b200_predictor.h"
#include "capi_internal.h"
#include "mlp.h"

namespace zrk {
namespace {

using bf16 = __nv_bfloat16;
namespace wm = nvcuda::wmma;

template <bool TA, bool TB>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const bf16 *__restrict__ A,
                                                        int lda, const bf16 *__restrict__ B, int ldb,
                                                        float *__restrict__ C, int ldc) {
  using LA = typename std::conditional<TA, wm::col_major, wm::row_major>::type;
  using LB = typename std::conditional<TB, wm::col_major, wm::row_major>::type;
  const int warp = threadIdx.x >> 5;
  const int m0 = blockIdx.y * 64 + (warp >> 1) * 32;
  const int n0 = blockIdx.x * 64 + (warp & 1) * 32;
  wm::fragment<wm::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) wm::fill_fragment(acc[i][j], 0.0f);
  const bool mi[2] = {m0 < M, m0 + 16 < M}, nj[2] = {n0 < N, n0 + 16 < N};
  for (int k = 0; k < K; k += 16) {
    wm::fragment<wm::matrix_a, 16, 16, 16, bf16, LA> a[2];
    wm::fragment<wm::matrix_b, 16, 16, 16, bf16, LB> b[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (mi[i]) {
        const int r = m0 + 16 * i;
        wm::load_matrix_sync(a[i], TA ? A + (size_t)k * lda + r : A + (size_t)r * lda + k, lda);
      } else {
        wm::fill_fragment(a[i], __float2bfloat16(0.0f));
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (nj[j]) {
        const int c = n0 + 16 * j;
        wm::load_matrix_sync(b[j], TB ? B + (size_t)c * ldb + k : B + (size_t)k * ldb + c, ldb);
      } else {
        wm::fill_fragment(b[j], __float2bfloat16(0.0f));
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) wm::mma_sync(acc[i][j], a[i], b[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
      if (mi[i] && nj[j])
        wm::store_matrix_sync(C + (size_t)(m0 + 16 * i) * ldc + n0 + 16 * j, acc[i][j], ldc,
                              wm::mem_row_major);
}

template <bool TA, bool TB>
cudaError_t gemm(int M, int N, int K, const bf16 *A, int lda, const bf16 *B, int ldb, float *C, int ldc,
                 cudaStream_t s) {
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  gemm_bf16_kernel<TA, TB><<<grid, 128, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc);
  return cudaGetLastError();
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }

// input: f32 [batch x n_in] (row stride n_in) -> bf16 [batch x K0] zero-padded
__global__ void input_to_bf16(int rows, int n_in, int K0, const float *__restrict__ x, bf16 *__restrict__ X) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows * K0) return;
  const int r = (int)(i / K0), c = (int)(i - (long)r * K0);
  X[i] = __float2bfloat16(c < n_in ? x[(size_t)r * n_in + c] : 0.0f);
}

// hidden layer epilogue: Z += b; A = bf16(silu(Z))
__global__ void bias_silu(int rows, int N, float *__restrict__ Z, const float *__restrict__ b,
                          bf16 *__restrict__ A) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows * N) return;
  const float z = Z[i] + b[i % N];
  Z[i] = z;
  A[i] = __float2bfloat16(silu(z));
}

// output layer epilogue: y = Z + b (valid columns) into y [rows x n_out]
__global__ void bias_out(int rows, int N, int n_out, const float *__restrict__ Z, const float *__restrict__ b,
                         float *__restrict__ y) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows * n_out) return;
  const int r = (int)(i / n_out), c = (int)(i - (long)r * n_out);
  y[i] = Z[(size_t)r * N + c] + b[c];
}

// MSE loss gradient: dY = 2 (y - t) / (rows * n_out) on valid columns, 0 on
// padding; f32 copy for the bias gradient, bf16 for the products; per-row
// squared errors for the loss.
__global__ void mse_grad(int rows, int N, int n_out, const float *__restrict__ Z, const float *__restrict__ b,
                         const float *__restrict__ t, float *__restrict__ dZf, bf16 *__restrict__ dZ,
                         float *__restrict__ row_sq) {
  const int r = blockIdx.x;
  float sq = 0.0f;
  const float scale = 2.0f / ((float)rows * (float)n_out);
  for (int c = threadIdx.x; c < N; c += blockDim.x) {
    float g = 0.0f;
    if (c < n_out) {
      const float e = Z[(size_t)r * N + c] + b[c] - t[(size_t)r * n_out + c];
      sq += e * e;
      g = scale * e;
    }
    dZf[(size_t)r * N + c] = g;
    dZ[(size_t)r * N + c] = __float2bfloat16(g);
  }
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    row_sq[r] = s;
  }
}

// SiLU backward: dZ = dA * silu'(Z)  (dA f32 from the product)
__global__ void silu_bwd(int rows, int N, const float *__restrict__ dA, const float *__restrict__ Z,
                         float *__restrict__ dZf, bf16 *__restrict__ dZ) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows * N) return;
  const float z = Z[i], s = 1.0f / (1.0f + expf(-z));
  const float g = dA[i] * s * (1.0f + z * (1.0f - s));
  dZf[i] = g;
  dZ[i] = __float2bfloat16(g);
}

// bias gradient: column sums, one thread per column, rows in order
__global__ void col_sum(int rows, int N, const float *__restrict__ dZf, float *__restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += dZf[(size_t)r * N + c];
  db[c] = s;
}

__global__ void sum_rows(int rows, const float *__restrict__ row_sq, float *__restrict__ out) {
  float s = 0.0f;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) s += row_sq[r];
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *out = t;
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master copy; refreshes the BF16 copy
__global__ void adam_step(long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                          float *__restrict__ v, float lr, float b1, float b2, float eps, float c1,
                          float c2, bf16 *__restrict__ wb) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void to_bf16(long n, const float *__restrict__ a, bf16 *__restrict__ b) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16(a[i]);
}

inline int pad16(int x) { return (x + 15) / 16 * 16; }
inline unsigned blocks(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

Mlp::Mlp(int n_in, int hidden, int layers, int n_out, unsigned long long seed)
    : n_in_(n_in), n_out_(n_out) {
  dims_.push_back(pad16(n_in));
  for (int l = 0; l < layers; ++l) dims_.push_back(pad16(hidden));
  dims_.push_back(pad16(n_out));
  const int L = (int)dims_.size() - 1;
  woff_.assign(L + 1, 0);
  boff_.assign(L + 1, 0);
  for (int l = 0; l < L; ++l) {
    woff_[l + 1] = woff_[l] + (long)dims_[l] * dims_[l + 1];
    boff_[l + 1] = boff_[l] + dims_[l + 1];
  }
  nw_ = woff_[L];
  nb_ = boff_[L];
  // Kaiming-uniform weights on the real fan-in, zero padding rows/columns
  std::mt19937_64 rng(seed);
  std::vector<float> w(nw_, 0.0f), b(nb_, 0.0f);
  for (int l = 0; l < L; ++l) {
    const int fan_in = l == 0 ? n_in : hidden;
    const int kin = l == 0 ? n_in : hidden, kout = l == L - 1 ? n_out : hidden;
    const float bound = std::sqrt(6.0f / (float)fan_in) * (l == L - 1 ? 0.1f : 1.0f);
    std::uniform_real_distribution<float> U(-bound, bound);
    for (int i = 0; i < kin; ++i)
      for (int j = 0; j < kout; ++j) w[woff_[l] + (long)i * dims_[l + 1] + j] = U(rng);
  }
  auto ck = [](cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("mlp: ") + cudaGetErrorString(e));
  };
  const size_t np = nw_ + nb_;
  ck(cudaMalloc(&master_, np * sizeof(float)));
  ck(cudaMalloc(&grad_, np * sizeof(float)));
  ck(cudaMalloc(&m1_, np * sizeof(float)));
  ck(cudaMalloc(&m2_, np * sizeof(float)));
  ck(cudaMalloc(&wbf_, nw_ * sizeof(bf16)));
  ck(cudaMemset(m1_, 0, np * sizeof(float)));
  ck(cudaMemset(m2_, 0, np * sizeof(float)));
  ck(cudaMemset(grad_, 0, np * sizeof(float)));
  set_params(w.data(), b.data());
}

Mlp::~Mlp() {
  cudaFree(master_);
  cudaFree(grad_);
  cudaFree(m1_);
  cudaFree(m2_);
  cudaFree(wbf_);
  cudaFree(ws_);
}

void Mlp::set_params(const float *w, const float *b) {
  cudaMemcpy(master_, w, nw_ * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(master_ + nw_, b, nb_ * sizeof(float), cudaMemcpyHostToDevice);
  to_bf16<<<blocks(nw_, 256), 256>>>(nw_, master_, (bf16 *)wbf_);
  cudaDeviceSynchronize();
}

void Mlp::get_params(float *w, float *b) const {
  cudaMemcpy(w, master_, nw_ * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(b, master_ + nw_, nb_ * sizeof(float), cudaMemcpyDeviceToHost);
}

void Mlp::get_grads(float *w, float *b) const {
  cudaMemcpy(w, grad_, nw_ * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(b, grad_ + nw_, nb_ * sizeof(float), cudaMemcpyDeviceToHost);
}

cudaError_t Mlp::ensure_ws(int rows) {
  const int L = (int)dims_.size() - 1;
  int maxd = 0;
  for (int d : dims_) maxd = std::max(maxd, d);
  // per row: X_l bf16 for every layer input, Z_l f32 per layer, dZ f32 + bf16,
  // dA f32, row_sq
  size_t per_row = 0;
  for (int l = 0; l <= L; ++l) per_row += dims_[l] * sizeof(bf16);
  for (int l = 1; l <= L; ++l) per_row += dims_[l] * sizeof(float);
  per_row += maxd * (sizeof(float) * 2 + sizeof(bf16)) + sizeof(float);
  const size_t need = per_row * (size_t)rows + 256 * 32;
  if (need <= ws_bytes_) return cudaSuccess;
  cudaFree(ws_);
  ws_ = nullptr;
  ws_bytes_ = 0;
  cudaError_t e = cudaMalloc(&ws_, need);
  if (e == cudaSuccess) {
    ws_bytes_ = need;
    ws_rows_ = rows;
  }
  return e;
}

// Carve the workspace for `rows` rows (rows a multiple of 16).
void Mlp::carve(int rows, std::vector<bf16 *> &X, std::vector<float *> &Z, float *&dZf, bf16 *&dZ,
                float *&dA, float *&row_sq) {
  const int L = (int)dims_.size() - 1;
  int maxd = 0;
  for (int d : dims_) maxd = std::max(maxd, d);
  char *p = (char *)ws_;
  auto take = [&](size_t bytes) {
    char *q = p;
    p += (bytes + 255) / 256 * 256;
    return q;
  };
  X.assign(L + 1, nullptr);
  Z.assign(L + 1, nullptr);
  for (int l = 0; l <= L; ++l) X[l] = (bf16 *)take((size_t)rows * dims_[l] * sizeof(bf16));
  for (int l = 1; l <= L; ++l) Z[l] = (float *)take((size_t)rows * dims_[l] * sizeof(float));
  dZf = (float *)take((size_t)rows * maxd * sizeof(float));
  dZ = (bf16 *)take((size_t)rows * maxd * sizeof(bf16));
  dA = (float *)take((size_t)rows * maxd * sizeof(float));
  row_sq = (float *)take((size_t)rows * sizeof(float));
}

cudaError_t Mlp::forward_ws(int rows, const float *x, std::vector<bf16 *> &X, std::vector<float *> &Z,
                            cudaStream_t s) {
  const int L = (int)dims_.size() - 1;
  input_to_bf16<<<blocks((long)rows * dims_[0], 256), 256, 0, s>>>(rows, n_in_, dims_[0], x, X[0]);
  for (int l = 0; l < L; ++l) {
    cudaError_t e = gemm<false, false>(rows, dims_[l + 1], dims_[l], X[l], dims_[l],
                                       (const bf16 *)wbf_ + woff_[l], dims_[l + 1], Z[l + 1], dims_[l + 1], s);
    if (e != cudaSuccess) return e;
    if (l + 1 < L)
      bias_silu<<<blocks((long)rows * dims_[l + 1], 256), 256, 0, s>>>(rows, dims_[l + 1], Z[l + 1],
                                                                         master_ + nw_ + boff_[l], X[l + 1]);
  }
  return cudaGetLastError();
}

cudaError_t Mlp::forward(int n, const float *x, float *y, cudaStream_t s) {
  const int rows = pad16(std::max(n, 1));
  cudaError_t e = ensure_ws(rows);
  if (e != cudaSuccess) return e;
  std::vector<bf16 *> X;
  std::vector<float *> Z;
  float *dZf, *dA, *row_sq;
  bf16 *dZ;
  carve(rows, X, Z, dZf, dZ, dA, row_sq);
  // rows beyond n read no input: clear the padded tail of the bf16 input
  if (rows > n) cudaMemsetAsync(X[0] + (size_t)n * dims_[0], 0, (size_t)(rows - n) * dims_[0] * sizeof(bf16), s);
  const int L = (int)dims_.size() - 1;
  input_to_bf16<<<blocks((long)n * dims_[0], 256), 256, 0, s>>>(n, n_in_, dims_[0], x, X[0]);
  for (int l = 0; l < L; ++l) {
    e = gemm<false, false>(rows, dims_[l + 1], dims_[l], X[l], dims_[l], (const bf16 *)wbf_ + woff_[l],
                           dims_[l + 1], Z[l + 1], dims_[l + 1], s);
    if (e != cudaSuccess) return e;
    if (l + 1 < L)
      bias_silu<<<blocks((long)rows * dims_[l + 1], 256), 256, 0, s>>>(rows, dims_[l + 1], Z[l + 1],
                                                                         master_ + nw_ + boff_[l], X[l + 1]);
  }
  bias_out<<<blocks((long)n * n_out_, 256), 256, 0, s>>>(n, dims_[L], n_out_, Z[L],
                                                          master_ + nw_ + boff_[L - 1], y);
  return cudaGetLastError();
}

// Forward + backward on one batch (rows a multiple of 16, rows == n): the
// gradient of the mean squared error lands in grad_; returns the loss sum in
// *loss_dev (device float).
cudaError_t Mlp::backward(int n, const float *x, const float *t, float *loss_dev, cudaStream_t s) {
  if (n % 16) return cudaErrorInvalidValue;
  cudaError_t e = ensure_ws(n);
  if (e != cudaSuccess) return e;
  std::vector<bf16 *> X;
  std::vector<float *> Z;
  float *dZf, *dA, *row_sq;
  bf16 *dZ;
  carve(n, X, Z, dZf, dZ, dA, row_sq);
  if ((e = forward_ws(n, x, X, Z, s)) != cudaSuccess) return e;
  const int L = (int)dims_.size() - 1;
  mse_grad<<<n, 128, 0, s>>>(n, dims_[L], n_out_, Z[L], master_ + nw_ + boff_[L - 1], t, dZf, dZ, row_sq);
  sum_rows<<<1, 256, 0, s>>>(n, row_sq, loss_dev);
  for (int l = L - 1; l >= 0; --l) {
    const int K = dims_[l], N = dims_[l + 1];
    // dW_l = X_l^T dZ ; db_l = colsum(dZ)
    if ((e = gemm<true, false>(K, N, n, X[l], K, dZ, N, grad_ + woff_[l], N, s)) != cudaSuccess) return e;
    col_sum<<<blocks(N, 128), 128, 0, s>>>(n, N, dZf, grad_ + nw_ + boff_[l]);
    if (l == 0) break;
    // dA_{l} = dZ W_l^T ; dZ_{l} = dA * silu'(Z_l)
    if ((e = gemm<false, true>(n, K, N, dZ, N, (const bf16 *)wbf_ + woff_[l], N, dA, K, s)) != cudaSuccess)
      return e;
    silu_bwd<<<blocks((long)n * K, 256), 256, 0, s>>>(n, K, dA, Z[l], dZf, dZ);
  }
  return cudaGetLastError();
}

cudaError_t Mlp::adam(float lr, float b1, float b2, float eps, cudaStream_t s) {
  ++step_;
  const float c1 = 1.0f - std::pow(b1, (float)step_), c2 = 1.0f - std::pow(b2, (float)step_);
  adam_step<<<blocks(nw_, 256), 256, 0, s>>>(nw_, master_, grad_, m1_, m2_, lr, b1, b2, eps, c1, c2,
                                             (bf16 *)wbf_);
  adam_step<<<blocks(nb_, 256), 256, 0, s>>>(nb_, master_ + nw_, grad_ + nw_, m1_ + nw_, m2_ + nw_, lr, b1,
                                             b2, eps, c1, c2, nullptr);
  return cudaGetLastError();
}

MlpDev Mlp::device_view() const {
  MlpDev d{};
  d.layers = (int)dims_.size() - 1;
  for (int l = 0; l <= d.layers && l <= kMlpMaxLayers; ++l) d.dims[l] = dims_[l];
  for (int l = 0; l < d.layers && l < kMlpMaxLayers; ++l) {
    d.w[l] = (const bf16 *)wbf_ + woff_[l];
    d.b[l] = master_ + nw_ + boff_[l];
  }
  d.n_in = n_in_;
  d.n_out = n_out_;
  return d;
}

}  // namespace zrk

using namespace zrk;

extern "C" {

int zrk_mlp_create(int n_in, int hidden, int layers, int n_out, unsigned long long seed, zrk_mlp_t *out) {
  if (!out) return set_error(ZRK_ERR_INVALID_POINTER, "null output");
  if (n_in < 1 || hidden < 1 || layers < 1 || layers > kMlpMaxLayers - 1 || n_out < 1 || hidden > 1024 ||
      n_in > 1024 || n_out > 1024)
    return set_error(ZRK_ERR_INVALID_ARGUMENT, "mlp sizes out of range");
  try {
    *out = reinterpret_cast<zrk_mlp_t>(new Mlp(n_in, hidden, layers, n_out, seed));
  } catch (const std::exception &e) {
    return set_error(ZRK_ERR_CUDA, e.what());
  }
  return ZRK_OK;
}

int zrk_mlp_free(zrk_mlp_t m) {
  delete reinterpret_cast<Mlp *>(m);
  return ZRK_OK;
}

int zrk_mlp_sizes(zrk_mlp_t m, long *n_weights, long *n_biases) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null mlp");
  Mlp *p = reinterpret_cast<Mlp *>(m);
  if (n_weights) *n_weights = p->n_weights();
  if (n_biases) *n_biases = p->n_biases();
  return ZRK_OK;
}

int zrk_mlp_get_params(zrk_mlp_t m, float *w, float *b) {
  if (!m || !w || !b) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  reinterpret_cast<Mlp *>(m)->get_params(w, b);
  return ZRK_OK;
}

int zrk_mlp_set_params(zrk_mlp_t m, const float *w, const float *b) {
  if (!m || !w || !b) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  reinterpret_cast<Mlp *>(m)->set_params(w, b);
  return ZRK_OK;
}

int zrk_mlp_get_grads(zrk_mlp_t m, float *w, float *b) {
  if (!m || !w || !b) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  cudaDeviceSynchronize();
  reinterpret_cast<Mlp *>(m)->get_grads(w, b);
  return ZRK_OK;
}

int zrk_mlp_forward(zrk_mlp_t m, int n, const float *x, float *y, void *stream) {
  if (!m || !x || !y) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  if (n < 0) return set_error(ZRK_ERR_INVALID_ARGUMENT, "n < 0");
  if (n == 0) return ZRK_OK;
  cudaError_t e = reinterpret_cast<Mlp *>(m)->forward(n, x, y, (cudaStream_t)stream);
  return e == cudaSuccess ? ZRK_OK : cuda_error(e, "mlp forward");
}

int zrk_mlp_gradients(zrk_mlp_t m, int n, const float *x, const float *t, float *loss_sum_dev, void *stream) {
  if (!m || !x || !t || !loss_sum_dev) return set_error(ZRK_ERR_INVALID_POINTER, "null argument");
  if (n <= 0 || n % 16) return set_error(ZRK_ERR_INVALID_ARGUMENT, "batch must be a positive multiple of 16");
  cudaError_t e = reinterpret_cast<Mlp *>(m)->backward(n, x, t, loss_sum_dev, (cudaStream_t)stream);
  return e == cudaSuccess ? ZRK_OK : cuda_error(e, "mlp backward");
}

int zrk_mlp_adam(zrk_mlp_t m, float lr, float beta1, float beta2, float eps, void *stream) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null mlp");
  cudaError_t e = reinterpret_cast<Mlp *>(m)->adam(lr, beta1, beta2, eps, (cudaStream_t)stream);
  return e == cudaSuccess ? ZRK_OK : cuda_error(e, "mlp adam");
}

}  // extern "C"
