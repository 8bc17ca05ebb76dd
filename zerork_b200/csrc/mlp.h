// mlp.h -- the predictor network (mlp.cu) and its device view for kernels.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <vector>

namespace zrk {

constexpr int kMlpMaxLayers = 6;  // weight layers (hidden layers + output)

// Plain-pointer view for device code: layer l maps dims[l] -> dims[l + 1]
// (padded to multiples of 16) with bf16 weights w[l] [dims[l] x dims[l+1]]
// row-major and f32 biases b[l]; SiLU after every layer but the last.
struct MlpDev {
  int layers = 0;
  int dims[kMlpMaxLayers + 1] = {};
  const __nv_bfloat16 *w[kMlpMaxLayers] = {};
  const float *b[kMlpMaxLayers] = {};
  int n_in = 0, n_out = 0;
};

class Mlp {
 public:
  Mlp(int n_in, int hidden, int layers, int n_out, unsigned long long seed);
  ~Mlp();
  Mlp(const Mlp &) = delete;
  Mlp &operator=(const Mlp &) = delete;
  long n_weights() const { return nw_; }
  long n_biases() const { return nb_; }
  void set_params(const float *w, const float *b);
  void get_params(float *w, float *b) const;
  void get_grads(float *w, float *b) const;
  cudaError_t forward(int n, const float *x, float *y, cudaStream_t s);
  cudaError_t backward(int n, const float *x, const float *t, float *loss_dev, cudaStream_t s);
  cudaError_t adam(float lr, float b1, float b2, float eps, cudaStream_t s);
  MlpDev device_view() const;

 private:
  cudaError_t ensure_ws(int rows);
  void carve(int rows, std::vector<__nv_bfloat16 *> &X, std::vector<float *> &Z, float *&dZf,
             __nv_bfloat16 *&dZ, float *&dA, float *&row_sq);
  cudaError_t forward_ws(int rows, const float *x, std::vector<__nv_bfloat16 *> &X, std::vector<float *> &Z,
                         cudaStream_t s);
  int n_in_, n_out_;
  std::vector<int> dims_;
  std::vector<long> woff_, boff_;
  long nw_ = 0, nb_ = 0;
  float *master_ = nullptr, *grad_ = nullptr, *m1_ = nullptr, *m2_ = nullptr;
  void *wbf_ = nullptr;
  void *ws_ = nullptr;
  size_t ws_bytes_ = 0;
  int ws_rows_ = 0;
  long step_ = 0;
};

}  // namespace zrk
