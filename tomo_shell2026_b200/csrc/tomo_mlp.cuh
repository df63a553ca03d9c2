// Surrogate network of the learned-proposal orientation search: an FP32 MLP
// [sin yaw, cos yaw, sin pitch, cos pitch] -> 128 -> 128 -> 128 -> Vss with
// tanh hidden units and a linear output, trained full-batch with Adam by the
// hand-written kernels of tomo_mlp.cu: one fused kernel per block of 16
// samples runs the forward pass, the loss and the whole backward pass out of
// shared memory and writes that block's gradient; a second kernel sums the
// blocks' gradients in a fixed order (deterministic) and applies Adam.
// Nothing here is a dense contraction large enough for tensor cores: one
// training step on 936 samples is ~60 MFLOP.
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace tomo {

constexpr int kMlpIn = 4;
constexpr int kMlpHidden = 128;
constexpr int kMlpLayers = 4;   // 3 hidden + output

// Flat parameter layout: W1 [4][128], b1 [128], W2 [128][128], b2, W3 [128][128], b3, W4 [128][1], b4 [1];
// weights row-major [in][out].
struct MlpLayout {
  int in[kMlpLayers], out[kMlpLayers], w[kMlpLayers], b[kMlpLayers];
  int total;
  MlpLayout();
};

// x[n][4] = sin yaw, cos yaw, sin pitch, cos pitch of ypr[n][3] (device arrays).
cudaError_t mlp_features(const float* ypr, int n, float* x, cudaStream_t s);

class Mlp {
 public:
  ~Mlp();
  // Seeded initialisation (uniform +-sqrt(6 / (fan_in + fan_out)), zero biases), Adam state cleared.
  cudaError_t init(unsigned seed, cudaStream_t s);
  int param_count() const { return L.total; }
  cudaError_t get_params(float* host, cudaStream_t s) const;
  cudaError_t set_params(const float* host, cudaStream_t s);

  // Device-resident training data (features [n][4], targets [n]).
  cudaError_t set_data(const float* host_x, const float* host_y, int n, cudaStream_t s);
  cudaError_t set_data_device(const float* dev_x, const float* dev_y, int n, cudaStream_t s);
  // Forward + backward over the data; gradient (flat, parameter layout) and
  // the mean squared error are left on the device.
  cudaError_t grad(cudaStream_t s);
  cudaError_t read_grad(float* host, float* loss, cudaStream_t s);
  // One Adam step from the current gradient.
  cudaError_t adam(float lr, cudaStream_t s);
  // steps x (grad + Adam), replayed as one captured CUDA graph: the graph of a
  // (sample count, steps, learning rate, starting step, buffers) combination
  // is kept and replayed by later fits with the same combination.
  cudaError_t fit(int steps, float lr, cudaStream_t s, float* final_loss);
  // Prediction for n device feature rows.
  cudaError_t predict_device(const float* dev_x, int n, float* dev_out, cudaStream_t s);

  MlpLayout L;

 private:
  cudaError_t reserve(int n);
  cudaError_t step(float lr, bool update, cudaStream_t s);
  void free_all();

  float *params_ = nullptr, *wt_ = nullptr;   // parameters, and each weight matrix transposed ([out][in])
  float *grads_ = nullptr, *m_ = nullptr, *v_ = nullptr;
  float *x_ = nullptr, *y_ = nullptr, *loss_ = nullptr;
  float *part_ = nullptr, *part_loss_ = nullptr;   // per-block gradients [blocks][total], losses [blocks]
  int cap_ = 0, n_ = 0, steps_done_ = 0;
  cudaGraphExec_t fit_exec_ = nullptr;     // the last captured fit and what it was captured for
  int fit_n_ = 0, fit_steps_ = 0, fit_start_ = -1;
  float fit_lr_ = 0.f;
  const float* fit_bufs_[3] = {nullptr, nullptr, nullptr};
};

}  // namespace tomo
