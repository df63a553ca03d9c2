// Surrogate network of the learned-proposal orientation search: an FP32 MLP
// [sin yaw, cos yaw, sin pitch, cos pitch] -> 128 -> 128 -> 128 -> Vss with
// tanh hidden units and a linear output, trained full-batch with Adam by the
// hand-written kernels of tomo_mlp.cu (tiled SIMT GEMMs with fused bias /
// activation / activation-derivative epilogues, column sums, MSE gradient,
// Adam).  Nothing here is a dense contraction large enough for tensor cores:
// one training step is ~60 MFLOP.
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
  // steps x (grad + Adam), replayed from one captured CUDA graph per step.
  cudaError_t fit(int steps, float lr, cudaStream_t s, float* final_loss);
  // Prediction for n device feature rows.
  cudaError_t predict_device(const float* dev_x, int n, float* dev_out, cudaStream_t s);

  MlpLayout L;

 private:
  cudaError_t reserve(int n);
  cudaError_t forward(const float* x, int n, float* out, cudaStream_t s);
  void free_all();

  float *params_ = nullptr, *grads_ = nullptr, *m_ = nullptr, *v_ = nullptr;
  float *x_ = nullptr, *y_ = nullptr, *loss_ = nullptr;
  float *act_[kMlpLayers] = {nullptr, nullptr, nullptr, nullptr};   // tanh outputs of layers 1..3, output of layer 4
  float *dz_[2] = {nullptr, nullptr};
  int* step_ = nullptr;
  int cap_ = 0, n_ = 0;
  cudaGraphExec_t step_exec_ = nullptr;
  cudaGraph_t step_graph_ = nullptr;
  float step_lr_ = -1.f;
  int step_n_ = -1;
};

}  // namespace tomo
