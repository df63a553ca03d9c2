// Training and inference kernels of the surrogate MLP (see tomo_mlp.cuh).
//
// One generic tiled GEMM covers every product of a step:
//   forward      A[n][in] . W[in][out]        + bias, tanh or identity
//   weight grad  A^T . dZ     (A stored [n][in], reduction over samples)
//   input grad   dZ . W^T     then * (1 - a^2) (tanh derivative)
// 64x64 output tiles, 16-deep K slices staged in shared memory, 4x4 outputs
// per thread with explicit FMAs (the library is built with -fmad=false for
// the exact path; this code is not on it).
#include "tomo_mlp.cuh"

#include <cmath>
#include <cstring>
#include <random>

namespace tomo {

namespace {

enum : int { kEpiStore = 0, kEpiBiasTanh = 1, kEpiBias = 2, kEpiTanhGrad = 3 };

template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                              const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                              const float* __restrict__ bias, const float* __restrict__ aux)
{
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ float As[BK][BM + 4];
  __shared__ float Bs[BK][BN + 4];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.f;

  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int e = tid; e < BM * BK; e += 256) {
      const int mm = TA ? (e % BM) : (e / BK);
      const int kk = TA ? (e / BM) : (e % BK);
      const int gm = m0 + mm, gk = k0 + kk;
      float v = 0.f;
      if (gm < M && gk < K) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
      As[kk][mm] = v;
    }
    for (int e = tid; e < BK * BN; e += 256) {
      const int nn = TB ? (e / BK) : (e % BN);
      const int kk = TB ? (e % BK) : (e / BN);
      const int gk = k0 + kk, gn = n0 + nn;
      float v = 0.f;
      if (gk < K && gn < N) v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int r = m0 + ty + 16 * i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = n0 + tx + 16 * j;
      if (c >= N) continue;
      float v = acc[i][j];
      if (EPI == kEpiBiasTanh) v = tanhf(v + bias[c]);
      if (EPI == kEpiBias) v = v + bias[c];
      if (EPI == kEpiTanhGrad) { const float t = aux[(size_t)r * ldc + c]; v = v * (1.f - t * t); }
      C[(size_t)r * ldc + c] = v;
    }
  }
}

// out[j] = sum_m D[m][j]  (bias gradients)
__global__ void __launch_bounds__(128) k_colsum(const float* __restrict__ D, int M, int N, float* __restrict__ out)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; m++) s += D[(size_t)m * N + j];
  out[j] = s;
}

// dz = 2 (yhat - y) / n, loss += mean squared error
__global__ void __launch_bounds__(256) k_mse(const float* __restrict__ yhat, const float* __restrict__ y, int n,
                                             float* __restrict__ dz, float* __restrict__ loss)
{
  __shared__ float red[8];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float e = 0.f;
  if (i < n) {
    const float d = yhat[i] - y[i];
    dz[i] = 2.f * d / (float)n;
    e = d * d / (float)n;
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < 8; w++) t += red[w];
    atomicAdd(loss, t);
  }
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8); the step count lives on the
// device so a captured step graph can be replayed.
__global__ void __launch_bounds__(256) k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                              float* __restrict__ v, int n, float lr, const int* __restrict__ step)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float t = (float)(*step + 1);
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.f - powf(b1, t));
  const float vh = vi / (1.f - powf(b2, t));
  p[i] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_step_inc(int* step)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

template <bool TA, bool TB, int EPI>
cudaError_t gemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
                 const float* bias, const float* aux, cudaStream_t s)
{
  if (M <= 0 || N <= 0) return cudaSuccess;
  const dim3 grid((N + 63) / 64, (M + 63) / 64);
  k_gemm<TA, TB, EPI><<<grid, 256, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, aux);
  return cudaGetLastError();
}

#define MLP_TRY(call)                       \
  do {                                      \
    const cudaError_t e_ = (call);          \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

}  // namespace

MlpLayout::MlpLayout()
{
  const int dims[kMlpLayers + 1] = {kMlpIn, kMlpHidden, kMlpHidden, kMlpHidden, 1};
  int off = 0;
  for (int l = 0; l < kMlpLayers; l++) {
    in[l] = dims[l];
    out[l] = dims[l + 1];
    w[l] = off;
    off += in[l] * out[l];
    b[l] = off;
    off += out[l];
  }
  total = off;
}

Mlp::~Mlp() { free_all(); }

void Mlp::free_all()
{
  if (step_exec_) cudaGraphExecDestroy(step_exec_);
  if (step_graph_) cudaGraphDestroy(step_graph_);
  step_exec_ = nullptr; step_graph_ = nullptr;
  for (float** p : {&params_, &grads_, &m_, &v_, &x_, &y_, &loss_, &act_[0], &act_[1], &act_[2], &act_[3], &dz_[0], &dz_[1]})
    if (*p) { cudaFree(*p); *p = nullptr; }
  if (step_) { cudaFree(step_); step_ = nullptr; }
  cap_ = 0; n_ = 0;
}

cudaError_t Mlp::init(unsigned seed, cudaStream_t s)
{
  if (!params_) {
    MLP_TRY(cudaMalloc(&params_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&grads_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&m_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&v_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&loss_, sizeof(float)));
    MLP_TRY(cudaMalloc(&step_, sizeof(int)));
  }
  std::vector<float> h(L.total, 0.f);
  std::mt19937 rng(seed);
  for (int l = 0; l < kMlpLayers; l++) {
    const float r = std::sqrt(6.f / (float)(L.in[l] + L.out[l]));
    std::uniform_real_distribution<float> U(-r, r);
    for (int k = 0; k < L.in[l] * L.out[l]; k++) h[L.w[l] + k] = U(rng);
  }
  MLP_TRY(cudaMemcpyAsync(params_, h.data(), sizeof(float) * L.total, cudaMemcpyHostToDevice, s));
  MLP_TRY(cudaMemsetAsync(grads_, 0, sizeof(float) * L.total, s));
  MLP_TRY(cudaMemsetAsync(m_, 0, sizeof(float) * L.total, s));
  MLP_TRY(cudaMemsetAsync(v_, 0, sizeof(float) * L.total, s));
  MLP_TRY(cudaMemsetAsync(step_, 0, sizeof(int), s));
  return cudaStreamSynchronize(s);
}

cudaError_t Mlp::get_params(float* host, cudaStream_t s) const
{
  if (!params_) return cudaErrorInvalidValue;
  MLP_TRY(cudaMemcpyAsync(host, params_, sizeof(float) * L.total, cudaMemcpyDeviceToHost, s));
  return cudaStreamSynchronize(s);
}

cudaError_t Mlp::set_params(const float* host, cudaStream_t s)
{
  if (!params_) return cudaErrorInvalidValue;
  MLP_TRY(cudaMemcpyAsync(params_, host, sizeof(float) * L.total, cudaMemcpyHostToDevice, s));
  MLP_TRY(cudaMemsetAsync(m_, 0, sizeof(float) * L.total, s));
  MLP_TRY(cudaMemsetAsync(v_, 0, sizeof(float) * L.total, s));
  MLP_TRY(cudaMemsetAsync(step_, 0, sizeof(int), s));
  return cudaStreamSynchronize(s);
}

cudaError_t Mlp::reserve(int n)
{
  if (n <= cap_) return cudaSuccess;
  if (step_exec_) { cudaGraphExecDestroy(step_exec_); step_exec_ = nullptr; }
  if (step_graph_) { cudaGraphDestroy(step_graph_); step_graph_ = nullptr; }
  for (float** p : {&x_, &y_, &act_[0], &act_[1], &act_[2], &act_[3], &dz_[0], &dz_[1]})
    if (*p) { cudaFree(*p); *p = nullptr; }
  cap_ = 0;
  const size_t c = (size_t)n;
  MLP_TRY(cudaMalloc(&x_, sizeof(float) * c * kMlpIn));
  MLP_TRY(cudaMalloc(&y_, sizeof(float) * c));
  for (int l = 0; l < 3; l++) MLP_TRY(cudaMalloc(&act_[l], sizeof(float) * c * kMlpHidden));
  MLP_TRY(cudaMalloc(&act_[3], sizeof(float) * c));
  MLP_TRY(cudaMalloc(&dz_[0], sizeof(float) * c * kMlpHidden));
  MLP_TRY(cudaMalloc(&dz_[1], sizeof(float) * c * kMlpHidden));
  cap_ = n;
  return cudaSuccess;
}

cudaError_t Mlp::set_data(const float* host_x, const float* host_y, int n, cudaStream_t s)
{
  if (!params_ || n <= 0) return cudaErrorInvalidValue;
  MLP_TRY(reserve(n));
  MLP_TRY(cudaMemcpyAsync(x_, host_x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice, s));
  MLP_TRY(cudaMemcpyAsync(y_, host_y, sizeof(float) * n, cudaMemcpyHostToDevice, s));
  n_ = n;
  return cudaStreamSynchronize(s);
}

cudaError_t Mlp::set_data_device(const float* dev_x, const float* dev_y, int n, cudaStream_t s)
{
  if (!params_ || n <= 0) return cudaErrorInvalidValue;
  MLP_TRY(reserve(n));
  MLP_TRY(cudaMemcpyAsync(x_, dev_x, sizeof(float) * n * kMlpIn, cudaMemcpyDeviceToDevice, s));
  MLP_TRY(cudaMemcpyAsync(y_, dev_y, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
  n_ = n;
  return cudaSuccess;
}

cudaError_t Mlp::forward(const float* x, int n, float* out, cudaStream_t s)
{
  const float* in = x;
  for (int l = 0; l < 3; l++) {
    MLP_TRY((gemm<false, false, kEpiBiasTanh>(n, L.out[l], L.in[l], in, L.in[l], params_ + L.w[l], L.out[l], act_[l],
                                              L.out[l], params_ + L.b[l], nullptr, s)));
    in = act_[l];
  }
  return gemm<false, false, kEpiBias>(n, 1, kMlpHidden, in, kMlpHidden, params_ + L.w[3], 1, out, 1, params_ + L.b[3],
                                      nullptr, s);
}

cudaError_t Mlp::grad(cudaStream_t s)
{
  const int n = n_;
  if (n <= 0) return cudaErrorInvalidValue;
  MLP_TRY(forward(x_, n, act_[3], s));
  MLP_TRY(cudaMemsetAsync(loss_, 0, sizeof(float), s));
  k_mse<<<(n + 255) / 256, 256, 0, s>>>(act_[3], y_, n, dz_[0], loss_);
  MLP_TRY(cudaGetLastError());
  // dZ of layer l lives in dz[cur]; layer inputs are x (l = 0) or act[l-1]
  int cur = 0;
  for (int l = kMlpLayers - 1; l >= 0; l--) {
    const float* a_in = l == 0 ? x_ : act_[l - 1];
    const int fin = L.in[l], fout = L.out[l];
    MLP_TRY((gemm<true, false, kEpiStore>(fin, fout, n, a_in, fin, dz_[cur], fout, grads_ + L.w[l], fout, nullptr,
                                          nullptr, s)));
    k_colsum<<<(fout + 127) / 128, 128, 0, s>>>(dz_[cur], n, fout, grads_ + L.b[l]);
    MLP_TRY(cudaGetLastError());
    if (l > 0) {
      MLP_TRY((gemm<false, true, kEpiTanhGrad>(n, fin, fout, dz_[cur], fout, params_ + L.w[l], fout, dz_[cur ^ 1], fin,
                                               nullptr, act_[l - 1], s)));
      cur ^= 1;
    }
  }
  return cudaSuccess;
}

cudaError_t Mlp::read_grad(float* host, float* loss, cudaStream_t s)
{
  if (host) MLP_TRY(cudaMemcpyAsync(host, grads_, sizeof(float) * L.total, cudaMemcpyDeviceToHost, s));
  if (loss) MLP_TRY(cudaMemcpyAsync(loss, loss_, sizeof(float), cudaMemcpyDeviceToHost, s));
  return cudaStreamSynchronize(s);
}

cudaError_t Mlp::adam(float lr, cudaStream_t s)
{
  k_adam<<<(L.total + 255) / 256, 256, 0, s>>>(params_, grads_, m_, v_, L.total, lr, step_);
  MLP_TRY(cudaGetLastError());
  k_step_inc<<<1, 32, 0, s>>>(step_);
  return cudaGetLastError();
}

cudaError_t Mlp::fit(int steps, float lr, cudaStream_t s, float* final_loss)
{
  if (n_ <= 0 || steps < 0) return cudaErrorInvalidValue;
  if (!step_exec_ || step_lr_ != lr || step_n_ != n_) {
    if (step_exec_) { cudaGraphExecDestroy(step_exec_); step_exec_ = nullptr; }
    if (step_graph_) { cudaGraphDestroy(step_graph_); step_graph_ = nullptr; }
    MLP_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = grad(s);
    if (e == cudaSuccess) e = adam(lr, s);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return e; }
    MLP_TRY(e2);
    step_graph_ = g;
    MLP_TRY(cudaGraphInstantiate(&step_exec_, step_graph_, 0));
    step_lr_ = lr;
    step_n_ = n_;
  }
  for (int i = 0; i < steps; i++) MLP_TRY(cudaGraphLaunch(step_exec_, s));
  if (final_loss) {
    MLP_TRY(cudaMemcpyAsync(final_loss, loss_, sizeof(float), cudaMemcpyDeviceToHost, s));
    MLP_TRY(cudaStreamSynchronize(s));
  }
  return cudaSuccess;
}

cudaError_t Mlp::predict_device(const float* dev_x, int n, float* dev_out, cudaStream_t s)
{
  if (!params_ || n <= 0) return cudaErrorInvalidValue;
  MLP_TRY(reserve(n));
  return forward(dev_x, n, dev_out, s);
}

}  // namespace tomo
