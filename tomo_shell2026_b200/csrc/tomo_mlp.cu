// Training and inference kernels of the surrogate MLP (see tomo_mlp.cuh).
//
// The network is small (33,793 parameters, 128-wide), and the training set
// is a coarse orientation grid (~10^3 samples), so a step is latency-bound,
// not FLOP-bound.  The design keeps a step to two launches:
//
//   k_mlp_block    one CTA per 16 samples: forward pass (activations in
//                  shared memory), loss, backward pass, and that block's
//                  gradient for every parameter written to its own row of a
//                  partial-gradient buffer;
//   k_mlp_reduce   one thread per parameter: the blocks' gradients summed in
//                  block order (deterministic), optionally followed by the
//                  Adam update of the parameter and of its transposed copy.
//
// Weights are row-major [in][out]; the backward pass reads each matrix
// through a transposed copy [out][in] kept in step with the parameters, so
// both passes read weights with consecutive threads on consecutive
// addresses.  FMAs are explicit (the library is built with -fmad=false for
// the exact path; this code is not on it).
#include "tomo_mlp.cuh"

#include <cmath>
#include <cstring>
#include <random>

namespace tomo {

namespace {

constexpr int kSB = 8;           // samples per CTA
constexpr int kQ = kSB / 2;      // samples per thread (two groups of 128 threads)
constexpr int kThreads = 256;
constexpr int kH = kMlpHidden;   // 128
static_assert(kThreads == 2 * kH, "thread mapping assumes two groups of 128");
static_assert(kSB % 8 == 0 && kSB <= 32, "the output layer gives each of the 8 warps kSB / 8 samples");

// Padded row length of the partial-gradient buffer.
__host__ __device__ inline int part_stride(int total) { return (total + 31) / 32 * 32; }

struct alignas(16) Shared {
  float w[kH * kH];          // the 128 x 128 weight matrix in use (W or its transpose)
  float x[kSB][kMlpIn];
  float a[3][kSB][kH];       // tanh outputs of the three hidden layers
  float dz[2][kSB][kH];      // pre-activation gradients, ping-pong
  float yhat[kSB];
  float dz4[kSB];
};
constexpr size_t kSmemBytes = sizeof(Shared);   // ~106 KB: dynamic, opted in

__device__ __forceinline__ Shared& shared_block()
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  return *reinterpret_cast<Shared*>(smem_raw);
}

// Stage one 128 x 128 matrix into S.w (the caller synchronises).
__device__ __forceinline__ void stage(const float* __restrict__ src, Shared& S)
{
  const float4* s4 = reinterpret_cast<const float4*>(src);
  float4* d4 = reinterpret_cast<float4*>(S.w);
  for (int k = threadIdx.x; k < kH * kH / 4; k += blockDim.x) d4[k] = s4[k];
}

// Forward pass of one block of samples; rows s >= ns hold zero features.
__device__ void forward_block(const MlpLayout& L, const float* __restrict__ P, Shared& S)
{
  const int t = threadIdx.x, j = t & (kH - 1), g = t >> 7;
  {
    const float* W = P + L.w[0];
    const float b = P[L.b[0] + j];
#pragma unroll
    for (int q = 0; q < kQ; q++) {
      const int s = g * kQ + q;
      float acc = b;
#pragma unroll
      for (int i = 0; i < kMlpIn; i++) acc = __fmaf_rn(S.x[s][i], W[i * kH + j], acc);
      S.a[0][s][j] = tanhf(acc);
    }
  }
  __syncthreads();
  for (int l = 1; l < 3; l++) {
    stage(P + L.w[l], S);
    __syncthreads();
    const float* W = S.w;
    float acc[kQ];
    const float b = P[L.b[l] + j];
#pragma unroll
    for (int q = 0; q < kQ; q++) acc[q] = b;
#pragma unroll 4
    for (int i = 0; i < kH; i += 4) {
      const float w0 = W[(i + 0) * kH + j], w1 = W[(i + 1) * kH + j];
      const float w2 = W[(i + 2) * kH + j], w3 = W[(i + 3) * kH + j];
#pragma unroll
      for (int q = 0; q < kQ; q++) {
        const float4 a = *reinterpret_cast<const float4*>(&S.a[l - 1][g * kQ + q][i]);
        acc[q] = __fmaf_rn(a.x, w0, acc[q]);
        acc[q] = __fmaf_rn(a.y, w1, acc[q]);
        acc[q] = __fmaf_rn(a.z, w2, acc[q]);
        acc[q] = __fmaf_rn(a.w, w3, acc[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < kQ; q++) S.a[l][g * kQ + q][j] = tanhf(acc[q]);
    __syncthreads();
  }
  {
    const float* W = P + L.w[3];
    const int warp = t >> 5, lane = t & 31;
    for (int s = warp * (kSB / 8); s < (warp + 1) * (kSB / 8); s++) {
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < kH / 32; k++) acc = __fmaf_rn(S.a[2][s][lane + 32 * k], W[lane + 32 * k], acc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
      if (lane == 0) S.yhat[s] = acc + P[L.b[3]];
    }
  }
  __syncthreads();
}

__device__ void load_x(const float* __restrict__ x, int s0, int ns, Shared& S)
{
  for (int k = threadIdx.x; k < kSB * kMlpIn; k += blockDim.x) {
    const int s = k / kMlpIn, i = k % kMlpIn;
    S.x[s][i] = s < ns ? x[(size_t)(s0 + s) * kMlpIn + i] : 0.f;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_mlp_forward(MlpLayout L, const float* __restrict__ P,
                                                          const float* __restrict__ x, int n, float* __restrict__ out)
{
  Shared& S = shared_block();
  const int s0 = blockIdx.x * kSB, ns = min(kSB, n - s0);
  load_x(x, s0, ns, S);
  forward_block(L, P, S);
  if (threadIdx.x < ns) out[s0 + threadIdx.x] = S.yhat[threadIdx.x];
}

// Forward + MSE + backward of one block; gradient row `blockIdx.x` of `part`.
__global__ void __launch_bounds__(kThreads) k_mlp_block(MlpLayout L, const float* __restrict__ P,
                                                        const float* __restrict__ WT, const float* __restrict__ x,
                                                        const float* __restrict__ y, int n, float* __restrict__ part,
                                                        float* __restrict__ part_loss)
{
  Shared& S = shared_block();
  const int t = threadIdx.x, j = t & (kH - 1), g = t >> 7;
  const int s0 = blockIdx.x * kSB, ns = min(kSB, n - s0);
  float* G = part + (size_t)blockIdx.x * part_stride(L.total);
  load_x(x, s0, ns, S);
  forward_block(L, P, S);
  // loss and output-layer gradient
  if (t < 32) {
    float e = 0.f;
    if (t < kSB) {
      const float d = t < ns ? S.yhat[t] - y[s0 + t] : 0.f;
      S.dz4[t] = 2.f * d / (float)n;
      e = d * d / (float)n;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
    if (t == 0) part_loss[blockIdx.x] = e;
  }
  __syncthreads();
  // layer 4 (128 -> 1): dW4, db4, dZ3
  if (t < kH) {
    float acc = 0.f;
#pragma unroll
    for (int s = 0; s < kSB; s++) acc = __fmaf_rn(S.a[2][s][t], S.dz4[s], acc);
    G[L.w[3] + t] = acc;
  }
  if (t == 0) {
    float acc = 0.f;
    for (int s = 0; s < kSB; s++) acc += S.dz4[s];
    G[L.b[3]] = acc;
  }
  {
    const float w = P[L.w[3] + j];
#pragma unroll
    for (int q = 0; q < kQ; q++) {
      const int s = g * kQ + q;
      const float a = S.a[2][s][j];
      S.dz[0][s][j] = S.dz4[s] * w * (1.f - a * a);
    }
  }
  __syncthreads();
  // hidden layers 3 and 2 (128 -> 128): dZ in dz[cur], layer input a[l-1]
  int cur = 0;
  for (int l = 2; l >= 1; l--) {
    stage(WT + L.w[l], S);   // [out][in]
    __syncthreads();
    const float (*A)[kH] = S.a[l - 1];
    const float (*D)[kH] = S.dz[cur];
    {
      float d[kSB];
#pragma unroll
      for (int s = 0; s < kSB; s++) d[s] = D[s][j];
#pragma unroll 4
      for (int k = 0; k < kH / 2; k++) {
        const int i = g + 2 * k;
        float acc = 0.f;
#pragma unroll
        for (int s = 0; s < kSB; s++) acc = __fmaf_rn(A[s][i], d[s], acc);
        G[L.w[l] + i * kH + j] = acc;
      }
    }
    if (t < kH) {
      float acc = 0.f;
#pragma unroll
      for (int s = 0; s < kSB; s++) acc += D[s][t];
      G[L.b[l] + t] = acc;
    }
    {
      const float* Wt = S.w;
      const int i = j;
      float acc[kQ];
#pragma unroll
      for (int q = 0; q < kQ; q++) acc[q] = 0.f;
#pragma unroll 4
      for (int o = 0; o < kH; o += 4) {
        const float w0 = Wt[(o + 0) * kH + i], w1 = Wt[(o + 1) * kH + i];
        const float w2 = Wt[(o + 2) * kH + i], w3 = Wt[(o + 3) * kH + i];
#pragma unroll
        for (int q = 0; q < kQ; q++) {
          const float4 d = *reinterpret_cast<const float4*>(&D[g * kQ + q][o]);
          acc[q] = __fmaf_rn(d.x, w0, acc[q]);
          acc[q] = __fmaf_rn(d.y, w1, acc[q]);
          acc[q] = __fmaf_rn(d.z, w2, acc[q]);
          acc[q] = __fmaf_rn(d.w, w3, acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < kQ; q++) {
        const float a = A[g * kQ + q][i];
        S.dz[cur ^ 1][g * kQ + q][i] = acc[q] * (1.f - a * a);
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  // layer 1 (4 -> 128)
  {
    const float (*D)[kH] = S.dz[cur];
    for (int i = g; i < kMlpIn; i += 2) {
      float acc = 0.f;
#pragma unroll
      for (int s = 0; s < kSB; s++) acc = __fmaf_rn(S.x[s][i], D[s][j], acc);
      G[L.w[0] + i * kH + j] = acc;
    }
    if (t < kH) {
      float acc = 0.f;
#pragma unroll
      for (int s = 0; s < kSB; s++) acc += D[s][t];
      G[L.b[0] + t] = acc;
    }
  }
}

// Transposed-copy index of weight p (or -1 for a bias).
__device__ __forceinline__ int transposed_index(const MlpLayout& L, int p)
{
#pragma unroll
  for (int l = 0; l < kMlpLayers; l++) {
    const int r = p - L.w[l];
    if (r >= 0 && r < L.in[l] * L.out[l]) return L.w[l] + (r % L.out[l]) * L.in[l] + r / L.out[l];
  }
  return -1;
}

__device__ __forceinline__ void adam_update(const MlpLayout& L, int p, float gi, float* P, float* WT, float* m,
                                            float* v, float lr, float bc1, float bc2)
{
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float mi = b1 * m[p] + (1.f - b1) * gi;
  const float vi = b2 * v[p] + (1.f - b2) * gi * gi;
  m[p] = mi;
  v[p] = vi;
  const float np = P[p] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  P[p] = np;
  const int q = transposed_index(L, p);
  if (q >= 0) WT[q] = np;
}

// grad[p] = sum over blocks (fixed order); loss likewise; optional Adam.
// Block (32 parameters) x (8 lanes over the partial rows): lane r sums rows
// r, r + 8, ...; the 8 lane sums are then added in lane order.
__global__ void __launch_bounds__(256) k_mlp_reduce(MlpLayout L, const float* __restrict__ part,
                                                    const float* __restrict__ part_loss, int nblk,
                                                    float* __restrict__ grad, float* __restrict__ loss, int update,
                                                    float* P, float* WT, float* m, float* v, float lr, float bc1,
                                                    float bc2)
{
  __shared__ float red[8][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int p = blockIdx.x * 32 + tx;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float e = 0.f;
    for (int b = 0; b < nblk; b++) e += part_loss[b];
    *loss = e;
  }
  const int stride = part_stride(L.total);
  float gi = 0.f;
  if (p < L.total) {
#pragma unroll 4
    for (int b = ty; b < nblk; b += 8) gi += part[(size_t)b * stride + p];
  }
  red[ty][tx] = gi;
  __syncthreads();
  if (ty != 0 || p >= L.total) return;
  gi = 0.f;
#pragma unroll
  for (int r = 0; r < 8; r++) gi += red[r][tx];
  grad[p] = gi;
  if (update) adam_update(L, p, gi, P, WT, m, v, lr, bc1, bc2);
}

__global__ void __launch_bounds__(256) k_mlp_adam(MlpLayout L, const float* __restrict__ grad, float* P, float* WT,
                                                  float* m, float* v, float lr, float bc1, float bc2)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < L.total) adam_update(L, p, grad[p], P, WT, m, v, lr, bc1, bc2);
}

__global__ void k_features(const float* __restrict__ ypr, int n, float* __restrict__ x)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float y = ypr[(size_t)i * 3 + 0], p = ypr[(size_t)i * 3 + 1];
  float4 f;
  sincosf(y, &f.x, &f.y);
  sincosf(p, &f.z, &f.w);
  reinterpret_cast<float4*>(x)[i] = f;
}

#define MLP_TRY(call)                       \
  do {                                      \
    const cudaError_t e_ = (call);          \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

// Opt the two block kernels into their dynamic shared memory (per device, once).
cudaError_t configure()
{
  static bool done[64];
  int dev = 0;
  MLP_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (done[dev]) return cudaSuccess;
  MLP_TRY(cudaFuncSetAttribute(k_mlp_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  MLP_TRY(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  done[dev] = true;
  return cudaSuccess;
}

std::vector<float> transposed(const MlpLayout& L, const float* p)
{
  std::vector<float> t(p, p + L.total);
  for (int l = 0; l < kMlpLayers; l++)
    for (int i = 0; i < L.in[l]; i++)
      for (int o = 0; o < L.out[l]; o++) t[L.w[l] + o * L.in[l] + i] = p[L.w[l] + i * L.out[l] + o];
  return t;
}

}  // namespace

cudaError_t mlp_features(const float* ypr, int n, float* x, cudaStream_t s)
{
  if (n <= 0) return cudaSuccess;
  k_features<<<(n + 255) / 256, 256, 0, s>>>(ypr, n, x);
  return cudaGetLastError();
}

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
  if (fit_exec_) { cudaGraphExecDestroy(fit_exec_); fit_exec_ = nullptr; }
  for (float** p : {&params_, &wt_, &grads_, &m_, &v_, &x_, &y_, &loss_, &part_, &part_loss_})
    if (*p) { cudaFree(*p); *p = nullptr; }
  cap_ = 0; n_ = 0; steps_done_ = 0;
}

cudaError_t Mlp::init(unsigned seed, cudaStream_t s)
{
  std::vector<float> h(L.total, 0.f);
  std::mt19937 rng(seed);
  for (int l = 0; l < kMlpLayers; l++) {
    const float r = std::sqrt(6.f / (float)(L.in[l] + L.out[l]));
    std::uniform_real_distribution<float> U(-r, r);
    for (int k = 0; k < L.in[l] * L.out[l]; k++) h[L.w[l] + k] = U(rng);
  }
  if (!params_) {
    MLP_TRY(cudaMalloc(&params_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&wt_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&grads_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&m_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&v_, sizeof(float) * L.total));
    MLP_TRY(cudaMalloc(&loss_, sizeof(float)));
  }
  MLP_TRY(cudaMemsetAsync(grads_, 0, sizeof(float) * L.total, s));
  return set_params(h.data(), s);
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
  const std::vector<float> t = transposed(L, host);
  MLP_TRY(cudaMemcpyAsync(params_, host, sizeof(float) * L.total, cudaMemcpyHostToDevice, s));
  MLP_TRY(cudaMemcpyAsync(wt_, t.data(), sizeof(float) * L.total, cudaMemcpyHostToDevice, s));
  MLP_TRY(cudaMemsetAsync(m_, 0, sizeof(float) * L.total, s));
  MLP_TRY(cudaMemsetAsync(v_, 0, sizeof(float) * L.total, s));
  steps_done_ = 0;
  return cudaStreamSynchronize(s);
}

cudaError_t Mlp::reserve(int n)
{
  if (n <= cap_) return cudaSuccess;
  for (float** p : {&x_, &y_, &part_, &part_loss_})
    if (*p) { cudaFree(*p); *p = nullptr; }
  cap_ = 0;
  const size_t c = (size_t)n, nblk = (c + kSB - 1) / kSB;
  MLP_TRY(cudaMalloc(&x_, sizeof(float) * c * kMlpIn));
  MLP_TRY(cudaMalloc(&y_, sizeof(float) * c));
  MLP_TRY(cudaMalloc(&part_, sizeof(float) * nblk * part_stride(L.total)));
  MLP_TRY(cudaMalloc(&part_loss_, sizeof(float) * nblk));
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

cudaError_t Mlp::step(float lr, bool update, cudaStream_t s)
{
  const int n = n_;
  if (n <= 0 || !params_) return cudaErrorInvalidValue;
  const int nblk = (n + kSB - 1) / kSB;
  MLP_TRY(configure());
  k_mlp_block<<<nblk, kThreads, kSmemBytes, s>>>(L, params_, wt_, x_, y_, n, part_, part_loss_);
  MLP_TRY(cudaGetLastError());
  float bc1 = 1.f, bc2 = 1.f;
  if (update) {
    const int t = steps_done_ + 1;
    bc1 = 1.f - std::pow(0.9f, (float)t);
    bc2 = 1.f - std::pow(0.999f, (float)t);
  }
  k_mlp_reduce<<<(L.total + 31) / 32, 256, 0, s>>>(L, part_, part_loss_, nblk, grads_, loss_, update ? 1 : 0,
                                                      params_, wt_, m_, v_, lr, bc1, bc2);
  MLP_TRY(cudaGetLastError());
  if (update) steps_done_++;
  return cudaSuccess;
}

cudaError_t Mlp::grad(cudaStream_t s) { return step(0.f, false, s); }

cudaError_t Mlp::read_grad(float* host, float* loss, cudaStream_t s)
{
  if (host) MLP_TRY(cudaMemcpyAsync(host, grads_, sizeof(float) * L.total, cudaMemcpyDeviceToHost, s));
  if (loss) MLP_TRY(cudaMemcpyAsync(loss, loss_, sizeof(float), cudaMemcpyDeviceToHost, s));
  return cudaStreamSynchronize(s);
}

cudaError_t Mlp::adam(float lr, cudaStream_t s)
{
  if (!params_) return cudaErrorInvalidValue;
  const int t = steps_done_ + 1;
  const float bc1 = 1.f - std::pow(0.9f, (float)t), bc2 = 1.f - std::pow(0.999f, (float)t);
  k_mlp_adam<<<(L.total + 255) / 256, 256, 0, s>>>(L, grads_, params_, wt_, m_, v_, lr, bc1, bc2);
  MLP_TRY(cudaGetLastError());
  steps_done_++;
  return cudaSuccess;
}

cudaError_t Mlp::fit(int steps, float lr, cudaStream_t s, float* final_loss)
{
  if (n_ <= 0 || steps < 0) return cudaErrorInvalidValue;
  if (steps > 0) {
    // Adam's bias corrections are launch arguments, so a graph is tied to
    // the step it starts from as well as to the shapes and buffers
    const bool reuse = fit_exec_ && fit_n_ == n_ && fit_steps_ == steps && fit_lr_ == lr &&
                       fit_start_ == steps_done_ && fit_bufs_[0] == x_ && fit_bufs_[1] == y_ && fit_bufs_[2] == part_;
    if (!reuse) {
      if (fit_exec_) { cudaGraphExecDestroy(fit_exec_); fit_exec_ = nullptr; }
      MLP_TRY(configure());
      const int start = steps_done_;
      MLP_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = cudaSuccess;
      for (int i = 0; i < steps && e == cudaSuccess; i++) e = step(lr, true, s);
      cudaGraph_t g = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(s, &g);
      steps_done_ = start;
      if (e == cudaSuccess) e = e2;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&fit_exec_, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) { fit_exec_ = nullptr; return e; }
      fit_n_ = n_; fit_steps_ = steps; fit_lr_ = lr; fit_start_ = start;
      fit_bufs_[0] = x_; fit_bufs_[1] = y_; fit_bufs_[2] = part_;
    }
    MLP_TRY(cudaGraphLaunch(fit_exec_, s));
    steps_done_ += steps;
  }
  if (final_loss) {
    MLP_TRY(cudaMemcpyAsync(final_loss, loss_, sizeof(float), cudaMemcpyDeviceToHost, s));
    MLP_TRY(cudaStreamSynchronize(s));
  }
  return cudaSuccess;
}

cudaError_t Mlp::predict_device(const float* dev_x, int n, float* dev_out, cudaStream_t s)
{
  if (!params_ || n <= 0) return cudaErrorInvalidValue;
  MLP_TRY(configure());
  k_mlp_forward<<<(n + kSB - 1) / kSB, kThreads, kSmemBytes, s>>>(L, params_, dev_x, n, dev_out);
  return cudaGetLastError();
}

}  // namespace tomo
