// mlp.cu -- the learned warm start's network: a dense MLP with GELU hidden layers,
// trained and evaluated by this library's own kernels in FP32.
//
// Layout: one parameter vector P = [W1 (H x I), b1 (H), W2 (H x H), b2 (H),
// W3 (O x H), b3 (O)], row-major weights, and gradient / Adam moments of the same shape.
// Activations are row-major [batch][width].  Every reduction (GEMM inner products,
// bias-gradient column sums, the loss) runs in a fixed order, so training is bitwise
// reproducible for a given seed.
//
// Kernels: one tiled FP32 GEMM with arbitrary operand strides serves the forward pass
// (bias + GELU fused into its epilogue, pre-activations kept for the backward pass), the
// weight gradients (A^T B shapes) and the back-propagated deltas (GELU' fused); column
// sums give bias gradients; one elementwise kernel applies Adam.  GELU is the exact
// erf form, 0.5 x (1 + erf(x / sqrt 2)).
#include "mlp.h"

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

namespace fg
{
namespace
{

constexpr int kTile = 32;    // GEMM output tile (kTile x kTile) per 256-thread CTA
constexpr int kTileK = 16;   // inner-dimension slab staged in shared memory
constexpr int kThreads = 256;

enum Epilogue : int { kStore = 0, kBiasGelu = 1, kBias = 2, kGeluGrad = 3 };

__device__ __forceinline__ float Gelu(float x)
{
  return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float GeluGrad(float x)
{
  const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// C(m, n) = epilogue(sum_k A(m, k) B(k, n)), A(m, k) = A[m * am + k * ak],
// B(k, n) = B[k * bk + n * bn], C row-major with leading dimension ldc.
// kBiasGelu: pre = acc + bias[n] -> aux(m, n) = pre, C = GELU(pre);  kBias: C = acc + bias[n];
// kGeluGrad: C = acc * GELU'(aux(m, n)).
__global__ void __launch_bounds__(kThreads)
    GemmKernel(int M, int N, int K, const float *__restrict__ A, int am, int ak,
               const float *__restrict__ B, int bk, int bn, float *__restrict__ C, int ldc,
               int epilogue, const float *__restrict__ bias, float *__restrict__ aux)
{
  __shared__ float As[kTileK][kTile + 1];
  __shared__ float Bs[kTileK][kTile + 1];
  const int tx = threadIdx.x % kTile, ty = threadIdx.x / kTile; // ty in [0, 8)
  const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += kTileK) {
    for (int t = threadIdx.x; t < kTileK * kTile; t += kThreads) {
      const int kk = t / kTile, mm = t % kTile;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? A[static_cast<size_t>(m) * am + static_cast<size_t>(k) * ak] : 0.f;
      const int n = n0 + mm;
      Bs[kk][mm] = (n < N && k < K) ? B[static_cast<size_t>(k) * bk + static_cast<size_t>(n) * bn] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTileK; ++kk) {
      const float b = Bs[kk][tx];
#pragma unroll
      for (int i = 0; i < 4; ++i)
        acc[i] = fmaf(As[kk][ty + 8 * i], b, acc[i]);
    }
    __syncthreads();
  }
  const int n = n0 + tx;
  if (n >= N)
    return;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 8 * i;
    if (m >= M)
      continue;
    const size_t o = static_cast<size_t>(m) * ldc + n;
    float v = acc[i];
    if (epilogue == kBiasGelu) {
      v += bias[n];
      aux[o] = v;
      v = Gelu(v);
    } else if (epilogue == kBias) {
      v += bias[n];
    } else if (epilogue == kGeluGrad) {
      v *= GeluGrad(aux[o]);
    }
    C[o] = v;
  }
}

// out[n] = sum over rows m of X[m][n] (fixed row order), for bias gradients.
__global__ void ColumnSumKernel(int M, int N, const float *__restrict__ X, float *__restrict__ out)
{
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N)
    return;
  float s = 0.f;
  for (int m = 0; m < M; ++m)
    s += X[static_cast<size_t>(m) * N + n];
  out[n] = s;
}

// d = (y - t) / batch, and per-row partial 0.5 * sum (y - t)^2 for the loss.
__global__ void OutputDeltaKernel(int batch, int O, const float *__restrict__ y,
                                  const float *__restrict__ t, float *__restrict__ d,
                                  float *__restrict__ row_loss)
{
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch)
    return;
  float l = 0.f;
  for (int o = 0; o < O; ++o) {
    const size_t i = static_cast<size_t>(b) * O + o;
    const float e = y[i] - t[i];
    d[i] = e / static_cast<float>(batch);
    l += e * e;
  }
  row_loss[b] = 0.5f * l;
}

__global__ void SumKernel(int n, const float *__restrict__ x, float scale, float *__restrict__ out)
{
  if (blockIdx.x != 0 || threadIdx.x != 0)
    return;
  float s = 0.f;
  for (int i = 0; i < n; ++i)
    s += x[i];
  *out = s * scale;
}

__global__ void GatherRowsKernel(int rows, int width, const int32_t *__restrict__ index,
                                 const float *__restrict__ src, float *__restrict__ dst)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(rows) * width)
    return;
  const int r = static_cast<int>(t / width), c = static_cast<int>(t % width);
  dst[t] = src[static_cast<size_t>(index[r]) * width + c];
}

// Adam (Kingma & Ba 2015) with bias correction folded into the step size.
__global__ void AdamKernel(int64_t n, float *__restrict__ p, const float *__restrict__ g,
                           float *__restrict__ m, float *__restrict__ v, float lr_t, float beta1,
                           float beta2, float eps)
{
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const float gi = g[i];
  const float mi = beta1 * m[i] + (1.f - beta1) * gi;
  const float vi = beta2 * v[i] + (1.f - beta2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr_t * mi / (sqrtf(vi) + eps);
}

unsigned Grid(size_t threads, int block) { return static_cast<unsigned>((threads + block - 1) / block); }

cudaError_t Gemm(int M, int N, int K, const float *A, int am, int ak, const float *B, int bk, int bn,
                 float *C, int ldc, int epilogue, const float *bias, float *aux, cudaStream_t st)
{
  const dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  GemmKernel<<<grid, kThreads, 0, st>>>(M, N, K, A, am, ak, B, bk, bn, C, ldc, epilogue, bias, aux);
  return cudaGetLastError();
}

} // namespace

Status Mlp::Create(int inputs, int hidden, int outputs, uint64_t seed)
{
  if (inputs < 1 || hidden < 1 || outputs < 1 || inputs > 4096 || hidden > 4096 || outputs > 4096)
    return Status::kInvalidArgument;
  I_ = inputs;
  H_ = hidden;
  O_ = outputs;
  const int64_t n = ParameterCount();
  Status s;
  if ((s = p_.ensure(n)) != Status::kOk || (s = g_.ensure(n)) != Status::kOk ||
      (s = m_.ensure(n)) != Status::kOk || (s = v_.ensure(n)) != Status::kOk)
    return s;
  // Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases from a seeded generator.
  std::mt19937_64 rng(seed);
  std::vector<float> host(n);
  size_t o = 0;
  auto fill = [&](int rows, int fan_in) {
    std::uniform_real_distribution<float> u(-1.0f / std::sqrt(float(fan_in)), 1.0f / std::sqrt(float(fan_in)));
    for (int i = 0; i < rows * fan_in; ++i)
      host[o++] = u(rng);
    for (int i = 0; i < rows; ++i)
      host[o++] = u(rng);
  };
  fill(H_, I_);
  fill(H_, H_);
  fill(O_, H_);
  if ((s = p_.upload(host.data(), n)) != Status::kOk)
    return s;
  steps_ = 0;
  return cudaMemset(m_.get(), 0, n * sizeof(float)) == cudaSuccess &&
                 cudaMemset(v_.get(), 0, n * sizeof(float)) == cudaSuccess &&
                 cudaDeviceSynchronize() == cudaSuccess
             ? Status::kOk
             : Status::kInternalError;
}

int64_t Mlp::ParameterCount() const
{
  return static_cast<int64_t>(H_) * I_ + H_ + static_cast<int64_t>(H_) * H_ + H_ +
         static_cast<int64_t>(O_) * H_ + O_;
}

Status Mlp::EnsureBatch(int batch)
{
  if (batch <= batch_cap_)
    return Status::kOk;
  Status s;
  const size_t b = batch;
  if ((s = x_.ensure(b * I_)) != Status::kOk || (s = t_.ensure(b * O_)) != Status::kOk ||
      (s = h1_.ensure(b * H_)) != Status::kOk || (s = a1_.ensure(b * H_)) != Status::kOk ||
      (s = h2_.ensure(b * H_)) != Status::kOk || (s = a2_.ensure(b * H_)) != Status::kOk ||
      (s = y_.ensure(b * O_)) != Status::kOk || (s = dy_.ensure(b * O_)) != Status::kOk ||
      (s = d2_.ensure(b * H_)) != Status::kOk || (s = d1_.ensure(b * H_)) != Status::kOk ||
      (s = row_loss_.ensure(b)) != Status::kOk || (s = loss_.ensure(1)) != Status::kOk)
    return s;
  batch_cap_ = batch;
  return Status::kOk;
}

// Pointers into the parameter-shaped vector q (P, G or a moment).
Mlp::Views Mlp::Split(float *q) const
{
  Views v;
  v.w1 = q;
  v.b1 = v.w1 + static_cast<size_t>(H_) * I_;
  v.w2 = v.b1 + H_;
  v.b2 = v.w2 + static_cast<size_t>(H_) * H_;
  v.w3 = v.b2 + H_;
  v.b3 = v.w3 + static_cast<size_t>(O_) * H_;
  return v;
}

// y = f(x) for `batch` rows of x (device), keeping pre-activations for Backward.
Status Mlp::Forward(int batch, const float *x, float *y, cudaStream_t st)
{
  const Views w = Split(p_.get());
  // h1 = GELU(x W1^T + b1): A = x [b][i], B(k=i, n=h) = W1[h][i].
  if (Gemm(batch, H_, I_, x, I_, 1, w.w1, 1, I_, a1_.get(), H_, kBiasGelu, w.b1, h1_.get(), st) != cudaSuccess ||
      Gemm(batch, H_, H_, a1_.get(), H_, 1, w.w2, 1, H_, a2_.get(), H_, kBiasGelu, w.b2, h2_.get(), st) != cudaSuccess ||
      Gemm(batch, O_, H_, a2_.get(), H_, 1, w.w3, 1, H_, y, O_, kBias, w.b3, nullptr, st) != cudaSuccess)
    return Status::kInternalError;
  launches_ += 3;
  return Status::kOk;
}

// Gradient of 0.5 / batch * sum (y - t)^2 into g_, after Forward(x) -> y_.
Status Mlp::Backward(int batch, const float *x, const float *t, cudaStream_t st)
{
  const Views w = Split(p_.get());
  const Views g = Split(g_.get());
  OutputDeltaKernel<<<Grid(batch, 128), 128, 0, st>>>(batch, O_, y_.get(), t, dy_.get(), row_loss_.get());
  // dW3 = dy^T a2 (O x H), db3 = colsum(dy); d2 = (dy W3) * GELU'(h2).
  if (cudaGetLastError() != cudaSuccess ||
      Gemm(O_, H_, batch, dy_.get(), 1, O_, a2_.get(), H_, 1, g.w3, H_, kStore, nullptr, nullptr, st) != cudaSuccess)
    return Status::kInternalError;
  ColumnSumKernel<<<Grid(O_, 128), 128, 0, st>>>(batch, O_, dy_.get(), g.b3);
  if (cudaGetLastError() != cudaSuccess ||
      Gemm(batch, H_, O_, dy_.get(), O_, 1, w.w3, H_, 1, d2_.get(), H_, kGeluGrad, nullptr, h2_.get(), st) != cudaSuccess ||
      Gemm(H_, H_, batch, d2_.get(), 1, H_, a1_.get(), H_, 1, g.w2, H_, kStore, nullptr, nullptr, st) != cudaSuccess)
    return Status::kInternalError;
  ColumnSumKernel<<<Grid(H_, 128), 128, 0, st>>>(batch, H_, d2_.get(), g.b2);
  if (cudaGetLastError() != cudaSuccess ||
      Gemm(batch, H_, H_, d2_.get(), H_, 1, w.w2, H_, 1, d1_.get(), H_, kGeluGrad, nullptr, h1_.get(), st) != cudaSuccess ||
      Gemm(H_, I_, batch, d1_.get(), 1, H_, x, I_, 1, g.w1, I_, kStore, nullptr, nullptr, st) != cudaSuccess)
    return Status::kInternalError;
  ColumnSumKernel<<<Grid(H_, 128), 128, 0, st>>>(batch, H_, d1_.get(), g.b1);
  if (cudaGetLastError() != cudaSuccess)
    return Status::kInternalError;
  launches_ += 9;
  return Status::kOk;
}

Status Mlp::Predict(int batch, const float *x_host, float *y_host)
{
  if (batch < 1 || !x_host || !y_host)
    return Status::kInvalidArgument;
  Status s = EnsureBatch(batch);
  if (s != Status::kOk || (s = x_.upload(x_host, static_cast<size_t>(batch) * I_)) != Status::kOk ||
      (s = Forward(batch, x_.get(), y_.get(), nullptr)) != Status::kOk)
    return s;
  return cudaMemcpy(y_host, y_.get(), sizeof(float) * batch * O_, cudaMemcpyDeviceToHost) == cudaSuccess
             ? Status::kOk
             : Status::kInternalError;
}

Status Mlp::PredictDevice(int batch, const float *x_dev, float *y_dev, cudaStream_t st)
{
  Status s = EnsureBatch(batch);
  if (s != Status::kOk)
    return s;
  return Forward(batch, x_dev, y_dev, st);
}

Status Mlp::LossGradient(int batch, const float *x_host, const float *t_host, float *loss,
                         float *gradient_host)
{
  if (batch < 1 || !x_host || !t_host)
    return Status::kInvalidArgument;
  Status s = EnsureBatch(batch);
  if (s != Status::kOk || (s = x_.upload(x_host, static_cast<size_t>(batch) * I_)) != Status::kOk ||
      (s = t_.upload(t_host, static_cast<size_t>(batch) * O_)) != Status::kOk ||
      (s = Forward(batch, x_.get(), y_.get(), nullptr)) != Status::kOk ||
      (s = Backward(batch, x_.get(), t_.get(), nullptr)) != Status::kOk)
    return s;
  SumKernel<<<1, 1>>>(batch, row_loss_.get(), 1.0f / batch, loss_.get());
  if (cudaGetLastError() != cudaSuccess)
    return Status::kInternalError;
  if (loss && cudaMemcpy(loss, loss_.get(), sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return Status::kInternalError;
  if (gradient_host && cudaMemcpy(gradient_host, g_.get(), sizeof(float) * ParameterCount(),
                                  cudaMemcpyDeviceToHost) != cudaSuccess)
    return Status::kInternalError;
  return Status::kOk;
}

Status Mlp::Train(int samples, const float *x_host, const float *t_host, int epochs, int batch,
                  float learning_rate, uint64_t seed, float *final_loss)
{
  if (samples < 1 || epochs < 0 || batch < 1 || !x_host || !t_host || !(learning_rate > 0.f))
    return Status::kInvalidArgument;
  batch = std::min(batch, samples);
  Status s = EnsureBatch(std::max(batch, samples));
  DeviceArray<float> xs, ts;
  DeviceArray<int32_t> perm;
  if (s != Status::kOk || (s = xs.upload(x_host, static_cast<size_t>(samples) * I_)) != Status::kOk ||
      (s = ts.upload(t_host, static_cast<size_t>(samples) * O_)) != Status::kOk ||
      (s = perm.ensure(samples)) != Status::kOk)
    return s;
  std::mt19937_64 rng(seed);
  std::vector<int32_t> order(samples);
  constexpr float kBeta1 = 0.9f, kBeta2 = 0.999f, kEps = 1e-8f;
  const int64_t n = ParameterCount();
  for (int epoch = 0; epoch < epochs; ++epoch) {
    for (int i = 0; i < samples; ++i)
      order[i] = i;
    std::shuffle(order.begin(), order.end(), rng);
    if ((s = perm.upload(order.data(), samples)) != Status::kOk)
      return s;
    for (int first = 0; first + batch <= samples; first += batch) {
      GatherRowsKernel<<<Grid(static_cast<size_t>(batch) * I_, kThreads), kThreads>>>(
          batch, I_, perm.get() + first, xs.get(), x_.get());
      GatherRowsKernel<<<Grid(static_cast<size_t>(batch) * O_, kThreads), kThreads>>>(
          batch, O_, perm.get() + first, ts.get(), t_.get());
      if (cudaGetLastError() != cudaSuccess ||
          (s = Forward(batch, x_.get(), y_.get(), nullptr)) != Status::kOk ||
          (s = Backward(batch, x_.get(), t_.get(), nullptr)) != Status::kOk)
        return s != Status::kOk ? s : Status::kInternalError;
      ++steps_;
      const double c1 = 1.0 - std::pow(double(kBeta1), double(steps_));
      const double c2 = 1.0 - std::pow(double(kBeta2), double(steps_));
      const float lr_t = static_cast<float>(learning_rate * std::sqrt(c2) / c1);
      AdamKernel<<<Grid(n, kThreads), kThreads>>>(n, p_.get(), g_.get(), m_.get(), v_.get(), lr_t,
                                                  kBeta1, kBeta2, kEps);
      if (cudaGetLastError() != cudaSuccess)
        return Status::kInternalError;
      launches_ += 3;
    }
  }
  // Loss over the whole training set with the final parameters.
  if ((s = Forward(samples, xs.get(), y_.get(), nullptr)) != Status::kOk ||
      (s = Backward(samples, xs.get(), ts.get(), nullptr)) != Status::kOk)
    return s;
  SumKernel<<<1, 1>>>(samples, row_loss_.get(), 1.0f / samples, loss_.get());
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
    return Status::kInternalError;
  if (final_loss && cudaMemcpy(final_loss, loss_.get(), sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return Status::kInternalError;
  return Status::kOk;
}

Status Mlp::GetParameters(float *host) const
{
  return cudaMemcpy(host, p_.get(), sizeof(float) * ParameterCount(), cudaMemcpyDeviceToHost) == cudaSuccess
             ? Status::kOk
             : Status::kInternalError;
}

Status Mlp::SetParameters(const float *host)
{
  Status s = p_.upload(host, ParameterCount());
  if (s != Status::kOk)
    return s;
  return cudaDeviceSynchronize() == cudaSuccess ? Status::kOk : Status::kInternalError;
}

} // namespace fg
