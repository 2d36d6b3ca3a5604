// warm.cu -- the learned warm start: a reduced basis of A (mean + r orthonormal modes,
// FP64) whose coefficients a small MLP predicts from a sample's features.
//
//   features f [k][I] --(f - shift) / scale--> MLP (FP32) --> y [k][r]
//   c = coeff_shift + coeff_scale * y;   A = mean + sum_r c_r phi_r   (FP64)
//
// The Newton solve then starts from A under the residual guard of the solver: an item whose
// equation residual at A is not below the zero start's falls back to the zero start, and
// every item finishes at the unchanged tolerances.  Projection c = Phi (a - mean) gives
// the training targets from solved samples.
#include "warm.h"

#include <algorithm>
#include <vector>

namespace fg
{
namespace
{

constexpr int kThreads = 256;
constexpr int kExpandItems = 8;

__global__ void NormalizeKernel(int k, int inputs, const float *__restrict__ f,
                                const float *__restrict__ shift, const float *__restrict__ scale,
                                float *__restrict__ out)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k * inputs)
    return;
  const int i = t % inputs;
  out[t] = (f[t] - shift[i]) / scale[i];
}

// a[item][node] = mean[node] + sum_q c(item, q) phi_q[node], c = shift + scale * y.
__global__ void __launch_bounds__(kThreads)
    ExpandKernel(int N, int rank, int k, const double *__restrict__ mean,
                 const double *__restrict__ basis, const float *__restrict__ y,
                 const double *__restrict__ shift, const double *__restrict__ scale,
                 double *__restrict__ a)
{
  extern __shared__ double coef[]; // [kExpandItems][rank]
  const int item0 = blockIdx.y * kExpandItems;
  const int items = min(kExpandItems, k - item0);
  for (int t = threadIdx.x; t < kExpandItems * rank; t += blockDim.x) {
    const int j = t / rank, q = t % rank;
    coef[t] = j < items ? shift[q] + scale[q] * static_cast<double>(y[static_cast<size_t>(item0 + j) * rank + q])
                        : 0.0;
  }
  __syncthreads();
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N)
    return;
  double acc[kExpandItems];
  const double m = mean[node];
#pragma unroll
  for (int j = 0; j < kExpandItems; ++j)
    acc[j] = m;
  for (int q = 0; q < rank; ++q) {
    const double phi = basis[static_cast<size_t>(q) * N + node];
#pragma unroll
    for (int j = 0; j < kExpandItems; ++j)
      acc[j] = fma(coef[j * rank + q], phi, acc[j]);
  }
  for (int j = 0; j < items; ++j)
    a[static_cast<size_t>(item0 + j) * N + node] = acc[j];
}

// coeffs[item][q] = sum_node phi_q[node] (a[item][node] - mean[node]); one CTA per (q, item),
// fixed striding and tree order.
__global__ void __launch_bounds__(kThreads)
    ProjectKernel(int N, int rank, const double *__restrict__ mean, const double *__restrict__ basis,
                  const double *__restrict__ a, double *__restrict__ coeffs)
{
  __shared__ double red[kThreads];
  const int q = blockIdx.x, item = blockIdx.y;
  const double *phi = basis + static_cast<size_t>(q) * N;
  const double *ai = a + static_cast<size_t>(item) * N;
  double s = 0.0;
  for (int node = threadIdx.x; node < N; node += kThreads)
    s = fma(phi[node], ai[node] - mean[node], s);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    coeffs[static_cast<size_t>(item) * rank + q] = red[0];
}

} // namespace

Status WarmModel::Create(int N, int rank, const double *mean, const double *basis, Mlp *mlp,
                         const float *feature_shift, const float *feature_scale,
                         const double *coeff_shift, const double *coeff_scale)
{
  if (N < 1 || rank < 1 || rank > 1024 || !mean || !basis)
    return Status::kInvalidArgument;
  if (mlp && (mlp->outputs() != rank || !feature_shift || !feature_scale || !coeff_shift || !coeff_scale))
    return Status::kInvalidArgument;
  N_ = N;
  rank_ = rank;
  mlp_ = mlp;
  Status s;
  if ((s = mean_.upload(mean, N)) != Status::kOk ||
      (s = basis_.upload(basis, static_cast<size_t>(rank) * N)) != Status::kOk)
    return s;
  if (mlp) {
    const int I = mlp->inputs();
    if ((s = fshift_.upload(feature_shift, I)) != Status::kOk ||
        (s = fscale_.upload(feature_scale, I)) != Status::kOk ||
        (s = cshift_.upload(coeff_shift, rank)) != Status::kOk ||
        (s = cscale_.upload(coeff_scale, rank)) != Status::kOk)
      return s;
  }
  return cudaDeviceSynchronize() == cudaSuccess ? Status::kOk : Status::kInternalError;
}

Status WarmModel::ProjectDevice(int k, const double *a, double *coeffs, cudaStream_t st)
{
  if (k < 1 || k > 65535)
    return Status::kInvalidArgument;
  ProjectKernel<<<dim3(rank_, k), kThreads, 0, st>>>(N_, rank_, mean_.get(), basis_.get(), a, coeffs);
  return cudaGetLastError() == cudaSuccess ? Status::kOk : Status::kInternalError;
}

Status WarmModel::Project(int k, const double *a_host, double *coeffs_host)
{
  DeviceArray<double> a, c;
  Status s;
  if (k < 1 || !a_host || !coeffs_host)
    return Status::kInvalidArgument;
  if ((s = a.upload(a_host, static_cast<size_t>(k) * N_)) != Status::kOk ||
      (s = c.ensure(static_cast<size_t>(k) * rank_)) != Status::kOk ||
      (s = ProjectDevice(k, a.get(), c.get(), nullptr)) != Status::kOk)
    return s;
  return cudaMemcpy(coeffs_host, c.get(), sizeof(double) * k * rank_, cudaMemcpyDeviceToHost) == cudaSuccess
             ? Status::kOk
             : Status::kInternalError;
}

// Warm starts for k items from their features (device), into a (device [k][N]).
Status WarmModel::PredictDevice(int k, const float *features, double *a, cudaStream_t st)
{
  if (!mlp_ || k < 1)
    return Status::kInvalidArgument;
  const int I = mlp_->inputs();
  Status s;
  if ((s = xn_.ensure(static_cast<size_t>(k) * I)) != Status::kOk ||
      (s = y_.ensure(static_cast<size_t>(k) * rank_)) != Status::kOk)
    return s;
  NormalizeKernel<<<(k * I + kThreads - 1) / kThreads, kThreads, 0, st>>>(k, I, features, fshift_.get(),
                                                                          fscale_.get(), xn_.get());
  if (cudaGetLastError() != cudaSuccess)
    return Status::kInternalError;
  if ((s = mlp_->PredictDevice(k, xn_.get(), y_.get(), st)) != Status::kOk)
    return s;
  const dim3 grid((N_ + kThreads - 1) / kThreads, (k + kExpandItems - 1) / kExpandItems);
  const size_t smem = sizeof(double) * kExpandItems * rank_;
  ExpandKernel<<<grid, kThreads, smem, st>>>(N_, rank_, k, mean_.get(), basis_.get(), y_.get(),
                                             cshift_.get(), cscale_.get(), a);
  launches_ += 2;
  return cudaGetLastError() == cudaSuccess ? Status::kOk : Status::kInternalError;
}

Status WarmModel::Predict(int k, const float *features_host, double *a_host)
{
  if (k < 1 || !features_host || !a_host || !mlp_)
    return Status::kInvalidArgument;
  Status s;
  if ((s = f_.upload(features_host, static_cast<size_t>(k) * mlp_->inputs())) != Status::kOk ||
      (s = a_.ensure(static_cast<size_t>(k) * N_)) != Status::kOk ||
      (s = PredictDevice(k, f_.get(), a_.get(), nullptr)) != Status::kOk)
    return s;
  return cudaMemcpy(a_host, a_.get(), sizeof(double) * k * N_, cudaMemcpyDeviceToHost) == cudaSuccess
             ? Status::kOk
             : Status::kInternalError;
}

} // namespace fg
