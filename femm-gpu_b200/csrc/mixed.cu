// mixed.cu -- FP64 defect correction around the FP32 inner PCG (the mixed-precision form).
//
// Newton's linear system K x = b is assembled in FP64.  The mixed form keeps x, the
// defect r = b - K x and every norm in FP64 and only solves for corrections in FP32:
//   x = 0, r = b;  repeat { K32 d = r32 (FP32 PCG to a loose relative tolerance);
//                           x += d;  r = b - K x (FP64 SpMV) }  until ||r|| <= tol ||b||.
// The acceptance test is therefore the reference's true-residual rule
// (gpu_solver/src/solvers/pcg_kernels.cu:192-245) evaluated in FP64.
#include "kernels.cuh"

namespace fg
{
namespace
{

constexpr int kThreads = 256;
constexpr int kDefectBlocks = 256;

template <int KP>
__global__ void __launch_bounds__(kThreads)
    ToSingleKernel(DevicePlan p, uint32_t mask, const double *__restrict__ val64,
                   const double *__restrict__ diag64, float *__restrict__ val32,
                   float *__restrict__ diag32, float *__restrict__ invd32)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int r = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  if (r >= p.n_pad || !((mask >> item) & 1u))
    return;
  const size_t ri = static_cast<size_t>(r) * KP + item;
  const double d = diag64[ri];
  const float d32 = static_cast<float>(d);
  diag32[ri] = d32;
  // Padding rows read as an identity with a zero inverse, like the FP64 operator.
  invd32[ri] = (r < p.n && isfinite(d) && d > 0.0) ? static_cast<float>(1.0 / d) : 0.0f;
  if (r >= p.n)
    return;
  const size_t base = static_cast<size_t>(p.slice_off[r >> 5]) + (r & 31);
  const int len = p.row_len[r];
  for (int w = 0; w < len; ++w) {
    const size_t pos = (base + 32 * static_cast<size_t>(w)) * KP + item;
    val32[pos] = static_cast<float>(val64[pos]);
  }
}

// x = 0 (first step) or x += d; the FP32 right-hand side of the next step is written by
// the residual kernel.
template <int KP>
__global__ void AccumulateKernel(int n_pad, uint32_t mask, int first, const float *__restrict__ d,
                                 double *__restrict__ x)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(n_pad) * KP || !((mask >> (t % KP)) & 1u))
    return;
  x[t] = first ? static_cast<double>(d[t]) : x[t] + static_cast<double>(d[t]);
}

// r = b - K x in FP64 (CSR order), the FP32 copy of r for the next inner solve, and
// per-block partial sums of |r|^2 and |b|^2 per item.
template <int KP>
__global__ void __launch_bounds__(kThreads)
    DefectKernel(DevicePlan p, uint32_t mask, int zero_x, const double *__restrict__ val64,
                 const double *__restrict__ b, const double *__restrict__ x,
                 double *__restrict__ r, float *__restrict__ r32, double *__restrict__ partials)
{
  __shared__ double red[kThreads / 32][2][KP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, item = lane % KP;
  double rr = 0.0, bb = 0.0;
  const size_t total = static_cast<size_t>(p.n_pad) * KP;
  const bool on = (mask >> item) & 1u;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    if (!on)
      continue;
    const int row = static_cast<int>(t / KP);
    double acc = 0.0;
    if (!zero_x && row < p.n) {
      const size_t base = static_cast<size_t>(p.slice_off[row >> 5]) + (row & 31);
      const int len = p.row_len[row];
      for (int w = 0; w < len; ++w) {
        const size_t pos = base + 32 * static_cast<size_t>(w);
        acc = __fma_rn(val64[pos * KP + item], x[static_cast<size_t>(p.sell_col[pos]) * KP + item], acc);
      }
    }
    const double bv = row < p.n ? b[t] : 0.0;
    const double rv = bv - acc;
    r[t] = rv;
    r32[t] = static_cast<float>(rv);
    rr += rv * rv;
    bb += bv * bv;
  }
  for (int off = 16; off >= KP; off >>= 1) {
    rr += __shfl_xor_sync(0xffffffffu, rr, off);
    bb += __shfl_xor_sync(0xffffffffu, bb, off);
  }
  if (lane < KP) {
    red[warp][0][lane] = rr;
    red[warp][1][lane] = bb;
  }
  __syncthreads();
  if (threadIdx.x < 2 * KP) {
    const int q = threadIdx.x / KP, it = threadIdx.x % KP;
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w)
      s += red[w][q][it];
    partials[(static_cast<size_t>(q) * KP + it) * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void SumPartialsKernel(int kp, int blocks, const double *__restrict__ partials,
                                  double *__restrict__ out)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = warp; t < 2 * kp; t += blockDim.x / 32) {
    double s = 0.0;
    for (int b = lane; b < blocks; b += 32)
      s += partials[static_cast<size_t>(t) * blocks + b];
    for (int off = 16; off > 0; off >>= 1)
      s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0)
      out[t] = s;
  }
}

inline unsigned Blocks(size_t threads) { return static_cast<unsigned>((threads + kThreads - 1) / kThreads); }

} // namespace

#define FG_DISPATCH_KP(kp, CALL)                                                                   \
  switch (kp) {                                                                                    \
  case 1: { constexpr int KP = 1; CALL; } break;                                                    \
  case 2: { constexpr int KP = 2; CALL; } break;                                                    \
  case 4: { constexpr int KP = 4; CALL; } break;                                                    \
  case 8: { constexpr int KP = 8; CALL; } break;                                                    \
  case 16: { constexpr int KP = 16; CALL; } break;                                                  \
  case 32: { constexpr int KP = 32; CALL; } break;                                                  \
  default: return cudaErrorInvalidValue;                                                           \
  }

cudaError_t LaunchToSingle(const DevicePlan &p, int kp, uint32_t mask, const double *val64,
                           const double *diag64, float *val32, float *diag32, float *invd32,
                           cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n_pad) * kp);
  FG_DISPATCH_KP(kp, (ToSingleKernel<KP><<<blocks, kThreads, 0, stream>>>(p, mask, val64, diag64,
                                                                          val32, diag32, invd32)));
  return cudaGetLastError();
}

cudaError_t LaunchAccumulate(const DevicePlan &p, int kp, uint32_t mask, int first, const float *d,
                             double *x, cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n_pad) * kp);
  FG_DISPATCH_KP(kp, (AccumulateKernel<KP><<<blocks, kThreads, 0, stream>>>(p.n_pad, mask, first, d, x)));
  return cudaGetLastError();
}

// partials: [2][kp][256]; norms: [2][kp] = (|r|^2, |b|^2)
cudaError_t LaunchDefect(const DevicePlan &p, int kp, uint32_t mask, int zero_x, const double *val64,
                         const double *b, const double *x, double *r, float *r32,
                         double *partials, double *norms, cudaStream_t stream)
{
  FG_DISPATCH_KP(kp, (DefectKernel<KP><<<kDefectBlocks, kThreads, 0, stream>>>(
                         p, mask, zero_x, val64, b, x, r, r32, partials)));
  SumPartialsKernel<<<1, 1024, 0, stream>>>(kp, kDefectBlocks, partials, norms);
  return cudaGetLastError();
}

} // namespace fg
