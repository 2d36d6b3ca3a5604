// mixed.cu -- FP32 copies of the assembled FP64 operator for the mixed-precision form.
//
// Newton's linear system K x = b is assembled in FP64.  The mixed form's PCG stores the
// operator values, the diagonal and its inverse in FP32 (the inverse taken in FP64 before
// rounding); the FP64 originals stay resident for the reliable-update residuals.
#include "kernels.cuh"

namespace fg
{
namespace
{

constexpr int kThreads = 256;

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

} // namespace fg
