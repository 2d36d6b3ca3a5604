// pcg_f64_wide.cu -- FP64 Jacobi PCG in CTAs of 1024 threads (two row groups each, one CTA
// per SM): the same rows, per-warp order and partial sums as the 512-thread kernel, so the
// same bits; the plan's launch-shape autotuner picks whichever is faster.
#include "pcg_kernel.cuh"

namespace fg
{

const void *PcgKernelF64Wide(int kp)
{
  constexpr int NW = 2 * kPcgWarps;
  switch (kp) {
  case 1: return reinterpret_cast<const void *>(&PcgKernel<double, 1, 1, 0, NW>);
  case 2: return reinterpret_cast<const void *>(&PcgKernel<double, 2, 2, 0, NW>);
  case 4: return reinterpret_cast<const void *>(&PcgKernel<double, 4, 2, 0, NW>);
  case 8: return reinterpret_cast<const void *>(&PcgKernel<double, 8, 2, 0, NW>);
  case 16: return reinterpret_cast<const void *>(&PcgKernel<double, 16, 2, 0, NW>);
  case 32: return reinterpret_cast<const void *>(&PcgKernel<double, 32, 2, 0, NW>);
  default: return nullptr;
  }
}

} // namespace fg
