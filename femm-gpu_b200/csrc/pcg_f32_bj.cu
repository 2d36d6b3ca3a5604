// pcg_f32_bj.cu -- FP32 block-Jacobi instantiations of the PCG kernel (8- and 32-row
// blocks), the inner solve of the mixed form.
#include "pcg_kernel.cuh"

namespace fg
{

const void *PcgKernelF32Block(int kp, int bs)
{
  if (bs == 8) {
    switch (kp) {
    case 1: return reinterpret_cast<const void *>(&PcgKernel<float, 1, 1, 8>);
    case 2: return reinterpret_cast<const void *>(&PcgKernel<float, 2, 2, 8>);
    case 4: return reinterpret_cast<const void *>(&PcgKernel<float, 4, 4, 8>);
    case 8: return reinterpret_cast<const void *>(&PcgKernel<float, 8, 4, 8>);
    case 16: return reinterpret_cast<const void *>(&PcgKernel<float, 16, 4, 8>);
    case 32: return reinterpret_cast<const void *>(&PcgKernel<float, 32, 4, 8>);
    default: return nullptr;
    }
  }
  if (bs == 32) {
    switch (kp) {
    case 1: return reinterpret_cast<const void *>(&PcgKernel<float, 1, 1, 32>);
    case 2: return reinterpret_cast<const void *>(&PcgKernel<float, 2, 2, 32>);
    case 4: return reinterpret_cast<const void *>(&PcgKernel<float, 4, 4, 32>);
    case 8: return reinterpret_cast<const void *>(&PcgKernel<float, 8, 4, 32>);
    case 16: return reinterpret_cast<const void *>(&PcgKernel<float, 16, 4, 32>);
    case 32: return reinterpret_cast<const void *>(&PcgKernel<float, 32, 4, 32>);
    default: return nullptr;
    }
  }
  return nullptr;
}

} // namespace fg
