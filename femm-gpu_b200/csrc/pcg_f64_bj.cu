// pcg_f64_bj.cu -- FP64 block-Jacobi instantiations of the PCG kernel (8- and 32-row
// blocks; 32-row blocks up to 16 items, whose staging buffer still allows 2 CTAs per SM).
#include "pcg_kernel.cuh"

namespace fg
{

const void *PcgKernelF64Block(int kp, int bs)
{
  if (bs == 8) {
    switch (kp) {
    case 1: return reinterpret_cast<const void *>(&PcgKernel<double, 1, 1, 8>);
    case 2: return reinterpret_cast<const void *>(&PcgKernel<double, 2, 2, 8>);
    case 4: return reinterpret_cast<const void *>(&PcgKernel<double, 4, 2, 8>);
    case 8: return reinterpret_cast<const void *>(&PcgKernel<double, 8, 2, 8>);
    case 16: return reinterpret_cast<const void *>(&PcgKernel<double, 16, 2, 8>);
    case 32: return reinterpret_cast<const void *>(&PcgKernel<double, 32, 2, 8>);
    default: return nullptr;
    }
  }
  if (bs == 32) {
    switch (kp) {
    case 1: return reinterpret_cast<const void *>(&PcgKernel<double, 1, 1, 32>);
    case 2: return reinterpret_cast<const void *>(&PcgKernel<double, 2, 2, 32>);
    case 4: return reinterpret_cast<const void *>(&PcgKernel<double, 4, 2, 32>);
    case 8: return reinterpret_cast<const void *>(&PcgKernel<double, 8, 2, 32>);
    case 16: return reinterpret_cast<const void *>(&PcgKernel<double, 16, 2, 32>);
    default: return nullptr;
    }
  }
  return nullptr;
}

} // namespace fg
