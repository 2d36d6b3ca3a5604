// pcg_f32.cu -- FP32 Jacobi instantiations of the PCG kernel (inner solve of the mixed form).
#include "pcg_kernel.cuh"

namespace fg
{

const void *PcgKernelF32(int kp)
{
  switch (kp) {
  case 1: return reinterpret_cast<const void *>(&PcgKernel<float, 1, 1, 0>);
  case 2: return reinterpret_cast<const void *>(&PcgKernel<float, 2, 2, 0>);
  case 4: return reinterpret_cast<const void *>(&PcgKernel<float, 4, 4, 0>);
  case 8: return reinterpret_cast<const void *>(&PcgKernel<float, 8, 4, 0>);
  case 16: return reinterpret_cast<const void *>(&PcgKernel<float, 16, 4, 0>);
  case 32: return reinterpret_cast<const void *>(&PcgKernel<float, 32, 4, 0>);
  default: return nullptr;
  }
}

} // namespace fg
