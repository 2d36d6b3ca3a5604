// pcg_f64_1r.cu -- instantiations of the one-reduction FP64 Jacobi PCG (pcg1r_kernel.cuh).
#include "pcg1r_kernel.cuh"

namespace fg
{

const void *PcgKernelF64OneReduction(int kp)
{
  switch (kp) {
  case 1: return reinterpret_cast<const void *>(&Pcg1rKernel<1, 1>);
  case 2: return reinterpret_cast<const void *>(&Pcg1rKernel<2, 2>);
  case 4: return reinterpret_cast<const void *>(&Pcg1rKernel<4, 2>);
  case 8: return reinterpret_cast<const void *>(&Pcg1rKernel<8, 2>);
  case 16: return reinterpret_cast<const void *>(&Pcg1rKernel<16, 2>);
  case 32: return reinterpret_cast<const void *>(&Pcg1rKernel<32, 2>);
  default: return nullptr;
  }
}

} // namespace fg
