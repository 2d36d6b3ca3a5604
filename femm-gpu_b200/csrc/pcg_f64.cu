// pcg_f64.cu -- FP64 Jacobi instantiations of the PCG kernel (the drop-in solve).
#include "pcg_kernel.cuh"

namespace fg
{

const void *PcgKernelF64(int kp)
{
  switch (kp) {
  case 1: return reinterpret_cast<const void *>(&PcgKernel<double, 1, 1, 0>);
  case 2: return reinterpret_cast<const void *>(&PcgKernel<double, 2, 2, 0>);
  case 4: return reinterpret_cast<const void *>(&PcgKernel<double, 4, 2, 0>);
  case 8: return reinterpret_cast<const void *>(&PcgKernel<double, 8, 2, 0>);
  case 16: return reinterpret_cast<const void *>(&PcgKernel<double, 16, 2, 0>);
  case 32: return reinterpret_cast<const void *>(&PcgKernel<double, 32, 2, 0>);
  default: return nullptr;
  }
}

// The multi-plan kernel: FP64 Jacobi solves of one item per group (independent meshes), or
// of 32 items per group (the chunks of a wide shared-geometry batch).
const void *MultiPcgKernelF64(int kp)
{
  switch (kp) {
  case 1: return reinterpret_cast<const void *>(&MultiPcgKernel<double, 1, 1, 0>);
  case 32: return reinterpret_cast<const void *>(&MultiPcgKernel<double, 32, 2, 0>);
  default: return nullptr;
  }
}

} // namespace fg
