// csr_solver.cuh -- CPU stand-in for the reference's GpuCsrSolver, so that the reference's
// weighted-stress mask preparation (gpu_solver/src/postprocess/weighted_stress.cu) compiles
// as host C++ into oracle/_ref.  TEST INFRASTRUCTURE ONLY.
//
// Only the two calls weighted_stress.cu makes exist: Initialize keeps the reduced CSR
// system, Solve runs the oracle's restatement of the reference's deterministic Jacobi PCG
// (femm_oracle.c, or_pcg_block with the diagonal) on it.  The thresholded mask does not depend on the last bits of
// the linear solution, which is why a CPU PCG can stand in for the device one here.
#pragma once

#include "physics/linear_model.h"

#include "femm_oracle.h"

#include <vector>

namespace gpu_femm
{

class GpuCsrSolver
{
public:
  Status Initialize(const Assembly &assembly)
  {
    assembly_ = &assembly;
    return assembly.row_offsets.empty() ? Status::kInvalidArgument : Status::kOk;
  }

  SolveInfo Solve(const std::vector<double> &rhs, double relative_tolerance, int max_iterations,
                  std::vector<double> *solution)
  {
    SolveInfo info;
    const Assembly &a = *assembly_;
    const int32_t n = static_cast<int32_t>(a.diagonal.size());
    solution->assign(n, 0.0);
    int32_t iterations = 0;
    double residual = 0.0;
    // The reference's default preconditioner (Jacobi).
    const int status = or_pcg_block(n, a.row_offsets.data(), a.column_indices.data(),
                                    a.values.data(), a.diagonal.data(), rhs.data(),
                                    relative_tolerance, max_iterations, nullptr, 0,
                                    solution->data(), &iterations, &residual);
    info.status = static_cast<Status>(status);
    info.iterations = iterations;
    info.residual_l2 = residual;
    return info;
  }

private:
  const Assembly *assembly_ = nullptr;
};

} // namespace gpu_femm
