// csr_pcg.cpp -- fg_csr_pcg: the batched PCG kernel on an arbitrary CSR operator.
//
// Mirrors GpuCsrSolver::Initialize (validation, gpu_solver/src/solvers/csr_solver.cu:
// 25-102) followed by Solve / SolveBatch / SolveCurrentOperatorBatch (:139-390):
// values_per_item = 0 shares one operator between all right-hand sides.
#include "femm_gpu.h"
#include "common.h"
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

using fg::DeviceArray;
using fg::Status;
using fg::ToInt;

namespace
{

int PadItems(int k)
{
  int kp = 1;
  while (kp < k)
    kp <<= 1;
  return kp;
}

Status CsrPcg(int32_t n, const int32_t *ro, const int32_t *col, const double *val, int32_t vpi,
              const double *diag, int32_t items, const double *rhs, double tol, int32_t maxit,
              double *x, fg_linear_info *info)
{
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices < 1) {
    cudaGetLastError();
    return Status::kGpuUnavailable;
  }
  if (n <= 0 || items <= 0 || items > fg::kMaxItems || !ro || !col || !val || !diag || !rhs || !x ||
      !info || ro[0] != 0)
    return Status::kInvalidArgument;
  const int64_t nnz = ro[n];
  if (vpi != 0 && vpi != nnz)
    return Status::kInvalidArgument;
  for (int32_t r = 0; r < n; ++r)
    if (ro[r] > ro[r + 1])
      return Status::kInvalidArgument;
  const bool shared = vpi == 0;
  const int op_items = shared ? 1 : items;
  for (int i = 0; i < op_items; ++i) {
    for (int64_t k = 0; k < nnz; ++k)
      if (col[k] < 0 || col[k] >= n || !std::isfinite(val[i * nnz + k]))
        return Status::kInvalidArgument;
    for (int32_t r = 0; r < n; ++r)
      if (!std::isfinite(diag[static_cast<size_t>(i) * n + r]))
        return Status::kInvalidArgument;
  }
  for (int i = 0; i < items; ++i)
    info[i] = fg_linear_info{ToInt(Status::kInvalidArgument), 0,
                             std::numeric_limits<double>::infinity()};
  if (!(tol > 0.0) || !(tol < 1.0) || !std::isfinite(tol) || maxit < 0)
    return Status::kOk;

  const int kp = PadItems(items);
  const int n_pad = (n + 31) / 32 * 32, slices = n_pad / 32;
  std::vector<int32_t> row_len(n_pad, 0), slice_off(slices + 1, 0);
  for (int32_t r = 0; r < n; ++r)
    row_len[r] = ro[r + 1] - ro[r];
  for (int s = 0; s < slices; ++s) {
    int w = 0;
    for (int r = 32 * s; r < 32 * s + 32; ++r)
      w = std::max(w, row_len[r]);
    slice_off[s + 1] = slice_off[s] + 32 * w;
  }
  const int64_t positions = slice_off[slices];
  const int vk = shared ? 1 : kp;
  std::vector<int32_t> sell_col(positions, 0);
  std::vector<double> sell_val(static_cast<size_t>(positions) * vk, 0.0);
  for (int32_t r = 0; r < n; ++r)
    for (int w = 0; w < row_len[r]; ++w) {
      const size_t pos = static_cast<size_t>(slice_off[r / 32]) + 32 * w + r % 32;
      sell_col[pos] = col[ro[r] + w];
      for (int i = 0; i < op_items; ++i)
        sell_val[pos * vk + i] = val[static_cast<size_t>(i) * nnz + ro[r] + w];
    }
  // Inverse diagonal only when every reciprocal is normal (options.cpp:176-199).
  const int dk = shared ? 1 : kp;
  std::vector<double> d(static_cast<size_t>(n_pad) * dk, 1.0), inv(static_cast<size_t>(n_pad) * dk, 0.0);
  bool usable = true;
  for (int i = 0; i < op_items; ++i)
    for (int32_t r = 0; r < n; ++r) {
      const double v = diag[static_cast<size_t>(i) * n + r];
      d[static_cast<size_t>(r) * dk + i] = v;
      const double iv = 1.0 / v;
      if (!std::isfinite(v) || !(v > 0.0) || !std::isnormal(iv))
        usable = false;
      else
        inv[static_cast<size_t>(r) * dk + i] = iv;
    }
  std::vector<double> b(static_cast<size_t>(n_pad) * kp, 0.0);
  for (int i = 0; i < items; ++i)
    for (int32_t r = 0; r < n; ++r)
      b[static_cast<size_t>(r) * kp + i] = rhs[static_cast<size_t>(i) * n + r];

  DeviceArray<int32_t> d_len, d_off, d_col, d_err;
  DeviceArray<double> d_val, d_diag, d_inv, d_b, d_x, d_r, d_z, d_p0, d_p1, d_q, d_part, d_info;
  DeviceArray<unsigned> d_bar;
  const size_t vec = static_cast<size_t>(n_pad) * kp;
  const int grid_cap = fg::PcgMaxGrid(kp);
  if (grid_cap <= 0)
    return Status::kGpuUnavailable;
  Status s = Status::kOk;
  if ((s = d_len.upload(row_len.data(), row_len.size())) != Status::kOk ||
      (s = d_off.upload(slice_off.data(), slice_off.size())) != Status::kOk ||
      (s = d_col.upload(sell_col.data(), sell_col.size())) != Status::kOk ||
      (s = d_val.upload(sell_val.data(), sell_val.size())) != Status::kOk ||
      (s = d_diag.upload(d.data(), d.size())) != Status::kOk ||
      (s = d_inv.upload(inv.data(), inv.size())) != Status::kOk ||
      (s = d_b.upload(b.data(), b.size())) != Status::kOk || (s = d_x.ensure(vec)) != Status::kOk ||
      (s = d_r.ensure(vec)) != Status::kOk || (s = d_z.ensure(vec)) != Status::kOk ||
      (s = d_p0.ensure(vec)) != Status::kOk || (s = d_p1.ensure(vec)) != Status::kOk ||
      (s = d_q.ensure(vec)) != Status::kOk ||
      (s = d_part.ensure(static_cast<size_t>(2) * 64 * grid_cap)) != Status::kOk ||
      (s = d_info.ensure(3 * static_cast<size_t>(kp))) != Status::kOk ||
      (s = d_bar.ensure(1)) != Status::kOk || (s = d_err.ensure(1)) != Status::kOk)
    return s;
  fg::PcgArgs a{};
  a.n = n;
  a.n_pad = n_pad;
  a.slices = slices;
  a.kp = kp;
  a.items = items;
  a.slice_off = d_off.get();
  a.row_len = d_len.get();
  a.sell_col = d_col.get();
  a.values = d_val.get();
  a.value_stride = vk;
  a.value_item = shared ? 0 : 1;
  a.diag = d_diag.get();
  a.invd = d_inv.get();
  a.diag_stride = dk;
  a.diag_item = shared ? 0 : 1;
  a.use_inverse = usable ? 1 : 0;
  a.b = d_b.get();
  a.x = d_x.get();
  a.r = d_r.get();
  a.z = d_z.get();
  a.p0 = d_p0.get();
  a.p1 = d_p1.get();
  a.q = d_q.get();
  a.partials = d_part.get();
  a.barrier = d_bar.get();
  a.error = d_err.get();
  a.info = d_info.get();
  a.tolerance = tol;
  a.max_iterations = maxit;
  a.active_mask = items >= 32 ? 0xffffffffu : ((1u << items) - 1u);
  a.timeout_ns = fg::PcgWaitLimitNs();
  if (fg::LaunchPcg(a, nullptr, nullptr, nullptr) != cudaSuccess) {
    cudaGetLastError();
    return Status::kInternalError;
  }
  std::vector<double> xi(vec), pinfo(3 * kp);
  int32_t err = 0;
  if (cudaMemcpy(xi.data(), d_x.get(), vec * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(pinfo.data(), d_info.get(), pinfo.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(&err, d_err.get(), sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    return Status::kInternalError;
  if (err)
    return Status::kInternalError;
  for (int i = 0; i < items; ++i) {
    info[i].status = static_cast<int32_t>(pinfo[3 * i]);
    info[i].iterations = static_cast<int32_t>(pinfo[3 * i + 1]);
    info[i].residual_l2 = pinfo[3 * i + 2];
    for (int32_t r = 0; r < n; ++r)
      x[static_cast<size_t>(i) * n + r] = xi[static_cast<size_t>(r) * kp + i];
  }
  return Status::kOk;
}

} // namespace

extern "C" int fg_csr_pcg(int32_t n, const int32_t *row_offsets, const int32_t *columns,
                          const double *values, int32_t values_per_item, const double *diagonal,
                          int32_t items, const double *rhs, double relative_tolerance,
                          int32_t max_iterations, double *x, fg_linear_info *info)
{
  return ToInt(CsrPcg(n, row_offsets, columns, values, values_per_item, diagonal, items, rhs,
                      relative_tolerance, max_iterations, x, info));
}
