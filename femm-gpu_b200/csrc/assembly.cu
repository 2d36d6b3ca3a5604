// assembly.cu -- deterministic Newton assembly on the device.
//
// The reference evaluates B, nu and dnu/d(B^2) per element and then gathers every
// CSR slot from a fixed contributor list (gpu_solver/src/physics/nonlinear_assembly.cu:
// 56-206).  Here the element pass goes one step further and emits the element's
// symmetric 3x3 Newton matrix (K + C, six values) and its three load terms
// (C * A_old minus the Dirichlet lift), so the slot / row gathers only sum
// pre-computed numbers in element order: no atomics, fixed order, no recomputation.
#include "kernels.cuh"

#include <cmath>

namespace fg
{
namespace
{

constexpr int kThreads = 256;

__device__ __forceinline__ bool BhEval(const DevicePlan &p, int off, int cnt, double field_b,
                                       double *nu, double *dnu)
{
  const double b = fabs(field_b);
  const double *kb = p.curve_b + off, *kh = p.curve_h + off, *ks = p.curve_slope + off;
  if (b == 0.0) {
    *nu = ks[0];
    *dnu = 0.0;
    return isfinite(*nu);
  }
  double h, dh;
  const int last = cnt - 1;
  if (b > kb[last]) {
    h = kh[last] + ks[last] * (b - kb[last]);
    dh = ks[last];
  } else {
    // First segment i with b <= kb[i + 1]: the reference's ascending scan order.
    int lo = 1, hi = last;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (kb[mid] >= b)
        hi = mid;
      else
        lo = mid + 1;
    }
    const int i = lo - 1;
    if (!(b >= kb[i] && b <= kb[i + 1]))
      return false;
    const double len = kb[i + 1] - kb[i];
    const double z = (b - kb[i]) / len, z2 = z * z;
    h = (1.0 - 3.0 * z2 + 2.0 * z2 * z) * kh[i] + z * (1.0 - 2.0 * z + z2) * len * ks[i] +
        z2 * (3.0 - 2.0 * z) * kh[i + 1] + z2 * (z - 1.0) * len * ks[i + 1];
    dh = 6.0 * z * (z - 1.0) * kh[i] / len + (1.0 - 4.0 * z + 3.0 * z2) * ks[i] +
         6.0 * z * (1.0 - z) * kh[i + 1] / len + z * (3.0 * z - 2.0) * ks[i + 1];
  }
  *nu = h / b;
  *dnu = 0.5 * (dh / (b * b) - h / (b * b * b));
  return isfinite(*nu) && isfinite(*dnu);
}

// EvaluateNonlinearMaterial (nonlinear_model.cpp:428-451) with the device kernel's
// cold secant at iteration zero (nonlinear_assembly.cu:126-136).
__device__ __forceinline__ bool Material(const DevicePlan &p, int mat, double bmag, bool newton,
                                         double *nu, double *dnu)
{
  if (!isfinite(bmag))
    return false;
  const int off = p.mat_curve_off[mat];
  bool ok = true;
  if (off >= 0) {
    if (!newton) {
      *nu = p.mat_cold[mat];
      *dnu = 0.0;
    } else {
      ok = BhEval(p, off, p.mat_curve_cnt[mat], bmag, nu, dnu);
    }
  } else {
    const double nu0 = p.mat_nu0[mat], alpha = p.mat_alpha[mat];
    *nu = nu0 * (1.0 + alpha * bmag * bmag);
    *dnu = newton ? nu0 * alpha : 0.0;
  }
  return ok && *nu > 0.0 && isfinite(*nu) && isfinite(*dnu);
}

// Seven-point Dunavant rule (axisymmetric_p1.h:47-60).
__constant__ double kBary[7][3] = {
    {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0},
    {0.059715871789770, 0.470142064105115, 0.470142064105115},
    {0.470142064105115, 0.059715871789770, 0.470142064105115},
    {0.470142064105115, 0.470142064105115, 0.059715871789770},
    {0.797426985353087, 0.101286507323456, 0.101286507323456},
    {0.101286507323456, 0.797426985353087, 0.101286507323456},
    {0.101286507323456, 0.101286507323456, 0.797426985353087}};
__constant__ double kQw[7] = {0.225, 0.132394152788506, 0.132394152788506, 0.132394152788506,
                              0.125939180544827, 0.125939180544827, 0.125939180544827};

template <int KP, bool kAxi>
__global__ void __launch_bounds__(kThreads)
    ElementKernel(DevicePlan p, const double *__restrict__ state, uint32_t newton_mask,
                  uint32_t active_mask, double *__restrict__ ev, double *__restrict__ er,
                  int32_t *__restrict__ invalid)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int e = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  if (e >= p.E || !((active_mask >> item) & 1u))
    return;
  const bool newton = (newton_mask >> item) & 1u;
  const int nd[3] = {p.elem_nodes[3 * e], p.elem_nodes[3 * e + 1], p.elem_nodes[3 * e + 2]};
  const int mat = p.elem_mat[e];
  double a[3], bv[3];
  for (int l = 0; l < 3; ++l) {
    a[l] = state[static_cast<size_t>(nd[l]) * KP + item];
    bv[l] = p.boundary[nd[l]];
  }
  double m[6] = {0, 0, 0, 0, 0, 0}, rhs[3] = {0, 0, 0};
  bool ok = true;
  const size_t E = p.E;
  if constexpr (!kAxi) {
    const double area = p.elem_geo[e];
    double bx[3], by[3];
    for (int l = 0; l < 3; ++l) {
      bx[l] = p.elem_geo[(1 + l) * E + e];
      by[l] = p.elem_geo[(4 + l) * E + e];
    }
    double Bx = 0.0, By = 0.0;
    for (int l = 0; l < 3; ++l) {
      Bx += a[l] * bx[l];
      By += a[l] * by[l];
    }
    double nu = 0.0, dnu = 0.0;
    ok = Material(p, mat, hypot(Bx, By), newton, &nu, &dnu);
    double bd[3];
    for (int l = 0; l < 3; ++l)
      bd[l] = Bx * bx[l] + By * by[l];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const double k = area * nu * (bx[i] * bx[j] + by[i] * by[j]);
        const double c = newton ? 2.0 * area * dnu * bd[i] * bd[j] : 0.0;
        if (j >= i)
          m[i == 0 ? j : (i == 1 ? 2 + j : 5)] = k + c;
        if (newton)
          rhs[i] += c * a[j];
        if (bv[j] != 0.0)
          rhs[i] -= (k + c) * bv[j];
      }
  } else {
    double r[3], z[3];
    for (int l = 0; l < 3; ++l) {
      r[l] = p.elem_geo[l * E + e];
      z[l] = p.elem_geo[(3 + l) * E + e];
    }
    const double det = (r[1] - r[0]) * (z[2] - z[0]) - (r[2] - r[0]) * (z[1] - z[0]);
    const double dndr[3] = {(z[1] - z[2]) / det, (z[2] - z[0]) / det, (z[0] - z[1]) / det};
    const double dndz[3] = {(r[2] - r[1]) / det, (r[0] - r[2]) / det, (r[1] - r[0]) / det};
    const double area = 0.5 * det;
    for (int q = 0; q < 7; ++q) {
      double rq = 0.0;
      for (int l = 0; l < 3; ++l)
        rq += kBary[q][l] * r[l];
      double br[3], bz[3];
      for (int l = 0; l < 3; ++l) {
        br[l] = -dndz[l];
        bz[l] = dndr[l] + kBary[q][l] / rq;
      }
      double Br = 0.0, Bz = 0.0;
      for (int l = 0; l < 3; ++l) {
        Br += a[l] * br[l];
        Bz += a[l] * bz[l];
      }
      double nu = 0.0, dnu = 0.0;
      ok = ok && Material(p, mat, hypot(Br, Bz), newton, &nu, &dnu);
      const double w = 6.283185307179586476925286766559005768 * rq * (area * kQw[q]);
      double bd[3];
      for (int l = 0; l < 3; ++l)
        bd[l] = Br * br[l] + Bz * bz[l];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          const double k = w * nu * (br[i] * br[j] + bz[i] * bz[j]);
          const double c = newton ? 2.0 * w * dnu * bd[i] * bd[j] : 0.0;
          if (j >= i)
            m[i == 0 ? j : (i == 1 ? 2 + j : 5)] += k + c;
          if (newton)
            rhs[i] += c * a[j];
          if (bv[j] != 0.0)
            rhs[i] -= (k + c) * bv[j];
        }
    }
  }
  const size_t stride = E * KP, base = static_cast<size_t>(e) * KP + item;
  for (int s = 0; s < 6; ++s)
    ev[s * stride + base] = m[s];
  for (int i = 0; i < 3; ++i)
    er[i * stride + base] = rhs[i];
  if (!ok)
    atomicOr(invalid + item, 1);
}

template <int KP>
__global__ void __launch_bounds__(kThreads)
    GatherValuesKernel(DevicePlan p, const double *__restrict__ ev, uint32_t active_mask,
                       double *__restrict__ val, double *__restrict__ diag,
                       double *__restrict__ invd, int32_t *__restrict__ invalid)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int r = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  if (r >= p.n_pad)
    return;
  if (r >= p.n) {
    diag[static_cast<size_t>(r) * KP + item] = 1.0;
    invd[static_cast<size_t>(r) * KP + item] = 0.0;
    return;
  }
  if (!((active_mask >> item) & 1u))
    return;
  const size_t stride = static_cast<size_t>(p.E) * KP;
  const int s0 = p.row_offsets[r], len = p.row_len[r];
  const size_t base = static_cast<size_t>(p.slice_off[r >> 5]) + (r & 31);
  bool bad = false;
  for (int w = 0; w < len; ++w) {
    const int s = s0 + w;
    double sum = 0.0;
    for (int k = p.contrib_off[s]; k < p.contrib_off[s + 1]; ++k) {
      const int code = p.contrib[k];
      const double v = ev[((code >> 1) & 7) * stride + static_cast<size_t>(code >> 4) * KP + item];
      sum += (code & 1) ? -v : v;
    }
    // The air-gap stiffness joins after every triangle, as the reference orders it.
    if (p.age_val)
      sum += p.age_val[s];
    val[(base + 32 * static_cast<size_t>(w)) * KP + item] = sum;
    if (p.columns[s] == r) {
      diag[static_cast<size_t>(r) * KP + item] = sum;
      const bool good = isfinite(sum) && sum > 0.0;
      invd[static_cast<size_t>(r) * KP + item] = good ? 1.0 / sum : 0.0;
      bad = bad || !good;
    }
  }
  if (bad)
    atomicOr(invalid + item, 1);
}

template <int KP>
__global__ void __launch_bounds__(kThreads)
    GatherRhsKernel(DevicePlan p, const double *__restrict__ er,
                    const double *__restrict__ currents, const double *__restrict__ hc_scale,
                    uint32_t active_mask, double *__restrict__ rhs)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int r = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  if (r >= p.n_pad)
    return;
  if (r >= p.n) {
    rhs[static_cast<size_t>(r) * KP + item] = 0.0;
    return;
  }
  if (!((active_mask >> item) & 1u))
    return;
  double sum = hc_scale ? p.pm_rhs[r] * hc_scale[item] : p.pm_rhs[r];
  if (p.age_rhs)
    sum += p.age_rhs[r];
  for (int c = 0; c < p.C; ++c)
    sum += currents[item * p.C + c] * p.circuit_rhs[static_cast<size_t>(c) * p.n + r];
  const size_t stride = static_cast<size_t>(p.E) * KP;
  for (int k = p.rhs_off[r]; k < p.rhs_off[r + 1]; ++k) {
    const int code = p.rhs_contrib[k];
    const double v = er[((code >> 1) & 3) * stride + static_cast<size_t>(code >> 3) * KP + item];
    sum += (code & 1) ? -v : v;
  }
  rhs[static_cast<size_t>(r) * KP + item] = sum;
}

template <int KP>
__global__ void ExtractCsrKernel(DevicePlan p, int item, const double *__restrict__ val,
                                 const double *__restrict__ diag, const double *__restrict__ rhs,
                                 double *csr, double *diag_out, double *rhs_out)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.n)
    return;
  const size_t base = static_cast<size_t>(p.slice_off[r >> 5]) + (r & 31);
  if (csr)
    for (int w = 0; w < p.row_len[r]; ++w)
      csr[p.row_offsets[r] + w] = val[(base + 32 * static_cast<size_t>(w)) * KP + item];
  if (diag_out)
    diag_out[r] = diag[static_cast<size_t>(r) * KP + item];
  if (rhs_out)
    rhs_out[r] = rhs[static_cast<size_t>(r) * KP + item];
}

template <int KP>
__global__ void ScatterCsrKernel(DevicePlan p, int items, const double *__restrict__ csr,
                                 int values_per_item, double *__restrict__ val)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int r = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  if (r >= p.n)
    return;
  const int src_item = values_per_item ? (item < items ? item : 0) : 0;
  const size_t base = static_cast<size_t>(p.slice_off[r >> 5]) + (r & 31);
  for (int w = 0; w < p.row_len[r]; ++w)
    val[(base + 32 * static_cast<size_t>(w)) * KP + item] =
        csr[static_cast<size_t>(src_item) * values_per_item + p.row_offsets[r] + w];
}

__global__ void InterleaveKernel(int kp, int items, int len, int len_pad, const double *in,
                                 double *out)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(len_pad) * kp)
    return;
  const int i = static_cast<int>(t / kp), item = static_cast<int>(t % kp);
  out[t] = (i < len && item < items) ? in[static_cast<size_t>(item) * len + i] : 0.0;
}

__global__ void DeinterleaveKernel(int kp, int items, int len, const double *in, double *out)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(len) * items)
    return;
  const int item = static_cast<int>(t / len), i = static_cast<int>(t % len);
  out[t] = in[static_cast<size_t>(i) * kp + item];
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

cudaError_t LaunchElementKernel(const DevicePlan &p, int kp, const double *state,
                                uint32_t newton_mask, uint32_t active_mask, double *ev, double *er,
                                int32_t *invalid, cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.E) * kp);
  if (p.problem_type == 0) {
    FG_DISPATCH_KP(kp, (ElementKernel<KP, false><<<blocks, kThreads, 0, stream>>>(
                           p, state, newton_mask, active_mask, ev, er, invalid)));
  } else {
    FG_DISPATCH_KP(kp, (ElementKernel<KP, true><<<blocks, kThreads, 0, stream>>>(
                           p, state, newton_mask, active_mask, ev, er, invalid)));
  }
  return cudaGetLastError();
}

cudaError_t LaunchGatherValues(const DevicePlan &p, int kp, const double *ev, uint32_t active_mask,
                               double *values, double *diag, double *invd, int32_t *invalid,
                               cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n_pad) * kp);
  FG_DISPATCH_KP(kp, (GatherValuesKernel<KP><<<blocks, kThreads, 0, stream>>>(
                         p, ev, active_mask, values, diag, invd, invalid)));
  return cudaGetLastError();
}

cudaError_t LaunchGatherRhs(const DevicePlan &p, int kp, const double *er, const double *currents,
                            const double *hc_scale, uint32_t active_mask, double *rhs,
                            cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n_pad) * kp);
  FG_DISPATCH_KP(kp, (GatherRhsKernel<KP><<<blocks, kThreads, 0, stream>>>(
                         p, er, currents, hc_scale, active_mask, rhs)));
  return cudaGetLastError();
}

cudaError_t LaunchExtractCsr(const DevicePlan &p, int kp, int item, const double *values,
                             const double *diag, const double *rhs, double *csr, double *diag_out,
                             double *rhs_out, cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n));
  FG_DISPATCH_KP(kp, (ExtractCsrKernel<KP><<<blocks, kThreads, 0, stream>>>(
                         p, item, values, diag, rhs, csr, diag_out, rhs_out)));
  return cudaGetLastError();
}

cudaError_t LaunchScatterCsr(const DevicePlan &p, int kp, int items, const double *csr,
                             int32_t values_per_item, double *values, cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n) * kp);
  FG_DISPATCH_KP(kp, (ScatterCsrKernel<KP><<<blocks, kThreads, 0, stream>>>(
                         p, items, csr, values_per_item, values)));
  return cudaGetLastError();
}

cudaError_t LaunchInterleave(int kp, int items, int len, int len_pad, const double *in,
                             double *out, cudaStream_t stream)
{
  InterleaveKernel<<<Blocks(static_cast<size_t>(len_pad) * kp), kThreads, 0, stream>>>(
      kp, items, len, len_pad, in, out);
  return cudaGetLastError();
}

cudaError_t LaunchDeinterleave(int kp, int items, int len, const double *in, double *out,
                               cudaStream_t stream)
{
  DeinterleaveKernel<<<Blocks(static_cast<size_t>(len) * items), kThreads, 0, stream>>>(
      kp, items, len, in, out);
  return cudaGetLastError();
}

} // namespace fg
