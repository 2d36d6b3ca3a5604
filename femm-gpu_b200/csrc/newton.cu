// newton.cu -- device side of the Newton update and of B / flux-linkage recovery.
//
// Step norm: the reference expands the free solution to nodes and forms
// ||cand - A|| / ||cand|| on the host (gpu_solver/src/solvers/nonlinear_solver.cu:
// 326-335); here both sums are a deterministic two-level device reduction and only
// 2 x items doubles cross to the host.  Relaxation (:344-351) is applied on the
// device with the per-item factor the host chose.  Recovery (FinalizeResult, :16-83)
// evaluates element B and the per-circuit flux linkage as fixed-order reductions.
#include "kernels.cuh"

#include <cmath>

namespace fg
{
namespace
{

constexpr int kThreads = 256;
constexpr int kNormBlocks = 256;

__device__ __forceinline__ double Candidate(const DevicePlan &p, int kp, const double *x, int node,
                                            int item)
{
  const int row = p.node_to_free[node];
  return row >= 0 ? static_cast<double>(p.node_sign[node]) * x[static_cast<size_t>(row) * kp + item]
                  : p.boundary[node];
}

template <int KP>
__global__ void __launch_bounds__(kThreads)
    NormsKernel(DevicePlan p, const double *__restrict__ x, const double *__restrict__ state,
                double *__restrict__ partials)
{
  __shared__ double red[kThreads / 32][2][KP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, item = lane % KP;
  double dd = 0.0, cc = 0.0;
  const size_t total = static_cast<size_t>(p.N) * KP;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int node = static_cast<int>(t / KP);
    const double c = Candidate(p, KP, x, node, item);
    const double d = c - state[t];
    dd += d * d;
    cc += c * c;
  }
  for (int off = 16; off >= KP; off >>= 1) {
    dd += __shfl_xor_sync(0xffffffffu, dd, off);
    cc += __shfl_xor_sync(0xffffffffu, cc, off);
  }
  if (lane < KP) {
    red[warp][0][lane] = dd;
    red[warp][1][lane] = cc;
  }
  __syncthreads();
  if (threadIdx.x < 2 * KP) {
    const int q = threadIdx.x / KP, it = threadIdx.x % KP;
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w)
      s += red[w][q][it];
    partials[(static_cast<size_t>(q) * KP + it) * gridDim.x + blockIdx.x] = s;
  }
}

__global__ void NormsFinalKernel(int kp, int blocks, const double *__restrict__ partials,
                                 double *__restrict__ norms)
{
  // One warp per (quantity, item); lanes stride the block partials in fixed order.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int qk = 2 * kp;
  for (int t = warp; t < qk; t += blockDim.x / 32) {
    double s = 0.0;
    for (int b = lane; b < blocks; b += 32)
      s += partials[static_cast<size_t>(t) * blocks + b];
    for (int off = 16; off > 0; off >>= 1)
      s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0)
      norms[t] = s;
  }
}

template <int KP>
__global__ void UpdateKernel(DevicePlan p, const double *__restrict__ x, double *__restrict__ state,
                             ItemScalars relax, uint32_t mask)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.N) * KP)
    return;
  const int node = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  if (!((mask >> item) & 1u))
    return;
  const double c = Candidate(p, KP, x, node, item);
  const double s = state[t];
  state[t] = s + relax.v[item] * (c - s);
}

// Recovery (SolveSafeguarded): state = saved + alpha (candidate - saved) for the items in
// mask (an Armijo trial point), a masked copy, and a masked reset to the zero start.
template <int KP>
__global__ void TrialKernel(DevicePlan p, const double *__restrict__ x, const double *__restrict__ saved,
                            double *__restrict__ state, ItemScalars alpha, uint32_t mask)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.N) * KP)
    return;
  const int node = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  if (!((mask >> item) & 1u))
    return;
  const double c = Candidate(p, KP, x, node, item);
  const double s = saved[t];
  state[t] = s + alpha.v[item] * (c - s);
}

__global__ void MaskedCopyKernel(size_t count, int kp, uint32_t mask, const double *__restrict__ from,
                                 double *__restrict__ to)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t < count && ((mask >> (t % kp)) & 1u))
    to[t] = from[t];
}

__global__ void ResetStateKernel(DevicePlan p, int kp, uint32_t mask, double *__restrict__ state)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.N) * kp)
    return;
  if ((mask >> (t % kp)) & 1u)
    state[t] = p.boundary[t / kp];
}

__global__ void InitStateKernel(DevicePlan p, int kp, const double *__restrict__ warm, int items,
                                uint32_t warm_mask, double *__restrict__ state)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.N) * kp)
    return;
  const int node = static_cast<int>(t / kp), item = static_cast<int>(t % kp);
  // Zero start with the expanded fixed values (nonlinear_solver.cu:193-209, :234-242);
  // a warm start replaces the free values and keeps the Dirichlet ones (:686-693).
  double v = p.boundary[node];
  if (warm && item < items && ((warm_mask >> item) & 1u) && p.node_to_free[node] >= 0)
    v = warm[static_cast<size_t>(item) * p.N + node];
  state[t] = v;
}

// Free-row form of a nodal state: the value of each row's root node (sign +1).
template <int KP>
__global__ void StateToFreeKernel(DevicePlan p, const double *__restrict__ state,
                                  double *__restrict__ x)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.n_pad) * KP)
    return;
  const int r = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  x[t] = r < p.n ? state[static_cast<size_t>(p.free_roots[r]) * KP + item] : 0.0;
}

// Defect of the Newton system assembled at a state with free-row form x: with the
// Jacobian J = K + C and rhs = b + C A (the assembly's own right-hand side),
// rhs - J x = b - K(A) A, the nonlinear residual at A.  Partials [2][KP][blocks]:
// ||rhs - J x||^2, ||rhs||^2; d (optional) receives rhs - J x.
template <int KP>
__global__ void __launch_bounds__(kThreads)
    EquationResidualKernel(DevicePlan p, const double *__restrict__ values,
                           const double *__restrict__ rhs, const double *__restrict__ x,
                           double *__restrict__ d, double *__restrict__ partials)
{
  __shared__ double red[kThreads / 32][2][KP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, item = lane % KP;
  double rr = 0.0, bb = 0.0;
  const size_t total = static_cast<size_t>(p.n_pad) * KP;
  for (size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(t / KP);
    double e = 0.0, b = 0.0;
    if (r < p.n) {
      const size_t base = static_cast<size_t>(p.slice_off[r >> 5]) + (r & 31);
      const int len = p.row_len[r];
      double acc = 0.0;
      for (int w = 0; w < len; ++w) {
        const size_t pos = base + 32 * static_cast<size_t>(w);
        acc = fma(values[pos * KP + item], x[static_cast<size_t>(p.sell_col[pos]) * KP + item], acc);
      }
      b = rhs[t];
      e = b - acc;
    }
    if (d)
      d[t] = e;
    rr += e * e;
    bb += b * b;
  }
  for (int off = 16; off >= KP; off >>= 1) {
    rr += __shfl_xor_sync(0xffffffffu, rr, off);
    bb += __shfl_xor_sync(0xffffffffu, bb, off);
  }
  if (lane < KP) {
    red[warp][0][lane] = rr;
    red[warp][1][lane] = bb;
  }
  __syncthreads();
  if (threadIdx.x < 2 * KP) {
    const int q = threadIdx.x / KP, it = threadIdx.x % KP;
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w)
      s += red[w][q][it];
    partials[(static_cast<size_t>(q) * KP + it) * gridDim.x + blockIdx.x] = s;
  }
}

template <int KP>
__global__ void AddCorrectionKernel(int n_pad, uint32_t mask, const double *__restrict__ x0,
                                    const double *__restrict__ delta, double *__restrict__ x)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(n_pad) * KP)
    return;
  const int item = static_cast<int>(t % KP);
  x[t] = ((mask >> item) & 1u) ? x0[t] + delta[t] : x0[t];
}

template <bool kAxi>
__global__ void FieldKernel(DevicePlan p, int kp, int items, const double *__restrict__ state,
                            double *__restrict__ b1, double *__restrict__ b2)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.E) * items)
    return;
  const int item = static_cast<int>(t / p.E), e = static_cast<int>(t % p.E);
  const size_t E = p.E;
  double a[3];
  for (int l = 0; l < 3; ++l)
    a[l] = state[static_cast<size_t>(p.elem_nodes[3 * e + l]) * kp + item];
  double f1 = 0.0, f2 = 0.0;
  if constexpr (!kAxi) {
    for (int l = 0; l < 3; ++l) {
      f1 += a[l] * p.elem_geo[(1 + l) * E + e];
      f2 += a[l] * p.elem_geo[(4 + l) * E + e];
    }
  } else {
    // Centroid of the r-z element (axisymmetric_p1.h:79-94).
    double r[3], z[3];
    for (int l = 0; l < 3; ++l) {
      r[l] = p.elem_geo[l * E + e];
      z[l] = p.elem_geo[(3 + l) * E + e];
    }
    const double det = (r[1] - r[0]) * (z[2] - z[0]) - (r[2] - r[0]) * (z[1] - z[0]);
    const double dndr[3] = {(z[1] - z[2]) / det, (z[2] - z[0]) / det, (z[0] - z[1]) / det};
    const double dndz[3] = {(r[2] - r[1]) / det, (r[0] - r[2]) / det, (r[1] - r[0]) / det};
    double rc = 0.0;
    for (int l = 0; l < 3; ++l)
      rc += (1.0 / 3.0) * r[l];
    for (int l = 0; l < 3; ++l) {
      f1 += a[l] * (-dndz[l]);
      f2 += a[l] * (dndr[l] + (1.0 / 3.0) / rc);
    }
  }
  if (b1)
    b1[t] = f1;
  if (b2)
    b2[t] = f2;
}

// Seven-point rule for the axisymmetric flux integral.
__constant__ double kBaryF[7][3] = {
    {1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0},
    {0.059715871789770, 0.470142064105115, 0.470142064105115},
    {0.470142064105115, 0.059715871789770, 0.470142064105115},
    {0.470142064105115, 0.470142064105115, 0.059715871789770},
    {0.797426985353087, 0.101286507323456, 0.101286507323456},
    {0.101286507323456, 0.797426985353087, 0.101286507323456},
    {0.101286507323456, 0.101286507323456, 0.797426985353087}};
__constant__ double kQwF[7] = {0.225, 0.132394152788506, 0.132394152788506, 0.132394152788506,
                               0.125939180544827, 0.125939180544827, 0.125939180544827};

// One block per (circuit, item): fixed-order block reduction over the circuit's elements.
template <bool kAxi>
__global__ void __launch_bounds__(kThreads)
    FluxKernel(DevicePlan p, int kp, const double *__restrict__ state, double *__restrict__ flux)
{
  __shared__ double red[kThreads / 32];
  const int c = blockIdx.x, item = blockIdx.y;
  const size_t E = p.E;
  double sum = 0.0;
  for (int k = p.circuit_elem_off[c] + threadIdx.x; k < p.circuit_elem_off[c + 1]; k += blockDim.x) {
    const int e = p.circuit_elems[k];
    const double jpa = p.mat_jpa[p.elem_mat[e]];
    double a[3];
    for (int l = 0; l < 3; ++l)
      a[l] = state[static_cast<size_t>(p.elem_nodes[3 * e + l]) * kp + item];
    if constexpr (!kAxi) {
      sum += p.elem_geo[e] * jpa / 3.0 * (a[0] + a[1] + a[2]);
    } else {
      double r[3], z[3];
      for (int l = 0; l < 3; ++l) {
        r[l] = p.elem_geo[l * E + e];
        z[l] = p.elem_geo[(3 + l) * E + e];
      }
      const double area = 0.5 * ((r[1] - r[0]) * (z[2] - z[0]) - (r[2] - r[0]) * (z[1] - z[0]));
      double f = 0.0;
      for (int q = 0; q < 7; ++q) {
        double rq = 0.0, av = 0.0;
        for (int l = 0; l < 3; ++l) {
          rq += kBaryF[q][l] * r[l];
          av += kBaryF[q][l] * a[l];
        }
        f += 6.283185307179586476925286766559005768 * rq * (area * kQwF[q]) * jpa * av;
      }
      sum += f;
    }
  }
  for (int off = 16; off > 0; off >>= 1)
    sum += __shfl_xor_sync(0xffffffffu, sum, off);
  if ((threadIdx.x & 31) == 0)
    red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kThreads / 32; ++w)
      s += red[w];
    if (!kAxi)
      s *= p.depth_m;
    flux[static_cast<size_t>(item) * p.C + c] = s;
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

// partials: [2][kp][kNormBlocks]; norms: [2][kp] (sum of squared step, sum of squared candidate)
cudaError_t LaunchNewtonNorms(const DevicePlan &p, int kp, const double *x, const double *state,
                              double *partials, double *norms, cudaStream_t stream)
{
  FG_DISPATCH_KP(kp, (NormsKernel<KP><<<kNormBlocks, kThreads, 0, stream>>>(p, x, state, partials)));
  NormsFinalKernel<<<1, 1024, 0, stream>>>(kp, kNormBlocks, partials, norms);
  return cudaGetLastError();
}

cudaError_t LaunchNewtonUpdate(const DevicePlan &p, int kp, const double *x, double *state,
                               ItemScalars relax, uint32_t update_mask, cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.N) * kp);
  FG_DISPATCH_KP(kp, (UpdateKernel<KP><<<blocks, kThreads, 0, stream>>>(p, x, state, relax, update_mask)));
  return cudaGetLastError();
}

cudaError_t LaunchInitState(const DevicePlan &p, int kp, const double *warm, int items,
                            uint32_t warm_mask, double *state, cudaStream_t stream)
{
  InitStateKernel<<<Blocks(static_cast<size_t>(p.N) * kp), kThreads, 0, stream>>>(p, kp, warm, items,
                                                                                 warm_mask, state);
  return cudaGetLastError();
}

cudaError_t LaunchTrial(const DevicePlan &p, int kp, const double *x, const double *saved,
                        double *state, ItemScalars alpha, uint32_t mask, cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.N) * kp);
  FG_DISPATCH_KP(kp, (TrialKernel<KP><<<blocks, kThreads, 0, stream>>>(p, x, saved, state, alpha, mask)));
  return cudaGetLastError();
}

cudaError_t LaunchMaskedCopy(const DevicePlan &p, int kp, uint32_t mask, const double *from, double *to,
                             cudaStream_t stream)
{
  const size_t count = static_cast<size_t>(p.N) * kp;
  MaskedCopyKernel<<<Blocks(count), kThreads, 0, stream>>>(count, kp, mask, from, to);
  return cudaGetLastError();
}

cudaError_t LaunchResetState(const DevicePlan &p, int kp, uint32_t mask, double *state, cudaStream_t stream)
{
  ResetStateKernel<<<Blocks(static_cast<size_t>(p.N) * kp), kThreads, 0, stream>>>(p, kp, mask, state);
  return cudaGetLastError();
}

cudaError_t LaunchStateToFree(const DevicePlan &p, int kp, const double *state, double *x,
                              cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n_pad) * kp);
  FG_DISPATCH_KP(kp, (StateToFreeKernel<KP><<<blocks, kThreads, 0, stream>>>(p, state, x)));
  return cudaGetLastError();
}

cudaError_t LaunchEquationResidual(const DevicePlan &p, int kp, const double *values,
                                   const double *rhs, const double *x, double *d,
                                   double *partials, double *norms, cudaStream_t stream)
{
  FG_DISPATCH_KP(kp, (EquationResidualKernel<KP><<<kNormBlocks, kThreads, 0, stream>>>(p, values, rhs, x, d, partials)));
  NormsFinalKernel<<<1, 1024, 0, stream>>>(kp, kNormBlocks, partials, norms);
  return cudaGetLastError();
}

cudaError_t LaunchAddCorrection(const DevicePlan &p, int kp, uint32_t mask, const double *x0,
                                const double *delta, double *x, cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n_pad) * kp);
  FG_DISPATCH_KP(kp, (AddCorrectionKernel<KP><<<blocks, kThreads, 0, stream>>>(p.n_pad, mask, x0, delta, x)));
  return cudaGetLastError();
}

// Tangent right-hand sides (SolveTangentMultiRhs, nonlinear_solver.cu:131-144): for each
// direction i, b_i = sum over circuits of dI_c / dI times the circuit's folded per-amp load;
// no magnet or boundary terms.  Rows >= n and pad items are zero.
template <int KP>
__global__ void TangentRhsKernel(DevicePlan p, int items, const double *__restrict__ directions,
                                 double *__restrict__ rhs)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.n_pad) * KP)
    return;
  const int r = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  double sum = 0.0;
  if (r < p.n && item < items)
    for (int c = 0; c < p.C; ++c) {
      const double scale = directions[item * p.C + c];
      if (scale != 0.0)
        sum += scale * p.circuit_rhs[static_cast<size_t>(c) * p.n + r];
    }
  rhs[t] = sum;
}

// The nodal derivative dA (ExpandAssemblyDerivative, nonlinear_model.cpp:412-422): the
// signed free-row value, zero on fixed nodes.
template <int KP>
__global__ void DerivativeStateKernel(DevicePlan p, const double *__restrict__ x, double *__restrict__ state)
{
  const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= static_cast<size_t>(p.N) * KP)
    return;
  const int node = static_cast<int>(t / KP), item = static_cast<int>(t % KP);
  const int row = p.node_to_free[node];
  state[t] = row >= 0 ? static_cast<double>(p.node_sign[node]) * x[static_cast<size_t>(row) * KP + item] : 0.0;
}

cudaError_t LaunchTangentRhs(const DevicePlan &p, int kp, int items, const double *directions, double *rhs,
                             cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.n_pad) * kp);
  FG_DISPATCH_KP(kp, (TangentRhsKernel<KP><<<blocks, kThreads, 0, stream>>>(p, items, directions, rhs)));
  return cudaGetLastError();
}

cudaError_t LaunchDerivativeState(const DevicePlan &p, int kp, const double *x, double *state,
                                  cudaStream_t stream)
{
  const unsigned blocks = Blocks(static_cast<size_t>(p.N) * kp);
  FG_DISPATCH_KP(kp, (DerivativeStateKernel<KP><<<blocks, kThreads, 0, stream>>>(p, x, state)));
  return cudaGetLastError();
}

cudaError_t LaunchFinalize(const DevicePlan &p, int kp, int items, const double *state,
                           double *a_out, double *b1_out, double *b2_out, double *flux_out,
                           cudaStream_t stream)
{
  if (a_out) {
    cudaError_t e = LaunchDeinterleave(kp, items, p.N, state, a_out, stream);
    if (e != cudaSuccess)
      return e;
  }
  if (b1_out || b2_out) {
    const unsigned blocks = Blocks(static_cast<size_t>(p.E) * items);
    if (p.problem_type == 0)
      FieldKernel<false><<<blocks, kThreads, 0, stream>>>(p, kp, items, state, b1_out, b2_out);
    else
      FieldKernel<true><<<blocks, kThreads, 0, stream>>>(p, kp, items, state, b1_out, b2_out);
  }
  if (flux_out && p.C > 0) {
    if (p.problem_type == 0)
      FluxKernel<false><<<dim3(p.C, items), kThreads, 0, stream>>>(p, kp, state, flux_out);
    else
      FluxKernel<true><<<dim3(p.C, items), kThreads, 0, stream>>>(p, kp, state, flux_out);
  }
  return cudaGetLastError();
}

} // namespace fg
