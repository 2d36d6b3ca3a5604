// pcg.cu -- batched deterministic Jacobi PCG as one persistent cooperative kernel.
//
// Algorithm: the reference's DeterministicPcgKernel (gpu_solver/src/solvers/
// pcg_kernels.cu:10-344): x = 0, RHS max-scaling, Jacobi-preconditioned CG, and on
// reaching the threshold a true-residual check ||b/s - A x|| <= tol ||b/s|| that
// either accepts or restarts from the true residual; the same status codes.
//
// B200 mapping: one launch runs the whole solve for up to 32 items that share the
// SELL-32 pattern.  Every CTA owns a contiguous range of rows for all items, so
// column indices are read once per row for the whole batch.  A CG iteration has
// exactly two grid-wide synchronisations, each fused with its reduction: every CTA
// publishes its per-item partial sums, arrives on a release counter, and after the
// acquire reads all CTAs' partials and sums them in CTA order -- so every CTA holds
// bitwise-identical scalars and takes identical branches without a broadcast step.
// The search-direction update p = z + beta p is folded into the next SpMV
// (A p = sum a_ij (z_j + beta p_j), p double-buffered), which removes the third
// barrier a textbook CG needs.  Waits are bounded by a %globaltimer budget: on
// expiry the kernel records an error and every CTA returns.
#include "kernels.cuh"

#include <cmath>

namespace fg
{
namespace
{

constexpr int kPcgThreads = 512;
constexpr int kPcgWarps = kPcgThreads / 32;
constexpr int kMaxQ = 64; // reduced quantities x items per reduction

enum : int { kOk = 0, kNotConverged = 9, kBreakdown = 10, kNonfinite = 11, kInternal = 13 };

struct Control {
  double rho[kMaxItems], alpha[kMaxItems], beta[kMaxItems], thr[kMaxItems], scale[kMaxItems];
  double resid[kMaxItems], rz[kMaxItems];
  int active[kMaxItems], restart[kMaxItems], status[kMaxItems], iters[kMaxItems];
  int flag[kMaxItems]; // 1 threshold reached, 2 verified, 3 restart
};

struct Reduce {
  double warp[kPcgWarps][kMaxQ];
  double result[kMaxQ];
  int err;
};

__device__ __forceinline__ unsigned LoadAcquire(const unsigned *p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void AddRelease(unsigned *p, unsigned v)
{
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long GlobalTimer()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier over a monotonically increasing arrival counter, bounded in time.
__device__ bool GridBarrier(const PcgArgs &a, unsigned &epoch, Reduce &sm)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    epoch += 1;
    const unsigned target = epoch * gridDim.x;
    __threadfence();
    AddRelease(a.barrier, 1u);
    const unsigned long long t0 = GlobalTimer();
    int err = 0;
    for (;;) {
      const unsigned v = LoadAcquire(a.barrier);
      if (static_cast<int>(v - target) >= 0)
        break;
      if (*reinterpret_cast<volatile int32_t *>(a.error) != 0) {
        err = 1;
        break;
      }
      if (GlobalTimer() - t0 > static_cast<unsigned long long>(a.timeout_ns)) {
        atomicExch(a.error, 2);
        err = 1;
        break;
      }
    }
    __threadfence();
    sm.err = err;
  }
  __syncthreads();
  return sm.err == 0;
}

// Sum (or max) of Q per-item quantities over the whole grid, deterministic for a
// fixed launch shape.  v[q] is this thread's partial for its lane's item.
template <int KP, int Q, bool kMax>
__device__ bool GridReduce(const PcgArgs &a, double (&v)[Q], Reduce &sm, unsigned &epoch, int &buf)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    double x = v[q];
#pragma unroll
    for (int off = 16; off >= KP; off >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, x, off);
      x = kMax ? fmax(x, y) : x + y;
    }
    if (lane < KP)
      sm.warp[warp][q * KP + lane] = x;
  }
  __syncthreads();
  constexpr int QK = Q * KP;
  const int G = gridDim.x;
  double *part = a.partials + static_cast<size_t>(buf) * kMaxQ * G;
  if (threadIdx.x < QK) {
    double s = sm.warp[0][threadIdx.x];
    for (int w = 1; w < kPcgWarps; ++w)
      s = kMax ? fmax(s, sm.warp[w][threadIdx.x]) : s + sm.warp[w][threadIdx.x];
    part[static_cast<size_t>(threadIdx.x) * G + blockIdx.x] = s;
  }
  if (!GridBarrier(a, epoch, sm))
    return false;
  for (int t = warp; t < QK; t += kPcgWarps) {
    double s = 0.0;
    for (int g = lane; g < G; g += 32) {
      const double y = __ldcg(part + static_cast<size_t>(t) * G + g);
      s = kMax ? fmax(s, y) : s + y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, s, off);
      s = kMax ? fmax(s, y) : s + y;
    }
    if (lane == 0)
      sm.result[t] = s;
  }
  __syncthreads();
  buf ^= 1;
  return true;
}

// One row's SpMV for one item: sum_w a_rw * v_c(w), v = z (+ beta p), in CSR order.
// Column indices and values of up to eight entries are loaded before any gather so a
// thread keeps ~16 independent loads in flight instead of one dependent chain per entry.
template <int KP, bool kFold>
__device__ __forceinline__ double RowProduct(const double *__restrict__ vals,
                                             const int32_t *__restrict__ cols, size_t base,
                                             int len, int vstride, int vitem, int item,
                                             const double *z, const double *p, bool restart,
                                             double beta)
{
  double acc = 0.0;
  for (int w0 = 0; w0 < len; w0 += 8) {
    int c[8];
    double v[8], g[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      c[u] = 0;
      v[u] = 0.0;
      if (w0 + u < len) {
        const size_t pos = base + 32 * static_cast<size_t>(w0 + u);
        c[u] = __ldg(cols + pos);
        v[u] = __ldg(vals + pos * vstride + vitem);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      g[u] = 0.0;
      if (w0 + u < len) {
        const size_t ci = static_cast<size_t>(c[u]) * KP + item;
        const double zc = z[ci];
        g[u] = (!kFold || restart) ? zc : __fma_rn(beta, p[ci], zc);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (w0 + u < len)
        acc = __fma_rn(v[u], g[u], acc);
  }
  return acc;
}

template <int KP>
__global__ void __launch_bounds__(kPcgThreads, 2) PcgKernel(PcgArgs a)
{
  __shared__ Reduce sm;
  __shared__ Control ctl;
  constexpr int S = 32 / KP; // rows per warp
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int item = lane % KP;
  const int WS = a.n_pad / S;
  const int ws0 = static_cast<int>(static_cast<long long>(WS) * blockIdx.x / gridDim.x);
  const int ws1 = static_cast<int>(static_cast<long long>(WS) * (blockIdx.x + 1) / gridDim.x);
  unsigned epoch = 0;
  int buf = 0;
  const int vstride = a.value_stride, vitem = a.value_item * item;
  const int dstride = a.diag_stride, ditem = a.diag_item * item;
  const double *__restrict__ vals = a.values;
  const int32_t *__restrict__ cols = a.sell_col;
  const int32_t *__restrict__ soff = a.slice_off;
  const int32_t *__restrict__ rlen = a.row_len;

  if (threadIdx.x < KP) {
    const int it = threadIdx.x;
    ctl.active[it] = (it < a.items && ((a.active_mask >> it) & 1u)) ? 1 : 0;
    ctl.status[it] = kInternal;
    ctl.iters[it] = 0;
    ctl.resid[it] = INFINITY;
    ctl.restart[it] = 1;
    ctl.flag[it] = 0;
    ctl.beta[it] = 0.0;
  }
  __syncthreads();

  auto precond = [&](double rv, int r) -> double {
    const size_t di = static_cast<size_t>(r) * dstride + ditem;
    return a.use_inverse ? rv * __ldg(a.invd + di) : rv / __ldg(a.diag + di);
  };

#define FG_ROWS_BEGIN                                                                              \
  for (int ws = ws0 + warp; ws < ws1; ws += kPcgWarps) {                                           \
    const int r = ws * S + lane / KP;                                                              \
    const size_t ri = static_cast<size_t>(r) * KP + item;
#define FG_ROWS_END }

  // Validity (first invalid row decides the status) and RHS max-scaling.
  {
    double v[2] = {0.0, 0.0};
    const bool on = ctl.active[item];
    FG_ROWS_BEGIN
    if (on && r < a.n) {
      const double bb = a.b[ri], dd = a.diag[static_cast<size_t>(r) * dstride + ditem];
      const bool nonfinite = !isfinite(bb) || !isfinite(dd);
      if (nonfinite || !(dd > 0.0))
        v[0] = fmax(v[0], 2.0 * static_cast<double>(a.n - r) + (nonfinite ? 1.0 : 0.0));
      v[1] = fmax(v[1], fabs(bb));
    }
    a.x[ri] = 0.0;
    FG_ROWS_END
    if (!GridReduce<KP, 2, true>(a, v, sm, epoch, buf))
      return;
    if (threadIdx.x < KP) {
      const int it = threadIdx.x;
      if (ctl.active[it]) {
        const double pr = sm.result[it];
        if (pr != 0.0) {
          const bool nonfinite = pr - 2.0 * floor(0.5 * pr) != 0.0;
          ctl.status[it] = nonfinite ? kNonfinite : kBreakdown;
          ctl.active[it] = 0;
        } else {
          ctl.scale[it] = sm.result[KP + it];
          if (ctl.scale[it] == 0.0) {
            ctl.resid[it] = 0.0;
            ctl.status[it] = kOk;
            ctl.active[it] = 0;
          }
        }
      }
    }
    __syncthreads();
  }

  // r = b / s, z = M^-1 r, rho = r.z
  {
    double v[2] = {0.0, 0.0};
    if (ctl.active[item]) {
      const double s = ctl.scale[item];
      FG_ROWS_BEGIN
      const double rv = a.b[ri] / s;
      const double zv = precond(rv, r);
      a.r[ri] = rv;
      a.z[ri] = zv;
      v[0] += rv * rv;
      v[1] += rv * zv;
      FG_ROWS_END
    }
    if (!GridReduce<KP, 2, false>(a, v, sm, epoch, buf))
      return;
    if (threadIdx.x < KP) {
      const int it = threadIdx.x;
      if (ctl.active[it]) {
        const double rr = sm.result[it], rho = sm.result[KP + it];
        if (!isfinite(rr) || !isfinite(rho)) {
          ctl.status[it] = kNonfinite;
          ctl.active[it] = 0;
        } else {
          ctl.resid[it] = sqrt(rr);
          ctl.thr[it] = a.tolerance * sqrt(rr);
          ctl.rho[it] = rho;
          ctl.restart[it] = 1;
        }
      }
    }
    __syncthreads();
  }

  double *pc = a.p0, *pn = a.p1;
  for (int iteration = 0; iteration < a.max_iterations; ++iteration) {
    bool any = false;
#pragma unroll
    for (int it = 0; it < KP; ++it)
      any = any || ctl.active[it];
    if (!any)
      break;

    // Phase A: p_new = z + beta p (folded into the gather), q = A p_new, p_new . q
    {
      double v[1] = {0.0};
      if (ctl.active[item]) {
        const bool rs = ctl.restart[item];
        const double be = ctl.beta[item];
        FG_ROWS_BEGIN
        const int len = __ldg(rlen + r);
        const size_t base = static_cast<size_t>(__ldg(soff + (r >> 5))) + (r & 31);
        const double acc = RowProduct<KP, true>(vals, cols, base, len, vstride, vitem, item, a.z,
                                                pc, rs, be);
        const double zr = a.z[ri];
        const double pnew = rs ? zr : __fma_rn(be, pc[ri], zr);
        pn[ri] = pnew;
        a.q[ri] = acc;
        v[0] += pnew * acc;
        FG_ROWS_END
      }
      if (!GridReduce<KP, 1, false>(a, v, sm, epoch, buf))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        if (ctl.active[it]) {
          const double pq = sm.result[it], rho = ctl.rho[it];
          if (!isfinite(pq) || !isfinite(rho)) {
            ctl.status[it] = kNonfinite;
            ctl.active[it] = 0;
          } else if (!(pq > 0.0) || !(rho > 0.0)) {
            ctl.status[it] = kBreakdown;
            ctl.active[it] = 0;
          } else {
            ctl.alpha[it] = rho / pq;
          }
        }
      }
      __syncthreads();
      double *t = pc;
      pc = pn;
      pn = t;
    }

    // Phase B: x += alpha p, r -= alpha q, z = M^-1 r, r.r and r.z
    {
      double v[2] = {0.0, 0.0};
      if (ctl.active[item]) {
        const double al = ctl.alpha[item];
        double *__restrict__ X = a.x;
        double *__restrict__ R = a.r;
        double *__restrict__ Z = a.z;
        const double *__restrict__ P = pc;
        const double *__restrict__ Q = a.q;
        // Two row groups per pass: all eight loads are issued before the first store.
        for (int ws = ws0 + warp; ws < ws1; ws += 2 * kPcgWarps) {
          const bool two = ws + kPcgWarps < ws1;
          const int r0 = ws * S + lane / KP, r1 = (ws + kPcgWarps) * S + lane / KP;
          const size_t i0 = static_cast<size_t>(r0) * KP + item, i1 = static_cast<size_t>(r1) * KP + item;
          const double x0 = X[i0], p0 = P[i0], rv0 = R[i0], q0 = Q[i0];
          double x1 = 0.0, p1 = 0.0, rv1 = 0.0, q1 = 0.0;
          if (two) {
            x1 = X[i1];
            p1 = P[i1];
            rv1 = R[i1];
            q1 = Q[i1];
          }
          const double rn0 = rv0 - al * q0;
          const double zn0 = precond(rn0, r0);
          X[i0] = x0 + al * p0;
          R[i0] = rn0;
          Z[i0] = zn0;
          v[0] += rn0 * rn0;
          v[1] += rn0 * zn0;
          if (two) {
            const double rn1 = rv1 - al * q1;
            const double zn1 = precond(rn1, r1);
            X[i1] = x1 + al * p1;
            R[i1] = rn1;
            Z[i1] = zn1;
            v[0] += rn1 * rn1;
            v[1] += rn1 * zn1;
          }
        }
      }
      if (!GridReduce<KP, 2, false>(a, v, sm, epoch, buf))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        ctl.flag[it] = 0;
        if (ctl.active[it]) {
          ctl.iters[it] = iteration + 1;
          const double rr = sm.result[it];
          ctl.rz[it] = sm.result[KP + it];
          if (!isfinite(rr)) {
            ctl.status[it] = kNonfinite;
            ctl.active[it] = 0;
          } else {
            ctl.resid[it] = sqrt(rr);
            if (!isfinite(ctl.resid[it])) {
              ctl.status[it] = kNonfinite;
              ctl.active[it] = 0;
            } else {
              ctl.flag[it] = ctl.resid[it] <= ctl.thr[it] ? 1 : 0;
            }
          }
        }
      }
      __syncthreads();
    }

    bool verify = false;
#pragma unroll
    for (int it = 0; it < KP; ++it)
      verify = verify || (ctl.active[it] && ctl.flag[it]);
    if (verify) {
      // True residual for items at the threshold.
      {
        double v[1] = {0.0};
        if (ctl.active[item] && ctl.flag[item]) {
          const double s = ctl.scale[item];
          FG_ROWS_BEGIN
          const int len = __ldg(rlen + r);
          const size_t base = static_cast<size_t>(__ldg(soff + (r >> 5))) + (r & 31);
          const double acc = RowProduct<KP, false>(vals, cols, base, len, vstride, vitem, item,
                                                   a.x, nullptr, true, 0.0);
          const double rt = a.b[ri] / s - acc;
          a.r[ri] = rt;
          v[0] += rt * rt;
          FG_ROWS_END
        }
        if (!GridReduce<KP, 1, false>(a, v, sm, epoch, buf))
          return;
        if (threadIdx.x < KP) {
          const int it = threadIdx.x;
          if (ctl.active[it] && ctl.flag[it]) {
            const double tr = sm.result[it];
            if (!isfinite(tr)) {
              ctl.status[it] = kNonfinite;
              ctl.active[it] = 0;
            } else {
              ctl.resid[it] = sqrt(tr);
              ctl.flag[it] = ctl.resid[it] <= ctl.thr[it] ? 2 : 3;
            }
          }
        }
        __syncthreads();
      }
      // Accept (scale x back) or restart from the true residual.
      {
        double v[2] = {0.0, 0.0};
        const int f = ctl.active[item] ? ctl.flag[item] : 0;
        if (f >= 2) {
          const double s = ctl.scale[item];
          FG_ROWS_BEGIN
          if (f == 2) {
            const double xs = a.x[ri] * s;
            a.x[ri] = xs;
            if (!isfinite(xs))
              v[1] += 1.0;
          } else {
            const double rv = a.r[ri];
            const double zv = precond(rv, r);
            a.z[ri] = zv;
            v[0] += rv * zv;
          }
          FG_ROWS_END
        }
        if (!GridReduce<KP, 2, false>(a, v, sm, epoch, buf))
          return;
        if (threadIdx.x < KP) {
          const int it = threadIdx.x;
          if (ctl.active[it] && ctl.flag[it] == 2) {
            if (sm.result[KP + it] != 0.0) {
              ctl.status[it] = kNonfinite;
            } else {
              ctl.resid[it] *= ctl.scale[it];
              ctl.status[it] = isfinite(ctl.resid[it]) ? kOk : kNonfinite;
            }
            ctl.active[it] = 0;
          } else if (ctl.active[it] && ctl.flag[it] == 3) {
            const double rho = sm.result[it];
            if (!isfinite(rho) || !(rho > 0.0)) {
              ctl.status[it] = kBreakdown;
              ctl.active[it] = 0;
            } else {
              ctl.rho[it] = rho;
              ctl.restart[it] = 1;
            }
          }
        }
        __syncthreads();
      }
    }
    if (threadIdx.x < KP) {
      const int it = threadIdx.x;
      if (ctl.active[it] && ctl.flag[it] == 0) {
        const double rz = ctl.rz[it];
        if (!isfinite(rz) || !(rz > 0.0)) {
          ctl.status[it] = kBreakdown;
          ctl.active[it] = 0;
        } else {
          ctl.beta[it] = rz / ctl.rho[it];
          ctl.rho[it] = rz;
          ctl.restart[it] = 0;
        }
      }
      ctl.flag[it] = 0;
    }
    __syncthreads();
  }

  // Iteration budget exhausted: report the true residual of the unscaled iterate.
  bool any = false;
#pragma unroll
  for (int it = 0; it < KP; ++it)
    any = any || ctl.active[it];
  if (any) {
    {
      double v[1] = {0.0};
      if (ctl.active[item]) {
        const double s = ctl.scale[item];
        FG_ROWS_BEGIN
        const int len = __ldg(rlen + r);
        const size_t base = static_cast<size_t>(__ldg(soff + (r >> 5))) + (r & 31);
        const double acc = RowProduct<KP, false>(vals, cols, base, len, vstride, vitem, item, a.x,
                                                 nullptr, true, 0.0);
        const double rt = a.b[ri] / s - acc;
        a.r[ri] = rt;
        v[0] += rt * rt;
        FG_ROWS_END
      }
      if (!GridReduce<KP, 1, false>(a, v, sm, epoch, buf))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        if (ctl.active[it]) {
          const double tr = sm.result[it];
          if (!isfinite(tr)) {
            ctl.status[it] = kNonfinite;
            ctl.active[it] = 0;
          } else {
            ctl.rz[it] = tr;
          }
        }
      }
      __syncthreads();
    }
    {
      double v[1] = {0.0};
      if (ctl.active[item]) {
        const double s = ctl.scale[item];
        FG_ROWS_BEGIN
        const double xs = a.x[ri] * s;
        a.x[ri] = xs;
        if (!isfinite(xs))
          v[0] += 1.0;
        FG_ROWS_END
      }
      if (!GridReduce<KP, 1, false>(a, v, sm, epoch, buf))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        if (ctl.active[it]) {
          if (sm.result[it] != 0.0) {
            ctl.status[it] = kNonfinite;
          } else {
            ctl.resid[it] = sqrt(ctl.rz[it]) * ctl.scale[it];
            ctl.status[it] = isfinite(ctl.resid[it]) ? kNotConverged : kNonfinite;
          }
          ctl.active[it] = 0;
        }
      }
      __syncthreads();
    }
  }
#undef FG_ROWS_BEGIN
#undef FG_ROWS_END

  if (blockIdx.x == 0 && threadIdx.x < a.items) {
    const int it = threadIdx.x;
    a.info[3 * it] = static_cast<double>(ctl.status[it]);
    a.info[3 * it + 1] = static_cast<double>(ctl.iters[it]);
    a.info[3 * it + 2] = ctl.resid[it];
  }
}

template <int KP> const void *KernelFor() { return reinterpret_cast<const void *>(&PcgKernel<KP>); }

const void *SelectKernel(int kp)
{
  switch (kp) {
  case 1: return KernelFor<1>();
  case 2: return KernelFor<2>();
  case 4: return KernelFor<4>();
  case 8: return KernelFor<8>();
  case 16: return KernelFor<16>();
  case 32: return KernelFor<32>();
  default: return nullptr;
  }
}

} // namespace

int PcgMaxGrid(int kp)
{
  const void *kernel = SelectKernel(kp);
  int device = 0, sms = 0, per_sm = 0;
  if (!kernel || cudaGetDevice(&device) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPcgThreads, 0) != cudaSuccess)
    return 0;
  return sms * (per_sm < 2 ? per_sm : 2);
}

cudaError_t LaunchPcg(PcgArgs args, int *grid_out, int *block_out, cudaStream_t stream)
{
  const void *kernel = SelectKernel(args.kp);
  if (!kernel)
    return cudaErrorInvalidValue;
  const int max_grid = PcgMaxGrid(args.kp);
  if (max_grid <= 0)
    return cudaErrorInvalidConfiguration;
  const int rows_per_warp = 32 / args.kp;
  const int warp_slices = args.n_pad / rows_per_warp;
  int grid = (warp_slices + kPcgWarps - 1) / kPcgWarps;
  if (grid > max_grid)
    grid = max_grid;
  if (grid < 1)
    grid = 1;
  cudaError_t e = cudaMemsetAsync(args.barrier, 0, sizeof(unsigned), stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(args.error, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess)
    return e;
  void *params[] = {&args};
  e = cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(kPcgThreads), params, 0, stream);
  if (grid_out)
    *grid_out = grid;
  if (block_out)
    *block_out = kPcgThreads;
  return e;
}

} // namespace fg
