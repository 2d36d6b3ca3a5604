// pcg.cu -- batched deterministic Jacobi PCG as one persistent cooperative kernel.
//
// Algorithm: the reference's DeterministicPcgKernel (gpu_solver/src/solvers/
// pcg_kernels.cu:10-344): x = 0, RHS max-scaling, Jacobi-preconditioned CG, and on
// reaching the threshold a true-residual check ||b/s - A x|| <= tol ||b/s|| that
// either accepts or restarts from the true residual; the same status codes.
//
// B200 mapping: one launch runs the whole solve for up to 32 items that share the
// SELL-32 pattern.  Every CTA owns a contiguous range of rows for all items, so
// column indices are read once per row for the whole batch; a thread owns one row and
// IV adjacent items (16-byte loads of values, gathers and vectors when IV = 2).  A CG
// iteration has exactly two grid-wide synchronisations, each fused with its
// reduction: every CTA publishes its per-item partial sums, arrives on a release
// counter, and after the acquire reads all CTAs' partials and sums them in CTA order,
// so every CTA holds bitwise-identical scalars and takes identical branches without a
// broadcast step.  The search-direction update p = z + beta p is folded into the next
// SpMV (A p = sum a_ij (z_j + beta p_j), p double-buffered), which removes the third
// barrier a textbook CG needs.  Waits are bounded by a %globaltimer budget: on expiry
// the kernel records an error and every CTA returns.
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

// IV consecutive doubles (16-byte aligned when IV = 2).
template <int IV> __device__ __forceinline__ void Load(const double *p, double (&o)[IV])
{
  if constexpr (IV == 2) {
    const double2 t = *reinterpret_cast<const double2 *>(p);
    o[0] = t.x;
    o[1] = t.y;
  } else {
    o[0] = *p;
  }
}
template <int IV> __device__ __forceinline__ void LoadRO(const double *p, double (&o)[IV])
{
  if constexpr (IV == 2) {
    const double2 t = __ldg(reinterpret_cast<const double2 *>(p));
    o[0] = t.x;
    o[1] = t.y;
  } else {
    o[0] = __ldg(p);
  }
}
template <int IV> __device__ __forceinline__ void Store(double *p, const double (&v)[IV])
{
  if constexpr (IV == 2)
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  else
    *p = v[0];
}
// A per-item (stride KP) or shared (stride 1, same value for every item) operand.
template <int IV>
__device__ __forceinline__ void LoadOperand(const double *base, size_t index, int stride, int per_item,
                                            int item0, double (&o)[IV])
{
  if (per_item) {
    LoadRO<IV>(base + index * stride + item0, o);
  } else {
    const double v = __ldg(base + index);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      o[j] = v;
  }
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

// Phase trace of CTA 0 (PcgArgs::trace): thread 0 accumulates wall-clock intervals.
struct Trace {
  unsigned long long slot[kPcgTraceSlots];
  unsigned long long mark;
};

__device__ __forceinline__ void TraceMark(const PcgArgs &a, Trace &tr, int slot)
{
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long now = GlobalTimer();
    tr.slot[slot] += now - tr.mark;
    tr.mark = now;
  }
}

// Sum (or max) of Q per-item quantities over the whole grid, deterministic for a
// fixed launch shape.  v[q][j] is this thread's partial for its item item0 + j.
template <int KP, int IV, int Q, bool kMax>
__device__ bool GridReduce(const PcgArgs &a, double (&v)[Q][IV], Reduce &sm, unsigned &epoch,
                           int &buf, Trace &tr, int phase)
{
  constexpr int LR = KP / IV; // lanes per row
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int j = 0; j < IV; ++j) {
      double x = v[q][j];
#pragma unroll
      for (int off = 16; off >= LR; off >>= 1) {
        const double y = __shfl_xor_sync(0xffffffffu, x, off);
        x = kMax ? fmax(x, y) : x + y;
      }
      if (lane < LR)
        sm.warp[warp][q * KP + lane * IV + j] = x;
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
  TraceMark(a, tr, 2 * phase);
  if (!GridBarrier(a, epoch, sm))
    return false;
  TraceMark(a, tr, 2 * phase + 1);
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
  TraceMark(a, tr, 8);
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0)
    tr.slot[9] += 1;
  buf ^= 1;
  return true;
}

// One row's product for IV items: acc_j = sum_w a_rw,j * v_j(col_w), v = z (+ beta p),
// in CSR order.  Column indices and values of a chunk of entries (8 scalar or 4 paired)
// are loaded before any gather so a thread keeps many independent loads in flight.
template <int KP, int IV, bool kFold>
__device__ __forceinline__ void RowProduct(const PcgArgs &a, size_t base, int len, int item0,
                                           const double *z, const double *p,
                                           const bool (&fold)[IV], const double (&beta)[IV],
                                           double (&acc)[IV])
{
#pragma unroll
  for (int j = 0; j < IV; ++j)
    acc[j] = 0.0;
  constexpr int U = 8 / IV; // entries per chunk: 8 scalar or 4 paired loads
  for (int w0 = 0; w0 < len; w0 += U) {
    int c[U];
    double v[U][IV];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      c[u] = 0;
#pragma unroll
      for (int j = 0; j < IV; ++j)
        v[u][j] = 0.0;
      if (w0 + u < len) {
        const size_t pos = base + 32 * static_cast<size_t>(w0 + u);
        c[u] = __ldg(a.sell_col + pos);
        LoadOperand<IV>(a.values, pos, a.value_stride, a.value_item, item0, v[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (w0 + u < len) {
        const size_t ci = static_cast<size_t>(c[u]) * KP + item0;
        double g[IV];
        Load<IV>(z + ci, g);
        if constexpr (kFold) {
          double pv[IV];
          Load<IV>(p + ci, pv);
#pragma unroll
          for (int j = 0; j < IV; ++j)
            if (fold[j])
              g[j] = __fma_rn(beta[j], pv[j], g[j]);
        }
#pragma unroll
        for (int j = 0; j < IV; ++j)
          acc[j] = __fma_rn(v[u][j], g[j], acc[j]);
      }
    }
  }
}

template <int KP, int IV>
__global__ void __launch_bounds__(kPcgThreads, 2) PcgKernel(PcgArgs a)
{
  __shared__ Reduce sm;
  __shared__ Control ctl;
  __shared__ Trace tr;
  constexpr int LR = KP / IV;  // lanes per row
  constexpr int S = 32 / LR;   // rows per warp
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int item0 = (lane % LR) * IV;
  const int WS = a.n_pad / S;
  const int ws0 = static_cast<int>(static_cast<long long>(WS) * blockIdx.x / gridDim.x);
  const int ws1 = static_cast<int>(static_cast<long long>(WS) * (blockIdx.x + 1) / gridDim.x);
  unsigned epoch = 0;
  int buf = 0;

  if (threadIdx.x < KP) {
    const int it = threadIdx.x;
    ctl.active[it] = (it < a.items && ((a.active_mask >> it) & 1u)) ? 1 : 0;
    ctl.status[it] = kInternal;
    ctl.iters[it] = 0;
    ctl.resid[it] = INFINITY;
    ctl.restart[it] = 1;
    ctl.flag[it] = 0;
    ctl.beta[it] = 0.0;
    ctl.scale[it] = 1.0;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kPcgTraceSlots; ++s)
      tr.slot[s] = 0;
    tr.mark = GlobalTimer();
  }
  __syncthreads();

  // z = M^-1 r for this thread's items.
  auto precond = [&](const double (&rv)[IV], int r, double (&zv)[IV]) {
    double d[IV];
    if (a.use_inverse) {
      LoadOperand<IV>(a.invd, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, d);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        zv[j] = rv[j] * d[j];
    } else {
      LoadOperand<IV>(a.diag, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, d);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        zv[j] = rv[j] / d[j];
    }
  };
  auto on = [&](int j) { return ctl.active[item0 + j] != 0; };

#define FG_ROWS_BEGIN                                                                              \
  for (int ws = ws0 + warp; ws < ws1; ws += kPcgWarps) {                                           \
    const int r = ws * S + lane / LR;                                                              \
    const size_t ri = static_cast<size_t>(r) * KP + item0;
#define FG_ROWS_END }

  // Validity (first invalid row decides the status) and RHS max-scaling.
  {
    double v[2][IV];
#pragma unroll
    for (int j = 0; j < IV; ++j)
      v[0][j] = v[1][j] = 0.0;
    FG_ROWS_BEGIN
    double bb[IV], dd[IV];
    Load<IV>(a.b + ri, bb);
    LoadOperand<IV>(a.diag, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, dd);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      if (on(j) && r < a.n) {
        const bool nonfinite = !isfinite(bb[j]) || !isfinite(dd[j]);
        if (nonfinite || !(dd[j] > 0.0))
          v[0][j] = fmax(v[0][j], 2.0 * static_cast<double>(a.n - r) + (nonfinite ? 1.0 : 0.0));
        v[1][j] = fmax(v[1][j], fabs(bb[j]));
      }
    double zero[IV];
#pragma unroll
    for (int j = 0; j < IV; ++j)
      zero[j] = 0.0;
    Store<IV>(a.x + ri, zero);
    FG_ROWS_END
    if (!GridReduce<KP, IV, 2, true>(a, v, sm, epoch, buf, tr, 3))
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
    double v[2][IV], s[IV];
#pragma unroll
    for (int j = 0; j < IV; ++j) {
      v[0][j] = v[1][j] = 0.0;
      s[j] = ctl.scale[item0 + j] != 0.0 ? ctl.scale[item0 + j] : 1.0;
    }
    FG_ROWS_BEGIN
    double bb[IV], rv[IV], zv[IV];
    Load<IV>(a.b + ri, bb);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      rv[j] = bb[j] / s[j];
    precond(rv, r, zv);
    Store<IV>(a.r + ri, rv);
    Store<IV>(a.z + ri, zv);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      if (on(j)) {
        v[0][j] += rv[j] * rv[j];
        v[1][j] += rv[j] * zv[j];
      }
    FG_ROWS_END
    if (!GridReduce<KP, IV, 2, false>(a, v, sm, epoch, buf, tr, 3))
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
      double v[1][IV];
      bool fold[IV];
      double be[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        fold[j] = !ctl.restart[item0 + j];
        be[j] = ctl.beta[item0 + j];
      }
      bool any_mine = false;
#pragma unroll
      for (int j = 0; j < IV; ++j)
        any_mine = any_mine || on(j);
      if (any_mine) {
        FG_ROWS_BEGIN
        const int len = __ldg(a.row_len + r);
        const size_t base = static_cast<size_t>(__ldg(a.slice_off + (r >> 5))) + (r & 31);
        double acc[IV], zr[IV], pr[IV], pnew[IV];
        RowProduct<KP, IV, true>(a, base, len, item0, a.z, pc, fold, be, acc);
        Load<IV>(a.z + ri, zr);
        Load<IV>(pc + ri, pr);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          pnew[j] = fold[j] ? __fma_rn(be[j], pr[j], zr[j]) : zr[j];
        Store<IV>(pn + ri, pnew);
        Store<IV>(a.q + ri, acc);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          if (on(j))
            v[0][j] += pnew[j] * acc[j];
        FG_ROWS_END
      }
      if (!GridReduce<KP, IV, 1, false>(a, v, sm, epoch, buf, tr, 0))
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
      double v[2][IV], al[IV];
      bool mine = false;
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = v[1][j] = 0.0;
        al[j] = on(j) ? ctl.alpha[item0 + j] : 0.0;
        mine = mine || on(j);
      }
      if (mine) {
        // Two row groups per pass: all loads are issued before the first store.
        for (int ws = ws0 + warp; ws < ws1; ws += 2 * kPcgWarps) {
          const bool two = ws + kPcgWarps < ws1;
          const int r0 = ws * S + lane / LR, r1 = (ws + kPcgWarps) * S + lane / LR;
          const size_t i0 = static_cast<size_t>(r0) * KP + item0;
          const size_t i1 = static_cast<size_t>(r1) * KP + item0;
          double x0[IV], p0[IV], rv0[IV], q0[IV], x1[IV], p1[IV], rv1[IV], q1[IV];
          Load<IV>(a.x + i0, x0);
          Load<IV>(pc + i0, p0);
          Load<IV>(a.r + i0, rv0);
          Load<IV>(a.q + i0, q0);
          if (two) {
            Load<IV>(a.x + i1, x1);
            Load<IV>(pc + i1, p1);
            Load<IV>(a.r + i1, rv1);
            Load<IV>(a.q + i1, q1);
          }
          double rn[IV], zn[IV], xn[IV];
#pragma unroll
          for (int j = 0; j < IV; ++j) {
            rn[j] = on(j) ? rv0[j] - al[j] * q0[j] : rv0[j];
            xn[j] = on(j) ? x0[j] + al[j] * p0[j] : x0[j];
          }
          precond(rn, r0, zn);
          Store<IV>(a.x + i0, xn);
          Store<IV>(a.r + i0, rn);
          Store<IV>(a.z + i0, zn);
#pragma unroll
          for (int j = 0; j < IV; ++j)
            if (on(j)) {
              v[0][j] += rn[j] * rn[j];
              v[1][j] += rn[j] * zn[j];
            }
          if (two) {
#pragma unroll
            for (int j = 0; j < IV; ++j) {
              rn[j] = on(j) ? rv1[j] - al[j] * q1[j] : rv1[j];
              xn[j] = on(j) ? x1[j] + al[j] * p1[j] : x1[j];
            }
            precond(rn, r1, zn);
            Store<IV>(a.x + i1, xn);
            Store<IV>(a.r + i1, rn);
            Store<IV>(a.z + i1, zn);
#pragma unroll
            for (int j = 0; j < IV; ++j)
              if (on(j)) {
                v[0][j] += rn[j] * rn[j];
                v[1][j] += rn[j] * zn[j];
              }
          }
        }
      }
      if (!GridReduce<KP, IV, 2, false>(a, v, sm, epoch, buf, tr, 1))
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
        double v[1][IV];
        bool mine[IV], any_mine = false;
        double s[IV];
#pragma unroll
        for (int j = 0; j < IV; ++j) {
          v[0][j] = 0.0;
          mine[j] = on(j) && ctl.flag[item0 + j];
          any_mine = any_mine || mine[j];
          s[j] = ctl.scale[item0 + j];
        }
        if (any_mine) {
          const bool nofold[IV] = {};
          const double nobeta[IV] = {};
          FG_ROWS_BEGIN
          const int len = __ldg(a.row_len + r);
          const size_t base = static_cast<size_t>(__ldg(a.slice_off + (r >> 5))) + (r & 31);
          double acc[IV], bb[IV], rv[IV];
          RowProduct<KP, IV, false>(a, base, len, item0, a.x, nullptr, nofold, nobeta, acc);
          Load<IV>(a.b + ri, bb);
          Load<IV>(a.r + ri, rv);
#pragma unroll
          for (int j = 0; j < IV; ++j)
            if (mine[j]) {
              rv[j] = bb[j] / s[j] - acc[j];
              v[0][j] += rv[j] * rv[j];
            }
          Store<IV>(a.r + ri, rv);
          FG_ROWS_END
        }
        if (!GridReduce<KP, IV, 1, false>(a, v, sm, epoch, buf, tr, 2))
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
        double v[2][IV];
        int f[IV];
        bool any_mine = false;
        double s[IV];
#pragma unroll
        for (int j = 0; j < IV; ++j) {
          v[0][j] = v[1][j] = 0.0;
          f[j] = on(j) ? ctl.flag[item0 + j] : 0;
          any_mine = any_mine || f[j] >= 2;
          s[j] = ctl.scale[item0 + j];
        }
        if (any_mine) {
          FG_ROWS_BEGIN
          double xv[IV], rv[IV], zv[IV], zo[IV];
          Load<IV>(a.x + ri, xv);
          Load<IV>(a.r + ri, rv);
          Load<IV>(a.z + ri, zo);
          precond(rv, r, zv);
#pragma unroll
          for (int j = 0; j < IV; ++j) {
            if (f[j] == 2) {
              xv[j] *= s[j];
              if (!isfinite(xv[j]))
                v[1][j] += 1.0;
            }
            if (f[j] == 3)
              v[0][j] += rv[j] * zv[j];
            else
              zv[j] = zo[j];
          }
          Store<IV>(a.x + ri, xv);
          Store<IV>(a.z + ri, zv);
          FG_ROWS_END
        }
        if (!GridReduce<KP, IV, 2, false>(a, v, sm, epoch, buf, tr, 2))
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

  // Iteration budget exhausted: report the true residual and scale the iterate back.
  bool any = false;
#pragma unroll
  for (int it = 0; it < KP; ++it)
    any = any || ctl.active[it];
  if (any) {
    {
      double v[1][IV];
      double s[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        s[j] = ctl.scale[item0 + j];
      }
      const bool nofold[IV] = {};
      const double nobeta[IV] = {};
      FG_ROWS_BEGIN
      const int len = __ldg(a.row_len + r);
      const size_t base = static_cast<size_t>(__ldg(a.slice_off + (r >> 5))) + (r & 31);
      double acc[IV], bb[IV], rv[IV];
      RowProduct<KP, IV, false>(a, base, len, item0, a.x, nullptr, nofold, nobeta, acc);
      Load<IV>(a.b + ri, bb);
      Load<IV>(a.r + ri, rv);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (on(j)) {
          rv[j] = bb[j] / s[j] - acc[j];
          v[0][j] += rv[j] * rv[j];
        }
      Store<IV>(a.r + ri, rv);
      FG_ROWS_END
      if (!GridReduce<KP, IV, 1, false>(a, v, sm, epoch, buf, tr, 3))
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
      double v[1][IV];
      double s[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        s[j] = ctl.scale[item0 + j];
      }
      FG_ROWS_BEGIN
      double xv[IV];
      Load<IV>(a.x + ri, xv);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (on(j)) {
          xv[j] *= s[j];
          if (!isfinite(xv[j]))
            v[0][j] += 1.0;
        }
      Store<IV>(a.x + ri, xv);
      FG_ROWS_END
      if (!GridReduce<KP, IV, 1, false>(a, v, sm, epoch, buf, tr, 3))
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
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0)
    for (int s = 0; s < kPcgTraceSlots; ++s)
      a.trace[s] += tr.slot[s];
}

template <int KP, int IV> const void *KernelFor()
{
  return reinterpret_cast<const void *>(&PcgKernel<KP, IV>);
}

const void *SelectKernel(int kp)
{
  switch (kp) {
  case 1: return KernelFor<1, 1>();
  case 2: return KernelFor<2, 2>();
  case 4: return KernelFor<4, 2>();
  case 8: return KernelFor<8, 2>();
  case 16: return KernelFor<16, 2>();
  case 32: return KernelFor<32, 2>();
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
  const int iv = args.kp >= 2 ? 2 : 1;
  const int rows_per_warp = 32 * iv / args.kp;
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
