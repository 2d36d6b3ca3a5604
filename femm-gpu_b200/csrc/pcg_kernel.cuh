// pcg_kernel.cuh -- batched deterministic PCG as one persistent cooperative kernel.
//
// Algorithm: the reference's DeterministicPcgKernel (gpu_solver/src/solvers/
// pcg_kernels.cu:10-344): x = 0, RHS max-scaling, Jacobi-preconditioned CG, and on
// reaching the threshold a true-residual check ||b/s - A x|| <= tol ||b/s|| that
// either accepts or restarts from the true residual; the same status codes.
//
// B200 mapping: one launch runs the whole solve for up to 32 items that share the
// SELL-32 pattern.  Every CTA owns a contiguous range of rows for all items, so
// column indices are read once per row for the whole batch; a thread owns one row and
// IV adjacent items (16-byte loads of values, gathers and vectors).  A CG iteration has
// exactly two grid-wide synchronisations, each fused with its reduction: every CTA
// publishes its per-item partial sums, arrives on a release counter, and after the
// acquire reads all CTAs' partials and sums them in CTA order, so every CTA holds
// bitwise-identical scalars and takes identical branches without a broadcast step.
// The search-direction update p = z + beta p is folded into the next SpMV
// (A p = sum a_ij (z_j + beta p_j), p double-buffered), which removes the third barrier
// a textbook CG needs.  Waits are bounded by a %globaltimer budget: on expiry the kernel
// records an error and every CTA returns.
//
// Storage type T: double (the drop-in FP64 solve) or float (the inner solve of the mixed
// form: FP32 values and vectors, SpMV accumulated in FP32, every dot product and every
// scalar in FP64; with verify = 0 the inner solve stops on its recursive residual and
// the FP64 defect correction around it checks the true residual).
//
// Preconditioner BS: 0 = Jacobi (the reference default), 8 or 32 = block-Jacobi with
// dense inverses of contiguous BS-row principal blocks (the reference's opt-in
// kBlockJacobi, pcg_device.cuh:62-79, has BS = 8).  For the block form the row loops
// of the set-up, update and restart phases run in warp-steps of U = max(BS, rows per
// warp) rows, so every block lies inside one warp: the new residuals of a warp-step are
// exchanged through shared memory and z = B^-1 r is formed from the item-interleaved
// inverse (16-byte loads, coalesced across the warp); a block marked unusable (NaN in
// its first entry) falls back to the diagonal for its rows, as the reference does.
#pragma once

#include "kernels.cuh"

#include <cmath>
#include <type_traits>

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
  int flag[kMaxItems]; // 1 threshold reached, 2 verified, 3 restart, 4 residual replaced
  double rmax[kMaxItems]; // reliable updates: largest residual since the last replacement
};

// Shared-memory staging of a grid reduction of up to QM quantities (quantities x items) in
// a CTA of NW warps; the partials buffer holds 2 x QM x (row groups) doubles.  A row group
// is kPcgWarps warps with one contiguous range of rows: a CTA of 512 threads is one group,
// a CTA of 1024 threads two, so both shapes partition the rows and sum the partials alike.
template <int QM, int NW = kPcgWarps> struct ReduceQ {
  static constexpr int kQ = QM;
  static constexpr int kW = NW;
  double warp[NW][QM];
  double result[QM];
  int err;
};
using Reduce = ReduceQ<kMaxQ>;

// Phase trace of CTA 0 (PcgArgs::trace): thread 0 accumulates wall-clock intervals.
struct Trace {
  unsigned long long slot[kPcgTraceSlots];
  unsigned long long mark;
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

// IV consecutive elements of T (aligned to IV * sizeof(T)), as one vector access.
template <typename T, int IV> __device__ __forceinline__ void Load(const T *p, T (&o)[IV])
{
  if constexpr (std::is_same_v<T, double> && IV == 2) {
    const double2 t = *reinterpret_cast<const double2 *>(p);
    o[0] = t.x;
    o[1] = t.y;
  } else if constexpr (std::is_same_v<T, double> && IV == 4) {
    const double2 t = *reinterpret_cast<const double2 *>(p);
    const double2 u = *reinterpret_cast<const double2 *>(p + 2);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = u.x;
    o[3] = u.y;
  } else if constexpr (std::is_same_v<T, float> && IV == 4) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
  } else if constexpr (std::is_same_v<T, float> && IV == 2) {
    const float2 t = *reinterpret_cast<const float2 *>(p);
    o[0] = t.x;
    o[1] = t.y;
  } else {
    static_assert(IV == 1, "unsupported vector width");
    o[0] = *p;
  }
}
template <typename T, int IV> __device__ __forceinline__ void LoadRO(const T *p, T (&o)[IV])
{
  if constexpr (std::is_same_v<T, double> && IV == 2) {
    const double2 t = __ldg(reinterpret_cast<const double2 *>(p));
    o[0] = t.x;
    o[1] = t.y;
  } else if constexpr (std::is_same_v<T, double> && IV == 4) {
    const double2 t = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 u = __ldg(reinterpret_cast<const double2 *>(p + 2));
    o[0] = t.x;
    o[1] = t.y;
    o[2] = u.x;
    o[3] = u.y;
  } else if constexpr (std::is_same_v<T, float> && IV == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
  } else if constexpr (std::is_same_v<T, float> && IV == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2 *>(p));
    o[0] = t.x;
    o[1] = t.y;
  } else {
    static_assert(IV == 1, "unsupported vector width");
    o[0] = __ldg(p);
  }
}
template <typename T, int IV> __device__ __forceinline__ void Store(T *p, const T (&v)[IV])
{
  if constexpr (std::is_same_v<T, double> && IV == 2) {
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
  } else if constexpr (std::is_same_v<T, double> && IV == 4) {
    *reinterpret_cast<double2 *>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2 *>(p + 2) = make_double2(v[2], v[3]);
  } else if constexpr (std::is_same_v<T, float> && IV == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else if constexpr (std::is_same_v<T, float> && IV == 2) {
    *reinterpret_cast<float2 *>(p) = make_float2(v[0], v[1]);
  } else {
    static_assert(IV == 1, "unsupported vector width");
    *p = v[0];
  }
}
// Streaming loads (ld.global.cs: evict-first in L1 and L2) for the operator values, which
// every iteration reads exactly once and which are larger than L2: they should not evict
// the vectors and column indices that the next iteration reads again.
template <typename T, int IV> __device__ __forceinline__ void LoadStream(const T *p, T (&o)[IV])
{
  if constexpr (std::is_same_v<T, double> && IV == 2) {
    const double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
    o[0] = t.x;
    o[1] = t.y;
  } else if constexpr (std::is_same_v<T, double> && IV == 4) {
    const double2 t = __ldcs(reinterpret_cast<const double2 *>(p));
    const double2 u = __ldcs(reinterpret_cast<const double2 *>(p + 2));
    o[0] = t.x;
    o[1] = t.y;
    o[2] = u.x;
    o[3] = u.y;
  } else if constexpr (std::is_same_v<T, float> && IV == 4) {
    const float4 t = __ldcs(reinterpret_cast<const float4 *>(p));
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
    o[3] = t.w;
  } else if constexpr (std::is_same_v<T, float> && IV == 2) {
    const float2 t = __ldcs(reinterpret_cast<const float2 *>(p));
    o[0] = t.x;
    o[1] = t.y;
  } else {
    static_assert(IV == 1, "unsupported vector width");
    o[0] = __ldcs(p);
  }
}
// Operator values of one position: per item (stride KP, streamed) or one shared operator
// (stride 1, the same value for every item, cached: a shared operator is small).
template <typename T, int IV>
__device__ __forceinline__ void LoadValues(const T *base, size_t index, int stride, int per_item,
                                           int item0, T (&o)[IV])
{
  if (per_item) {
    LoadStream<T, IV>(base + index * stride + item0, o);
  } else {
    const T v = __ldg(base + index);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      o[j] = v;
  }
}
// A per-item (stride KP) or shared (stride 1, same value for every item) operand.
template <typename T, int IV>
__device__ __forceinline__ void LoadOperand(const T *base, size_t index, int stride, int per_item,
                                            int item0, T (&o)[IV])
{
  if (per_item) {
    LoadRO<T, IV>(base + index * stride + item0, o);
  } else {
    const T v = __ldg(base + index);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      o[j] = v;
  }
}

__device__ __forceinline__ double Fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float Fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// The CTAs that solve one batch together: all of a plain launch, or one group of a
// multi-plan launch (rank = this CTA's index within its group).
struct GridShape {
  int size, rank;
};

__device__ __forceinline__ void TraceMark(const PcgArgs &a, const GridShape &gs, Trace &tr, int slot)
{
  if (a.trace && gs.rank == 0 && threadIdx.x == 0) {
    const unsigned long long now = GlobalTimer();
    tr.slot[slot] += now - tr.mark;
    tr.mark = now;
  }
}

// Grid-wide barrier over a monotonically increasing arrival counter, bounded in time.
template <class R> __device__ bool GridBarrier(const PcgArgs &a, const GridShape &gs, unsigned &epoch, R &sm)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    epoch += 1;
    const unsigned target = epoch * static_cast<unsigned>(gs.size);
    __threadfence();
    AddRelease(a.barrier, 1u);
    const unsigned long long t0 = GlobalTimer();
    int err = 0;
    for (unsigned spin = 0;; ++spin) {
      const unsigned v = LoadAcquire(a.barrier);
      if (static_cast<int>(v - target) >= 0)
        break;
      // Another CTA's failure ends the wait early.  Checked on every 16th poll only: the
      // flag's load cannot start before the acquire load has returned, so checking it on
      // every poll would double the time between polls.
      if ((spin & 15u) == 15u && *reinterpret_cast<volatile int32_t *>(a.error) != 0) {
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
// fixed launch shape.  v[q][j] is this thread's partial for its item item0 + j.
template <int KP, int IV, int Q, bool kMax, class R>
__device__ bool GridReduce(const PcgArgs &a, const GridShape &gs, double (&v)[Q][IV], R &sm, unsigned &epoch,
                           int &buf, Trace &tr, int phase)
{
  static_assert(Q * KP <= R::kQ, "reduction staging too small");
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
  constexpr int H = R::kW / kPcgWarps; // row groups per CTA
  const int G = gs.size * H;            // partials per quantity, one per row group
  double *part = a.partials + static_cast<size_t>(buf) * R::kQ * G;
  if (threadIdx.x < QK * H) {
    const int h = static_cast<int>(threadIdx.x) / QK, q = static_cast<int>(threadIdx.x) % QK;
    double s = sm.warp[h * kPcgWarps][q];
    for (int w = 1; w < kPcgWarps; ++w)
      s = kMax ? fmax(s, sm.warp[h * kPcgWarps + w][q]) : s + sm.warp[h * kPcgWarps + w][q];
    part[static_cast<size_t>(q) * G + gs.rank * H + h] = s;
  }
  TraceMark(a, gs, tr, 2 * phase);
  if (!GridBarrier(a, gs, epoch, sm))
    return false;
  TraceMark(a, gs, tr, 2 * phase + 1);
  for (int t = warp; t < QK; t += R::kW) {
    // Lane-strided partials in row-group order; all of a lane's partials (ten for up to 320
    // row groups) are loaded before their adds, so the sums cost one L2 round trip.  The add
    // order, and so the result, is that of the one-at-a-time loop.  (Two quantities per
    // pass where a warp sums several measured slower at 32 items.)
    const double *pt = part + static_cast<size_t>(t) * G;
    double s = 0.0;
    for (int g = lane; g < G; g += 32 * 10) {
      double y[10];
#pragma unroll
      for (int u = 0; u < 10; ++u)
        y[u] = g + 32 * u < G ? __ldcg(pt + g + 32 * u) : 0.0;
#pragma unroll
      for (int u = 0; u < 10; ++u)
        if (g + 32 * u < G)
          s = kMax ? fmax(s, y[u]) : s + y[u];
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
  TraceMark(a, gs, tr, 8);
  if (a.trace && gs.rank == 0 && threadIdx.x == 0)
    tr.slot[9] += 1;
  buf ^= 1;
  return true;
}

// One row's product for IV items: acc_j = sum_w a_rw,j * v_j(col_w), v = z (+ beta p),
// in CSR order and in T arithmetic.  Column indices and values of a chunk of entries are
// loaded before any gather so a thread keeps many independent loads in flight.
// Asynchronous global -> shared copies (cp.async, sm_80+): 16 bytes per thread, L2
// evict-first (the operator values are read once per iteration), grouped per chunk.
__device__ __forceinline__ unsigned long long EvictFirstPolicy()
{
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void CpAsync16(void *smem, const void *gmem, unsigned long long pol)
{
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const size_t g = __cvta_generic_to_global(gmem);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(s), "l"(g), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void CpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void CpAsyncWait()
{
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Column index of SELL position pos: from the CTA's shared-memory copy when cached.
__device__ __forceinline__ int Column(const PcgArgs &a, const int32_t *colc, size_t cbase, size_t pos)
{
  return colc ? colc[pos - cbase] : __ldg(a.sell_col + pos);
}

template <typename T, int KP, int IV, bool kFold>
__device__ __forceinline__ void RowProduct(const PcgArgs &a, const int32_t *colc, size_t cbase,
                                           size_t base, int len, int item0, const T *z, const T *p,
                                           const bool (&fold)[IV], const T (&beta)[IV], T (&acc)[IV])
{
  const T *vals = static_cast<const T *>(a.values);
#pragma unroll
  for (int j = 0; j < IV; ++j)
    acc[j] = T(0);
  constexpr int U = IV >= 2 ? 4 : 8; // entries per chunk
  for (int w0 = 0; w0 < len; w0 += U) {
    int c[U];
    T v[U][IV];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      c[u] = 0;
#pragma unroll
      for (int j = 0; j < IV; ++j)
        v[u][j] = T(0);
      if (w0 + u < len) {
        const size_t pos = base + 32 * static_cast<size_t>(w0 + u);
        c[u] = Column(a, colc, cbase, pos);
        LoadValues<T, IV>(vals, pos, a.value_stride, a.value_item, item0, v[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (w0 + u < len) {
        const size_t ci = static_cast<size_t>(c[u]) * KP + item0;
        T g[IV];
        Load<T, IV>(z + ci, g);
        if constexpr (kFold) {
          T pv[IV];
          Load<T, IV>(p + ci, pv);
#pragma unroll
          for (int j = 0; j < IV; ++j)
            if (fold[j])
              g[j] = Fma(beta[j], pv[j], g[j]);
        }
#pragma unroll
        for (int j = 0; j < IV; ++j)
          acc[j] = Fma(v[u][j], g[j], acc[j]);
      }
    }
  }
}

// Reliable updates: one row of the FP64 product A64 (x64 + x32) for IV items, in CSR
// order and FP64 arithmetic (the FP32 iterate is widened before it is added).
template <int KP, int IV>
__device__ __forceinline__ void RowProductReliable(const PcgArgs &a, const int32_t *colc, size_t cbase,
                                                   size_t base, int len, int item0,
                                                   const double *x64, const float *x32,
                                                   double (&acc)[IV])
{
  const double *vals = a.values64;
#pragma unroll
  for (int j = 0; j < IV; ++j)
    acc[j] = 0.0;
  constexpr int U = 4;
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
        c[u] = Column(a, colc, cbase, pos);
        LoadValues<double, IV>(vals, pos, a.value_stride, a.value_item, item0, v[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (w0 + u < len) {
        const size_t ci = static_cast<size_t>(c[u]) * KP + item0;
        double g[IV];
        float h[IV];
        Load<double, IV>(x64 + ci, g);
        Load<float, IV>(x32 + ci, h);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          acc[j] = __fma_rn(v[u][j], g[j] + static_cast<double>(h[j]), acc[j]);
      }
    }
  }
}

// NW: warps per CTA, kPcgWarps (512 threads, one row group) or 2 kPcgWarps (1024 threads,
// two row groups): a CTA of either shape runs the same rows in the same per-warp order and
// stores one partial per row group, so both give bitwise-identical results.
template <typename T, int KP, int IV, int BS, int NW = kPcgWarps>
__device__ __forceinline__ void PcgBody(const PcgArgs &a, const GridShape gs)
{
  __shared__ ReduceQ<kMaxQ, NW> sm;
  __shared__ Control ctl;
  __shared__ Trace tr;
  constexpr int LR = KP / IV;  // lanes per row
  constexpr int S = 32 / LR;   // rows per warp
  constexpr int H = NW / kPcgWarps; // row groups per CTA
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // The warp's place in its row group, and the row group's index over the grid.
  const int gw = H == 1 ? warp : (warp & (kPcgWarps - 1));
  const int rg = H == 1 ? gs.rank : gs.rank * H + warp / kPcgWarps, RG = gs.size * H;
  const int item0 = (lane % LR) * IV;
  const int WS = a.n_pad / S;
  const int ws0 = static_cast<int>(static_cast<long long>(WS) * rg / RG);
  const int ws1 = static_cast<int>(static_cast<long long>(WS) * (rg + 1) / RG);
  unsigned epoch = 0;
  int buf = 0;
  const T *B = static_cast<const T *>(a.b);
  const T *DG = static_cast<const T *>(a.diag);
  const T *IDG = static_cast<const T *>(a.invd);
  T *X = static_cast<T *>(a.x);
  T *R = static_cast<T *>(a.r);
  T *Z = static_cast<T *>(a.z);
  T *Qv = static_cast<T *>(a.q);

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

  // z = M^-1 r for this thread's items (FP64 arithmetic, stored in T).
  auto precond = [&](const double (&rv)[IV], int r, T (&zv)[IV]) {
    T d[IV];
    if (a.use_inverse) {
      LoadOperand<T, IV>(IDG, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, d);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        zv[j] = static_cast<T>(rv[j] * static_cast<double>(d[j]));
    } else {
      LoadOperand<T, IV>(DG, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, d);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        zv[j] = static_cast<T>(rv[j] / static_cast<double>(d[j]));
    }
  };
  auto on = [&](int j) { return ctl.active[item0 + j] != 0; };

  // Block-Jacobi: warp-steps of U rows (whole blocks), SUB rows per lane, the warp's
  // residuals staged in xb[U][KP].
  constexpr int U = BS > S ? BS : S;
  constexpr int SUB = U / S;
  extern __shared__ __align__(16) unsigned char fg_dynamic_smem[];
  T *xb = reinterpret_cast<T *>(fg_dynamic_smem) + static_cast<size_t>(warp) * U * KP;
  const int WU = a.n_pad / U;
  const int wu0 = static_cast<int>(static_cast<long long>(WU) * rg / RG);
  const int wu1 = static_cast<int>(static_cast<long long>(WU) * (rg + 1) / RG);
  const T *BLK = static_cast<const T *>(a.blocks);

  // Column indices of this CTA's rows (the Phase A partition, fixed for the launch) copied
  // once into shared memory: the SpMV then gathers without a dependent global load.
  const int32_t *colc = nullptr;
  size_t cbase = 0;
  if (a.col_cache) {
    int32_t *cs = reinterpret_cast<int32_t *>(fg_dynamic_smem + a.col_cache_offset);
    // The rows of all the CTA's row groups.
    const int cws0 = static_cast<int>(static_cast<long long>(WS) * (gs.rank * H) / RG);
    const int cws1 = static_cast<int>(static_cast<long long>(WS) * (gs.rank * H + H) / RG);
    if (cws1 > cws0) {
      const int s0 = (cws0 * S) >> 5, s1 = (cws1 * S - 1) >> 5;
      const size_t p0 = static_cast<size_t>(__ldg(a.slice_off + s0));
      const size_t p1 = static_cast<size_t>(__ldg(a.slice_off + s1 + 1));
      // Positions are multiples of 32 ints (whole slice columns): copy as int4.
      const int4 *src = reinterpret_cast<const int4 *>(a.sell_col + p0);
      int4 *dst = reinterpret_cast<int4 *>(cs);
      for (size_t i = threadIdx.x; i < (p1 - p0) / 4; i += NW * 32)
        dst[i] = __ldg(src + i);
      cbase = p0;
    }
    colc = cs;
    __syncthreads();
  }
  // Row of sub-row s of this lane in warp-step wu, and its offset in xb.
  auto sub_row = [&](int wu, int s) { return wu * U + s * S + lane / LR; };
  // z for sub-row s from the staged residuals (after __syncwarp): B^-1 r over the block,
  // or the diagonal for an unusable block.  rn receives the row's own residual.
  auto block_row = [&](int wu, int s, double (&rn)[IV], T (&zn)[IV]) {
    const int ib = s * S + lane / LR;
    const int row = wu * U + ib;
    const int ii = ib % (BS > 0 ? BS : 1), first = ib - ii;
    const size_t blk = static_cast<size_t>(row - ii) * (BS > 0 ? BS : 1);
    T own[IV], head[IV], acc[IV];
    Load<T, IV>(xb + ib * KP + item0, own);
    LoadOperand<T, IV>(BLK, blk, a.block_stride, a.block_item, item0, head);
#pragma unroll
    for (int j = 0; j < IV; ++j) {
      rn[j] = static_cast<double>(own[j]);
      acc[j] = T(0);
    }
#pragma unroll 8
    for (int jj = 0; jj < BS; ++jj) {
      T bv[IV], rv[IV];
      LoadOperand<T, IV>(BLK, blk + static_cast<size_t>(jj) * BS + ii, a.block_stride,
                         a.block_item, item0, bv);
      Load<T, IV>(xb + (first + jj) * KP + item0, rv);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        acc[j] = Fma(bv[j], rv[j], acc[j]);
    }
    bool fallback = false;
#pragma unroll
    for (int j = 0; j < IV; ++j)
      fallback = fallback || isnan(static_cast<double>(head[j]));
    if (fallback) {
      T zp[IV];
      precond(rn, row, zp);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (isnan(static_cast<double>(head[j])))
          acc[j] = zp[j];
    }
#pragma unroll
    for (int j = 0; j < IV; ++j)
      zn[j] = acc[j];
  };
  auto stage = [&](int s, const T (&v)[IV]) { Store<T, IV>(xb + (s * S + lane / LR) * KP + item0, v); };

  // Reliable updates (FP32 storage only): the solution accumulates in FP64 (x64) and the
  // residual is replaced by the FP64 true residual b/s - A64 (x64 + x) whenever the
  // recursive residual has dropped by reliable_delta since the last replacement.
  constexpr bool kFloat = std::is_same_v<T, float>;
  const bool rel = kFloat && a.reliable != 0;
  // The right-hand side in FP64: b64 when reliable, else the stored T values widened.
  auto load_b = [&](size_t ri, double (&bd)[IV]) {
    if (rel) {
      Load<double, IV>(a.b64 + ri, bd);
    } else {
      T bb[IV];
      Load<T, IV>(B + ri, bb);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        bd[j] = static_cast<double>(bb[j]);
    }
  };
  // Accept-phase update of this lane's iterate for flags f: with reliable updates x is
  // folded into x64 (flags 2 and 4) and accepted items are scaled back in FP64; otherwise
  // accepted items are scaled back in place.  bad[j] counts non-finite results.
  auto settle_x = [&](size_t ri, const int (&f)[IV], const double (&sc)[IV], double (&bad)[IV]) {
    T xv[IV];
    Load<T, IV>(X + ri, xv);
    if (rel) {
      double xd[IV];
      Load<double, IV>(a.x64 + ri, xd);
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        if (f[j] == 2 || f[j] == 4) {
          xd[j] += static_cast<double>(xv[j]);
          xv[j] = T(0);
        }
        if (f[j] == 2) {
          xd[j] *= sc[j];
          if (!isfinite(xd[j]))
            bad[j] += 1.0;
        }
      }
      Store<double, IV>(a.x64 + ri, xd);
    } else {
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (f[j] == 2) {
          xv[j] = static_cast<T>(static_cast<double>(xv[j]) * sc[j]);
          if (!isfinite(static_cast<double>(xv[j])))
            bad[j] += 1.0;
        }
    }
    Store<T, IV>(X + ri, xv);
  };
  // True residual of one row for IV items: b/s - A x in T arithmetic, or with reliable
  // updates b64/s - A64 (x64 + x) in FP64.
  auto true_residual = [&](int r, size_t ri, const double (&sc)[IV], double (&t)[IV]) {
    const int len = __ldg(a.row_len + r);
    const size_t base = static_cast<size_t>(__ldg(a.slice_off + (r >> 5))) + (r & 31);
    double bd[IV];
    load_b(ri, bd);
    if constexpr (kFloat) {
      if (rel) {
        double acc[IV];
        RowProductReliable<KP, IV>(a, colc, cbase, base, len, item0, a.x64, X, acc);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          t[j] = bd[j] / sc[j] - acc[j];
        return;
      }
    }
    const bool nofold[IV] = {};
    const T nobeta[IV] = {};
    T acc[IV];
    RowProduct<T, KP, IV, false>(a, colc, cbase, base, len, item0, X, nullptr, nofold, nobeta, acc);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      t[j] = bd[j] / sc[j] - static_cast<double>(acc[j]);
  };


#define FG_ROWS_BEGIN                                                                              \
  for (int ws = ws0 + gw; ws < ws1; ws += kPcgWarps) {                                             \
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
    T dd[IV];
    double bb[IV];
    load_b(ri, bb);
    LoadOperand<T, IV>(DG, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, dd);
    if (rel) {
      const double zd[IV] = {};
      Store<double, IV>(a.x64 + ri, zd);
    }
#pragma unroll
    for (int j = 0; j < IV; ++j)
      if (on(j) && r < a.n) {
        const double bj = bb[j], dj = dd[j];
        const bool nonfinite = !isfinite(bj) || !isfinite(dj);
        if (nonfinite || !(dj > 0.0))
          v[0][j] = fmax(v[0][j], 2.0 * static_cast<double>(a.n - r) + (nonfinite ? 1.0 : 0.0));
        v[1][j] = fmax(v[1][j], fabs(bj));
      }
    T zero[IV];
#pragma unroll
    for (int j = 0; j < IV; ++j)
      zero[j] = T(0);
    Store<T, IV>(X + ri, zero);
    FG_ROWS_END
    if (!GridReduce<KP, IV, 2, true>(a, gs, v, sm, epoch, buf, tr, 3))
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
    if constexpr (BS == 0) {
      FG_ROWS_BEGIN
      T rt[IV], zv[IV];
      double bb[IV], rv[IV], re[IV];
      load_b(ri, bb);
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        re[j] = bb[j] / s[j];
        rt[j] = static_cast<T>(re[j]);
        rv[j] = rt[j];
        if (!rel)
          re[j] = rv[j];
      }
      precond(rv, r, zv);
      Store<T, IV>(R + ri, rt);
      Store<T, IV>(Z + ri, zv);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (on(j)) {
          v[0][j] += re[j] * re[j];
          v[1][j] += rv[j] * static_cast<double>(zv[j]);
        }
      FG_ROWS_END
    } else {
      for (int wu = wu0 + gw; wu < wu1; wu += kPcgWarps) {
#pragma unroll
        for (int u = 0; u < SUB; ++u) {
          const size_t ri = static_cast<size_t>(sub_row(wu, u)) * KP + item0;
          T rt[IV];
          double bb[IV];
          load_b(ri, bb);
#pragma unroll
          for (int j = 0; j < IV; ++j) {
            const double re = bb[j] / s[j];
            rt[j] = static_cast<T>(re);
            const double rr = rel ? re : static_cast<double>(rt[j]);
            if (on(j))
              v[0][j] += rr * rr;
          }
          Store<T, IV>(R + ri, rt);
          stage(u, rt);
        }
        __syncwarp();
#pragma unroll
        for (int u = 0; u < SUB; ++u) {
          double rv[IV];
          T zv[IV];
          block_row(wu, u, rv, zv);
          Store<T, IV>(Z + static_cast<size_t>(sub_row(wu, u)) * KP + item0, zv);
#pragma unroll
          for (int j = 0; j < IV; ++j)
            if (on(j))
              v[1][j] += rv[j] * static_cast<double>(zv[j]);
        }
        __syncwarp();
      }
    }
    if (!GridReduce<KP, IV, 2, false>(a, gs, v, sm, epoch, buf, tr, 3))
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
          ctl.thr[it] = (a.item_tolerance ? a.item_tolerance[it] : a.tolerance) * sqrt(rr);
          ctl.rho[it] = rho;
          ctl.restart[it] = 1;
          ctl.rmax[it] = sqrt(rr);
        }
      }
    }
    __syncthreads();
  }

  T *pc = static_cast<T *>(a.p0), *pn = static_cast<T *>(a.p1);
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
      T be[IV];
      bool any_mine = false;
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        fold[j] = !ctl.restart[item0 + j];
        be[j] = static_cast<T>(ctl.beta[item0 + j]);
        any_mine = any_mine || on(j);
      }
      // Row epilogue: p_new of the row, q = acc, and p_new . q.
      auto finish_row = [&](int r, const T (&acc)[IV]) {
        const size_t ri = static_cast<size_t>(r) * KP + item0;
        T zr[IV], pr[IV], pnew[IV];
        Load<T, IV>(Z + ri, zr);
        Load<T, IV>(pc + ri, pr);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          pnew[j] = fold[j] ? Fma(be[j], pr[j], zr[j]) : zr[j];
        Store<T, IV>(pn + ri, pnew);
        Store<T, IV>(Qv + ri, acc);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          if (on(j))
            v[0][j] += static_cast<double>(pnew[j]) * static_cast<double>(acc[j]);
      };
      constexpr bool kRing = sizeof(T) * IV == 16;
      if constexpr (kRing) {
        if (any_mine && a.value_ring) {
          // Software pipeline over this lane's (row, chunk) sequence: the values of the next
          // chunk are copied to shared memory while the current chunk's gathers are in flight.
          constexpr int U = kRingEntries;
          T *ring = reinterpret_cast<T *>(fg_dynamic_smem + a.value_ring_offset) +
                    static_cast<size_t>(warp) * 2 * U * 32 * IV;
          const T *vals = static_cast<const T *>(a.values);
          const unsigned long long pol = EvictFirstPolicy();
          auto issue = [&](int stage, size_t base, int w0, int len) {
#pragma unroll
            for (int u = 0; u < U; ++u)
              if (w0 + u < len)
                CpAsync16(ring + ((stage * U + u) * 32 + lane) * IV,
                          vals + (base + 32 * static_cast<size_t>(w0 + u)) * a.value_stride + item0, pol);
            CpAsyncCommit();
          };
          int ws = ws0 + gw, r = 0, len = 0, w0 = 0, stage = 0;
          size_t base = 0;
          auto row_at = [&](int w, int &rr, int &ll, size_t &bb) {
            rr = w * S + lane / LR;
            ll = __ldg(a.row_len + rr);
            bb = static_cast<size_t>(__ldg(a.slice_off + (rr >> 5))) + (rr & 31);
          };
          int fr = 0, flen = 0;
          size_t fbase = 0;
          if (ws < ws1) {
            row_at(ws, r, len, base);
            issue(0, base, 0, len);
            if (ws + kPcgWarps < ws1)
              row_at(ws + kPcgWarps, fr, flen, fbase);
          }
          T acc[IV];
#pragma unroll
          for (int j = 0; j < IV; ++j)
            acc[j] = T(0);
          while (ws < ws1) {
            int nws = ws, nr = r, nlen = len, nw0 = w0 + U;
            size_t nbase = base;
            if (nw0 >= len) {
              nws = ws + kPcgWarps;
              nw0 = 0;
              nr = fr;
              nlen = flen;
              nbase = fbase;
              if (nws + kPcgWarps < ws1)
                row_at(nws + kPcgWarps, fr, flen, fbase);
            }
            if (nws < ws1)
              issue(stage ^ 1, nbase, nw0, nlen);
            else
              CpAsyncCommit();
            CpAsyncWait<1>(); // the current chunk's values have landed
            int c[U];
#pragma unroll
            for (int u = 0; u < U; ++u)
              c[u] = w0 + u < len ? Column(a, colc, cbase, base + 32 * static_cast<size_t>(w0 + u)) : 0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
              if (w0 + u < len) {
                const size_t ci = static_cast<size_t>(c[u]) * KP + item0;
                T g[IV], pv[IV], vv[IV];
                Load<T, IV>(Z + ci, g);
                Load<T, IV>(pc + ci, pv);
                Load<T, IV>(ring + ((stage * U + u) * 32 + lane) * IV, vv);
#pragma unroll
                for (int j = 0; j < IV; ++j) {
                  if (fold[j])
                    g[j] = Fma(be[j], pv[j], g[j]);
                  acc[j] = Fma(vv[j], g[j], acc[j]);
                }
              }
            }
            if (w0 + U >= len) {
              finish_row(r, acc);
#pragma unroll
              for (int j = 0; j < IV; ++j)
                acc[j] = T(0);
            }
            ws = nws;
            r = nr;
            len = nlen;
            w0 = nw0;
            base = nbase;
            stage ^= 1;
          }
          CpAsyncWait<0>();
          any_mine = false; // done
        }
      }
      if (any_mine) {
        FG_ROWS_BEGIN
        const int len = __ldg(a.row_len + r);
        const size_t base = static_cast<size_t>(__ldg(a.slice_off + (r >> 5))) + (r & 31);
        T acc[IV];
        RowProduct<T, KP, IV, true>(a, colc, cbase, base, len, item0, Z, pc, fold, be, acc);
        (void)ri;
        finish_row(r, acc);
        FG_ROWS_END
      }
      if (!GridReduce<KP, IV, 1, false>(a, gs, v, sm, epoch, buf, tr, 0))
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
      T *t = pc;
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
      if constexpr (BS > 0) {
        if (__any_sync(0xffffffffu, mine))
          for (int wu = wu0 + gw; wu < wu1; wu += kPcgWarps) {
            T xo[SUB][IV], po[SUB][IV], ro[SUB][IV], qo[SUB][IV];
#pragma unroll
            for (int u = 0; u < SUB; ++u) {
              const size_t ri = static_cast<size_t>(sub_row(wu, u)) * KP + item0;
              Load<T, IV>(X + ri, xo[u]);
              Load<T, IV>(pc + ri, po[u]);
              Load<T, IV>(R + ri, ro[u]);
              Load<T, IV>(Qv + ri, qo[u]);
            }
#pragma unroll
            for (int u = 0; u < SUB; ++u) {
              const size_t ri = static_cast<size_t>(sub_row(wu, u)) * KP + item0;
              T rt[IV], xn[IV];
#pragma unroll
              for (int j = 0; j < IV; ++j) {
                const double rr = on(j) ? static_cast<double>(ro[u][j]) - al[j] * static_cast<double>(qo[u][j])
                                        : static_cast<double>(ro[u][j]);
                rt[j] = static_cast<T>(rr);
                xn[j] = on(j) ? static_cast<T>(static_cast<double>(xo[u][j]) + al[j] * static_cast<double>(po[u][j]))
                              : xo[u][j];
              }
              Store<T, IV>(X + ri, xn);
              Store<T, IV>(R + ri, rt);
              stage(u, rt);
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < SUB; ++u) {
              double rn[IV];
              T zn[IV];
              block_row(wu, u, rn, zn);
              Store<T, IV>(Z + static_cast<size_t>(sub_row(wu, u)) * KP + item0, zn);
#pragma unroll
              for (int j = 0; j < IV; ++j)
                if (on(j)) {
                  v[0][j] += rn[j] * rn[j];
                  v[1][j] += rn[j] * static_cast<double>(zn[j]);
                }
            }
            __syncwarp();
          }
      } else if (mine) {
        // Two row groups per pass: all loads are issued before the first store.
        for (int ws = ws0 + gw; ws < ws1; ws += 2 * kPcgWarps) {
          const bool two = ws + kPcgWarps < ws1;
          const int r0 = ws * S + lane / LR, r1 = (ws + kPcgWarps) * S + lane / LR;
          const size_t i0 = static_cast<size_t>(r0) * KP + item0;
          const size_t i1 = static_cast<size_t>(r1) * KP + item0;
          T x0[IV], p0[IV], rv0[IV], q0[IV], x1[IV], p1[IV], rv1[IV], q1[IV];
          Load<T, IV>(X + i0, x0);
          Load<T, IV>(pc + i0, p0);
          Load<T, IV>(R + i0, rv0);
          Load<T, IV>(Qv + i0, q0);
          if (two) {
            Load<T, IV>(X + i1, x1);
            Load<T, IV>(pc + i1, p1);
            Load<T, IV>(R + i1, rv1);
            Load<T, IV>(Qv + i1, q1);
          }
          double rn[IV];
          T rt[IV], zn[IV], xn[IV];
#pragma unroll
          for (int j = 0; j < IV; ++j) {
            const double rr = on(j) ? static_cast<double>(rv0[j]) - al[j] * static_cast<double>(q0[j])
                                    : static_cast<double>(rv0[j]);
            rt[j] = static_cast<T>(rr);
            rn[j] = rt[j];
            xn[j] = on(j) ? static_cast<T>(static_cast<double>(x0[j]) + al[j] * static_cast<double>(p0[j]))
                          : x0[j];
          }
          precond(rn, r0, zn);
          Store<T, IV>(X + i0, xn);
          Store<T, IV>(R + i0, rt);
          Store<T, IV>(Z + i0, zn);
#pragma unroll
          for (int j = 0; j < IV; ++j)
            if (on(j)) {
              v[0][j] += rn[j] * rn[j];
              v[1][j] += rn[j] * static_cast<double>(zn[j]);
            }
          if (two) {
#pragma unroll
            for (int j = 0; j < IV; ++j) {
              const double rr = on(j) ? static_cast<double>(rv1[j]) - al[j] * static_cast<double>(q1[j])
                                      : static_cast<double>(rv1[j]);
              rt[j] = static_cast<T>(rr);
              rn[j] = rt[j];
              xn[j] = on(j) ? static_cast<T>(static_cast<double>(x1[j]) + al[j] * static_cast<double>(p1[j]))
                            : x1[j];
            }
            precond(rn, r1, zn);
            Store<T, IV>(X + i1, xn);
            Store<T, IV>(R + i1, rt);
            Store<T, IV>(Z + i1, zn);
#pragma unroll
            for (int j = 0; j < IV; ++j)
              if (on(j)) {
                v[0][j] += rn[j] * rn[j];
                v[1][j] += rn[j] * static_cast<double>(zn[j]);
              }
          }
        }
      }
      if (!GridReduce<KP, IV, 2, false>(a, gs, v, sm, epoch, buf, tr, 1))
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
            } else if (ctl.resid[it] <= ctl.thr[it]) {
              // The drop-in solve verifies the true residual; an inner solve whose caller
              // checks the true residual may accept here.
              ctl.flag[it] = a.skip_verification && !rel ? 2 : 1;
            } else if (rel && ctl.resid[it] < a.reliable_delta * ctl.rmax[it]) {
              ctl.flag[it] = 4;
            }
            if (rel)
              ctl.rmax[it] = fmax(ctl.rmax[it], ctl.resid[it]);
          }
        }
      }
      __syncthreads();
    }

    bool verify = false, accept = false;
#pragma unroll
    for (int it = 0; it < KP; ++it) {
      verify = verify || (ctl.active[it] && (ctl.flag[it] == 1 || (rel && ctl.flag[it] == 4)));
      accept = accept || (ctl.active[it] && ctl.flag[it] == 2);
    }
    if (verify) {
      // True residual for items at the threshold.
      double v[1][IV];
      bool mine[IV], any_mine = false;
      double s[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        const int fl = ctl.flag[item0 + j];
        mine[j] = on(j) && (fl == 1 || (rel && fl == 4));
        any_mine = any_mine || mine[j];
        s[j] = ctl.scale[item0 + j];
      }
      if (any_mine) {
        FG_ROWS_BEGIN
        T rv[IV];
        double t[IV];
        true_residual(r, ri, s, t);
        Load<T, IV>(R + ri, rv);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          if (mine[j]) {
            rv[j] = static_cast<T>(t[j]);
            v[0][j] += t[j] * t[j];
          }
        Store<T, IV>(R + ri, rv);
        FG_ROWS_END
      }
      if (!GridReduce<KP, IV, 1, false>(a, gs, v, sm, epoch, buf, tr, 2))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        if (ctl.active[it] && (ctl.flag[it] == 1 || (rel && ctl.flag[it] == 4))) {
          const double trr = sm.result[it];
          if (!isfinite(trr)) {
            ctl.status[it] = kNonfinite;
            ctl.active[it] = 0;
          } else {
            // Reliable updates keep the search direction after a replacement; the
            // drop-in solve restarts from the true residual as the reference does.
            ctl.resid[it] = sqrt(trr);
            ctl.flag[it] = ctl.resid[it] <= ctl.thr[it] ? 2 : (rel ? 4 : 3);
            if (rel)
              ctl.rmax[it] = ctl.resid[it];
          }
        }
      }
      __syncthreads();
    }
    if (verify || accept) {
      // Accept (scale x back) or restart from the true residual.
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
      if constexpr (BS > 0) {
        if (__any_sync(0xffffffffu, any_mine))
          for (int wu = wu0 + gw; wu < wu1; wu += kPcgWarps) {
#pragma unroll
            for (int u = 0; u < SUB; ++u) {
              T rv[IV];
              Load<T, IV>(R + static_cast<size_t>(sub_row(wu, u)) * KP + item0, rv);
              stage(u, rv);
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < SUB; ++u) {
              const size_t ri = static_cast<size_t>(sub_row(wu, u)) * KP + item0;
              T zv[IV], zo[IV];
              double rd[IV];
              settle_x(ri, f, s, v[1]);
              Load<T, IV>(Z + ri, zo);
              block_row(wu, u, rd, zv);
#pragma unroll
              for (int j = 0; j < IV; ++j) {
                if (f[j] == 3 || f[j] == 4)
                  v[0][j] += rd[j] * static_cast<double>(zv[j]);
                else
                  zv[j] = zo[j];
              }
              Store<T, IV>(Z + ri, zv);
            }
            __syncwarp();
          }
      } else if (any_mine) {
        FG_ROWS_BEGIN
        T rv[IV], zv[IV], zo[IV];
        double rd[IV];
        settle_x(ri, f, s, v[1]);
        Load<T, IV>(R + ri, rv);
        Load<T, IV>(Z + ri, zo);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          rd[j] = rv[j];
        precond(rd, r, zv);
#pragma unroll
        for (int j = 0; j < IV; ++j) {
          if (f[j] == 3 || f[j] == 4)
            v[0][j] += rd[j] * static_cast<double>(zv[j]);
          else
            zv[j] = zo[j];
        }
        Store<T, IV>(Z + ri, zv);
        FG_ROWS_END
      }
      if (!GridReduce<KP, IV, 2, false>(a, gs, v, sm, epoch, buf, tr, 2))
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
        } else if (ctl.active[it] && ctl.flag[it] == 4) {
          ctl.rz[it] = sm.result[it]; // r.z of the replaced residual; beta follows below
        }
      }
      __syncthreads();
    }
    if (threadIdx.x < KP) {
      const int it = threadIdx.x;
      if (ctl.active[it] && (ctl.flag[it] == 0 || ctl.flag[it] == 4)) {
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
      FG_ROWS_BEGIN
      T rv[IV];
      double t[IV];
      true_residual(r, ri, s, t);
      Load<T, IV>(R + ri, rv);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (on(j)) {
          rv[j] = static_cast<T>(t[j]);
          v[0][j] += t[j] * t[j];
        }
      Store<T, IV>(R + ri, rv);
      FG_ROWS_END
      if (!GridReduce<KP, IV, 1, false>(a, gs, v, sm, epoch, buf, tr, 3))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        if (ctl.active[it]) {
          const double trr = sm.result[it];
          if (!isfinite(trr)) {
            ctl.status[it] = kNonfinite;
            ctl.active[it] = 0;
          } else {
            ctl.rz[it] = trr;
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
      int f[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j)
        f[j] = on(j) ? 2 : 0;
      FG_ROWS_BEGIN
      settle_x(ri, f, s, v[0]);
      FG_ROWS_END
      if (!GridReduce<KP, IV, 1, false>(a, gs, v, sm, epoch, buf, tr, 3))
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

  if (gs.rank == 0 && threadIdx.x < a.items) {
    const int it = threadIdx.x;
    a.info[3 * it] = static_cast<double>(ctl.status[it]);
    a.info[3 * it + 1] = static_cast<double>(ctl.iters[it]);
    a.info[3 * it + 2] = ctl.resid[it];
  }
  if (a.trace && gs.rank == 0 && threadIdx.x == 0)
    for (int s = 0; s < kPcgTraceSlots; ++s)
      a.trace[s] += tr.slot[s];
}

template <typename T, int KP, int IV, int BS, int NW = kPcgWarps>
__global__ void __launch_bounds__(NW * 32, 2 * kPcgWarps / NW) PcgKernel(PcgArgs a)
{
  PcgBody<T, KP, IV, BS, NW>(a, GridShape{static_cast<int>(gridDim.x), static_cast<int>(blockIdx.x)});
}

// Several independent PCG solves (one per plan: its own operator, vectors, barrier and
// partials) in one cooperative launch: CTA b belongs to group cta_group[b] and is rank
// b - group_first of its group's group_size CTAs.
template <typename T, int KP, int IV, int BS>
__global__ void __launch_bounds__(kPcgThreads, 2) MultiPcgKernel(PcgGroups t)
{
  __shared__ PcgArgs group_args;
  const int g = t.cta_group[blockIdx.x];
  if (threadIdx.x == 0)
    group_args = t.args[g];
  __syncthreads();
  PcgBody<T, KP, IV, BS>(group_args,
                         GridShape{t.group_size[g], static_cast<int>(blockIdx.x) - t.group_first[g]});
}

} // namespace
} // namespace fg
