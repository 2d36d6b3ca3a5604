// pcg1r_kernel.cuh -- the one-reduction form of the batched FP64 Jacobi PCG (opt-in plan
// flag FG_PLAN_PCG_ONE_REDUCTION; no counterpart in the reference).
//
// The two-barrier kernel (pcg_kernel.cuh) needs two grid-wide reductions per CG
// iteration, p.Ap and then r.z, because the step length depends on the first.  At
// mid-size meshes (tens of thousands of rows) a CG iteration is short and the two grid
// barriers, with the wait for the slowest CTA at each, take half of it.  Chronopoulos and
// Gear's rearrangement (J. Comput. Appl. Math. 25 (1989) 153-168) carries w = A u beside
// the preconditioned residual u = M^-1 r, so that both inner products of an iteration,
// gamma = (r, u) and delta = (w, u), are taken together after the SpMV:
//
//   beta_i  = gamma_i / gamma_{i-1},  alpha_i = gamma_i / (delta_i - beta_i gamma_i / alpha_{i-1})
//   p_i = u_i + beta_i p_{i-1},   s_i = w_i + beta_i s_{i-1}
//   x_{i+1} = x_i + alpha_i p_i,  r_{i+1} = r_i - alpha_i s_i,  u_{i+1} = M^-1 r_{i+1}
//   w_{i+1} = A u_{i+1};  gamma_{i+1}, delta_{i+1}, (r_{i+1}, r_{i+1})  -- one reduction
//
// With the Jacobi preconditioner M = D every vector is kept divided by the diagonal:
// u = r / d, m = w / d, t = s / d, so u_{i+1} = u_i - alpha_i (m_i + beta_i t_{i-1}), and
// gamma = sum d u^2, delta = sum w u, (r, r) = sum (d u)^2.  After the reduction every CTA
// knows alpha_i and beta_i, and the SpMV forms u_{i+1} of each gathered column from the
// stored u_i, m_i, t_{i-1} (three gathered vectors instead of the two-barrier kernel's
// two) in exactly the operations the row's owner uses for its own row, so every CTA sees
// the same u_{i+1}.  u, m and t are double-buffered: a CTA writes iteration i+1's values
// of its rows while others still gather iteration i's.  One grid barrier per iteration.
//
// Acceptance is unchanged: RHS max-scaling, the threshold on the recursive residual, the
// true-residual check ||b/s - A x|| <= tol ||b/s|| that accepts or restarts from the true
// residual, the same status codes and iteration count (one x update per iteration).
// Rounding differs from the two-barrier form, so results agree with it within the
// solve's tolerance, not bit for bit; a launch is deterministic for a fixed shape.
#pragma once

#include "pcg_kernel.cuh"

namespace fg
{
namespace
{

// Three sums per item per iteration: up to 96 reduced quantities.
constexpr int kMaxQ1r = 96;

struct Control1r {
  double gamma[kMaxItems], delta[kMaxItems], alpha[kMaxItems], beta[kMaxItems];
  double thr[kMaxItems], scale[kMaxItems], resid[kMaxItems];
  int active[kMaxItems], restart[kMaxItems], status[kMaxItems], iters[kMaxItems];
  int flag[kMaxItems]; // 1 threshold reached, 2 accepted, 3 restart from the true residual
};

// Rows of this warp (warp-steps ws0 + warp, + kPcgWarps, ... < ws1) through the SpMV:
// `gather(ci, vv, acc)` accumulates entry (value vv, item-interleaved column offset ci) into
// acc, `finish(r, acc)` ends row r.  With the value ring the operator values of the next
// chunk of kRingEntries entries are copied to shared memory (cp.async) while the current chunk's
// gathers are in flight; otherwise they are streamed from global memory.
template <int KP, int IV, class Gather, class Finish>
__device__ __forceinline__ void SpmvRows(const PcgArgs &a, const int32_t *colc, size_t cbase, int ws0,
                                         int ws1, int item0, bool ring_on, Gather gather, Finish finish)
{
  using T = double;
  constexpr int LR = KP / IV;
  constexpr int S = 32 / LR;
  constexpr int U = kRingEntries; // the value ring's chunk (also the plain path's)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T *vals = static_cast<const T *>(a.values);
  if constexpr (sizeof(T) * IV == 16) {
    if (ring_on) {
      extern __shared__ __align__(16) unsigned char fg_dynamic_smem[];
      T *ring = reinterpret_cast<T *>(fg_dynamic_smem + a.value_ring_offset) +
                static_cast<size_t>(warp) * 2 * U * 32 * IV;
      const unsigned long long pol = EvictFirstPolicy();
      auto issue = [&](int stage, size_t base, int w0, int len) {
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (w0 + u < len)
            CpAsync16(ring + ((stage * U + u) * 32 + lane) * IV,
                      vals + (base + 32 * static_cast<size_t>(w0 + u)) * a.value_stride + item0, pol);
        CpAsyncCommit();
      };
      auto row_at = [&](int w, int &rr, int &ll, size_t &bb) {
        rr = w * S + lane / LR;
        ll = __ldg(a.row_len + rr);
        bb = static_cast<size_t>(__ldg(a.slice_off + (rr >> 5))) + (rr & 31);
      };
      int ws = ws0 + warp, r = 0, len = 0, w0 = 0, stage = 0, fr = 0, flen = 0;
      size_t base = 0, fbase = 0;
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
        CpAsyncWait<1>();
        int c[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
          c[u] = w0 + u < len ? Column(a, colc, cbase, base + 32 * static_cast<size_t>(w0 + u)) : 0;
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (w0 + u < len) {
            T vv[IV];
            Load<T, IV>(ring + ((stage * U + u) * 32 + lane) * IV, vv);
            gather(static_cast<size_t>(c[u]) * KP + item0, vv, acc);
          }
        if (w0 + U >= len) {
          finish(r, acc);
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
      return;
    }
  }
  for (int ws = ws0 + warp; ws < ws1; ws += kPcgWarps) {
    const int r = ws * S + lane / LR;
    const int len = __ldg(a.row_len + r);
    const size_t base = static_cast<size_t>(__ldg(a.slice_off + (r >> 5))) + (r & 31);
    T acc[IV];
#pragma unroll
    for (int j = 0; j < IV; ++j)
      acc[j] = T(0);
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
      for (int u = 0; u < U; ++u)
        if (w0 + u < len)
          gather(static_cast<size_t>(c[u]) * KP + item0, v[u], acc);
    }
    finish(r, acc);
  }
}

template <int KP, int IV>
__device__ __forceinline__ void Pcg1rBody(const PcgArgs &a, const GridShape gs)
{
  using T = double;
  __shared__ ReduceQ<kMaxQ1r> sm;
  __shared__ Control1r ctl;
  __shared__ Trace tr;
  constexpr int LR = KP / IV;
  constexpr int S = 32 / LR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int item0 = (lane % LR) * IV;
  const int WS = a.n_pad / S;
  const int ws0 = static_cast<int>(static_cast<long long>(WS) * gs.rank / gs.size);
  const int ws1 = static_cast<int>(static_cast<long long>(WS) * (gs.rank + 1) / gs.size);
  unsigned epoch = 0;
  int buf = 0;
  const T *B = static_cast<const T *>(a.b);
  const T *DG = static_cast<const T *>(a.diag);
  const T *IDG = static_cast<const T *>(a.invd);
  T *X = static_cast<T *>(a.x);
  T *P = static_cast<T *>(a.p0);
  // Double-buffered u = r / d, m = A u / d and t = s / d: Uc, Mc, Tc hold the current
  // iteration's values, Un, Mn, Tn receive the next; the pairs swap after each iteration.
  T *Uc = static_cast<T *>(a.r), *Un = static_cast<T *>(a.z);
  T *Mc = static_cast<T *>(a.q), *Mn = static_cast<T *>(a.p1);
  T *Tc = static_cast<T *>(a.t0), *Tn = static_cast<T *>(a.t1);

  if (threadIdx.x < KP) {
    const int it = threadIdx.x;
    ctl.active[it] = (it < a.items && ((a.active_mask >> it) & 1u)) ? 1 : 0;
    ctl.status[it] = kInternal;
    ctl.iters[it] = 0;
    ctl.resid[it] = INFINITY;
    ctl.restart[it] = 1;
    ctl.flag[it] = 0;
    ctl.alpha[it] = ctl.beta[it] = 0.0;
    ctl.scale[it] = 1.0;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kPcgTraceSlots; ++s)
      tr.slot[s] = 0;
    tr.mark = GlobalTimer();
  }
  __syncthreads();

  auto on = [&](int j) { return ctl.active[item0 + j] != 0; };
  auto load_d = [&](int r, T (&d)[IV]) {
    LoadOperand<T, IV>(DG, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, d);
  };
  // y / d (the Jacobi step, by the inverse diagonal when the plan keeps one).
  auto divide = [&](int r, const T (&y)[IV], const T (&d)[IV], T (&o)[IV]) {
    if (a.use_inverse) {
      T e[IV];
      LoadOperand<T, IV>(IDG, static_cast<size_t>(r), a.diag_stride, a.diag_item, item0, e);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        o[j] = y[j] * e[j];
    } else {
#pragma unroll
      for (int j = 0; j < IV; ++j)
        o[j] = y[j] / d[j];
    }
  };

  const int32_t *colc = nullptr;
  size_t cbase = 0;
  if (a.col_cache) {
    extern __shared__ __align__(16) unsigned char fg_dynamic_smem[];
    int32_t *cs = reinterpret_cast<int32_t *>(fg_dynamic_smem + a.col_cache_offset);
    if (ws1 > ws0) {
      const int s0 = (ws0 * S) >> 5, s1 = (ws1 * S - 1) >> 5;
      const size_t p0 = static_cast<size_t>(__ldg(a.slice_off + s0));
      const size_t p1 = static_cast<size_t>(__ldg(a.slice_off + s1 + 1));
      const int4 *src = reinterpret_cast<const int4 *>(a.sell_col + p0);
      int4 *dst = reinterpret_cast<int4 *>(cs);
      for (size_t i = threadIdx.x; i < (p1 - p0) / 4; i += kPcgThreads)
        dst[i] = __ldg(src + i);
      cbase = p0;
    }
    colc = cs;
    __syncthreads();
  }

  // True residual of one row: b/s - A x.
  auto true_residual = [&](int r, size_t ri, const double (&sc)[IV], double (&t)[IV]) {
    const int len = __ldg(a.row_len + r);
    const size_t base = static_cast<size_t>(__ldg(a.slice_off + (r >> 5))) + (r & 31);
    const bool nofold[IV] = {};
    const T nobeta[IV] = {};
    T acc[IV], bb[IV];
    RowProduct<T, KP, IV, false>(a, colc, cbase, base, len, item0, X, nullptr, nofold, nobeta, acc);
    Load<T, IV>(B + ri, bb);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      t[j] = bb[j] / sc[j] - acc[j];
  };

#define FG_ROWS_BEGIN                                                                              \
  for (int ws = ws0 + warp; ws < ws1; ws += kPcgWarps) {                                           \
    const int r = ws * S + lane / LR;                                                              \
    const size_t ri = static_cast<size_t>(r) * KP + item0;
#define FG_ROWS_END }

  // Start of a CG sequence from the stored u (Uc): m = A u / d, gamma = sum d u^2,
  // delta = sum (A u) u, then alpha = gamma / delta and beta = 0.  Every active item at the
  // first start; after a true-residual check (after_check) only the items restarting from
  // it (flag 3), while the accepted items (flag 2) scale x back in the same pass.
  auto restart_phase = [&](bool after_check) -> bool {
    double v[3][IV];
    bool mine[IV], settle[IV], any_mine = false;
    double sc[IV];
#pragma unroll
    for (int j = 0; j < IV; ++j) {
      v[0][j] = v[1][j] = v[2][j] = 0.0;
      const int fl = ctl.flag[item0 + j];
      mine[j] = on(j) && (!after_check || fl == 3);
      settle[j] = on(j) && after_check && fl == 2;
      any_mine = any_mine || mine[j] || settle[j];
      sc[j] = ctl.scale[item0 + j];
    }
    if (__any_sync(0xffffffffu, any_mine)) {
      auto gather = [&](size_t ci, const T (&vv)[IV], T (&acc)[IV]) {
        T g[IV];
        Load<T, IV>(Uc + ci, g);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          acc[j] = Fma(vv[j], g[j], acc[j]);
      };
      auto finish = [&](int r, const T (&acc)[IV]) {
        const size_t ri = static_cast<size_t>(r) * KP + item0;
        T uo[IV], d[IV], mo[IV], mn[IV];
        Load<T, IV>(Uc + ri, uo);
        Load<T, IV>(Mc + ri, mo);
        load_d(r, d);
        divide(r, acc, d, mn);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          if (mine[j]) {
            v[0][j] += d[j] * uo[j] * uo[j];
            v[1][j] += acc[j] * uo[j];
          } else {
            mn[j] = mo[j];
          }
        Store<T, IV>(Mc + ri, mn);
        if (after_check) {
          T xv[IV];
          Load<T, IV>(X + ri, xv);
#pragma unroll
          for (int j = 0; j < IV; ++j)
            if (settle[j]) {
              xv[j] = xv[j] * sc[j];
              if (!isfinite(xv[j]))
                v[2][j] += 1.0;
            }
          Store<T, IV>(X + ri, xv);
        }
      };
      SpmvRows<KP, IV>(a, colc, cbase, ws0, ws1, item0, a.value_ring != 0, gather, finish);
    }
    if (!GridReduce<KP, IV, 3, false>(a, gs, v, sm, epoch, buf, tr, 2))
      return false;
    if (threadIdx.x < KP) {
      const int it = threadIdx.x;
      const int fl = ctl.flag[it];
      if (ctl.active[it] && after_check && fl == 2) {
        if (sm.result[2 * KP + it] != 0.0) {
          ctl.status[it] = kNonfinite;
        } else {
          ctl.resid[it] *= ctl.scale[it];
          ctl.status[it] = isfinite(ctl.resid[it]) ? kOk : kNonfinite;
        }
        ctl.active[it] = 0;
      } else if (ctl.active[it] && (!after_check || fl == 3)) {
        const double g = sm.result[it], d = sm.result[KP + it];
        if (!isfinite(g) || !isfinite(d)) {
          ctl.status[it] = kNonfinite;
          ctl.active[it] = 0;
        } else if (!(g > 0.0) || !(d > 0.0)) {
          ctl.status[it] = kBreakdown;
          ctl.active[it] = 0;
        } else {
          ctl.gamma[it] = g;
          ctl.delta[it] = d;
          ctl.alpha[it] = g / d;
          ctl.beta[it] = 0.0;
          ctl.restart[it] = 1;
        }
      }
      ctl.flag[it] = 0;
    }
    __syncthreads();
    return true;
  };

  // Validity (first invalid row decides the status) and RHS max-scaling; x = 0.
  {
    double v[2][IV];
#pragma unroll
    for (int j = 0; j < IV; ++j)
      v[0][j] = v[1][j] = 0.0;
    FG_ROWS_BEGIN
    T dd[IV], bb[IV];
    Load<T, IV>(B + ri, bb);
    load_d(r, dd);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      if (on(j) && r < a.n) {
        const bool nonfinite = !isfinite(bb[j]) || !isfinite(dd[j]);
        if (nonfinite || !(dd[j] > 0.0))
          v[0][j] = fmax(v[0][j], 2.0 * static_cast<double>(a.n - r) + (nonfinite ? 1.0 : 0.0));
        v[1][j] = fmax(v[1][j], fabs(bb[j]));
      }
    const T zero[IV] = {};
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

  // r = b / s, u = r / d, (r, r).
  {
    double v[1][IV], s[IV];
#pragma unroll
    for (int j = 0; j < IV; ++j) {
      v[0][j] = 0.0;
      s[j] = ctl.scale[item0 + j] != 0.0 ? ctl.scale[item0 + j] : 1.0;
    }
    FG_ROWS_BEGIN
    T bb[IV], rr[IV], d[IV], u[IV];
    Load<T, IV>(B + ri, bb);
    load_d(r, d);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      rr[j] = bb[j] / s[j];
    divide(r, rr, d, u);
    Store<T, IV>(Uc + ri, u);
#pragma unroll
    for (int j = 0; j < IV; ++j)
      if (on(j))
        v[0][j] += rr[j] * rr[j];
    FG_ROWS_END
    if (!GridReduce<KP, IV, 1, false>(a, gs, v, sm, epoch, buf, tr, 3))
      return;
    if (threadIdx.x < KP) {
      const int it = threadIdx.x;
      if (ctl.active[it]) {
        const double rr = sm.result[it];
        if (!isfinite(rr)) {
          ctl.status[it] = kNonfinite;
          ctl.active[it] = 0;
        } else {
          ctl.resid[it] = sqrt(rr);
          ctl.thr[it] = (a.item_tolerance ? a.item_tolerance[it] : a.tolerance) * sqrt(rr);
        }
      }
      ctl.flag[it] = 0;
    }
    __syncthreads();
  }
  // m = A u / d, gamma, delta: the first step's scalars.
  if (!restart_phase(false))
    return;

  for (int iteration = 0; iteration < a.max_iterations; ++iteration) {
    bool any = false;
#pragma unroll
    for (int it = 0; it < KP; ++it)
      any = any || ctl.active[it];
    if (!any)
      break;

    // The iteration: p, t, x, u updates of this CTA's rows, w = A u_{i+1} (u_{i+1} of each
    // gathered column formed from u_i, m_i, t_{i-1}), m = w / d, and the three sums.
    {
      double v[3][IV];
      bool fold[IV], any_mine = false;
      T al[IV], be[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = v[1][j] = v[2][j] = 0.0;
        fold[j] = !ctl.restart[item0 + j];
        al[j] = ctl.alpha[item0 + j];
        be[j] = ctl.beta[item0 + j];
        any_mine = any_mine || on(j);
      }
      if (__any_sync(0xffffffffu, any_mine)) {
        auto gather = [&](size_t ci, const T (&vv)[IV], T (&acc)[IV]) {
          T uu[IV], mm[IV], tt[IV];
          Load<T, IV>(Uc + ci, uu);
          Load<T, IV>(Mc + ci, mm);
          Load<T, IV>(Tc + ci, tt); // unused (and possibly unset) where fold is false
#pragma unroll
          for (int j = 0; j < IV; ++j) {
            const T ts = fold[j] ? Fma(be[j], tt[j], mm[j]) : mm[j];
            acc[j] = Fma(vv[j], Fma(-al[j], ts, uu[j]), acc[j]);
          }
        };
        auto finish = [&](int r, const T (&acc)[IV]) {
          const size_t ri = static_cast<size_t>(r) * KP + item0;
          T uo[IV], mo[IV], to[IV], po[IV], xo[IV], d[IV], mn[IV];
          Load<T, IV>(Uc + ri, uo);
          Load<T, IV>(Mc + ri, mo);
          Load<T, IV>(Tc + ri, to);
          Load<T, IV>(P + ri, po);
          Load<T, IV>(X + ri, xo);
          load_d(r, d);
          divide(r, acc, d, mn);
          T pn[IV], tn[IV], un[IV];
#pragma unroll
          for (int j = 0; j < IV; ++j) {
            pn[j] = fold[j] ? Fma(be[j], po[j], uo[j]) : uo[j];
            tn[j] = fold[j] ? Fma(be[j], to[j], mo[j]) : mo[j];
            un[j] = Fma(-al[j], tn[j], uo[j]);
            if (on(j)) {
              xo[j] = Fma(al[j], pn[j], xo[j]);
              const double du = d[j] * un[j];
              v[0][j] += du * un[j];
              v[1][j] += acc[j] * un[j];
              v[2][j] += du * du;
            }
          }
          Store<T, IV>(P + ri, pn);
          Store<T, IV>(X + ri, xo);
          Store<T, IV>(Tn + ri, tn);
          Store<T, IV>(Un + ri, un);
          Store<T, IV>(Mn + ri, mn);
        };
        SpmvRows<KP, IV>(a, colc, cbase, ws0, ws1, item0, a.value_ring != 0, gather, finish);
      }
      if (!GridReduce<KP, IV, 3, false>(a, gs, v, sm, epoch, buf, tr, 0))
        return;
      T *sw = Uc;
      Uc = Un;
      Un = sw;
      sw = Mc;
      Mc = Mn;
      Mn = sw;
      sw = Tc;
      Tc = Tn;
      Tn = sw;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        ctl.flag[it] = 0;
        if (ctl.active[it]) {
          ctl.iters[it] = iteration + 1;
          const double g = sm.result[it], dl = sm.result[KP + it], rr = sm.result[2 * KP + it];
          if (!isfinite(g) || !isfinite(dl) || !isfinite(rr)) {
            ctl.status[it] = kNonfinite;
            ctl.active[it] = 0;
          } else {
            ctl.resid[it] = sqrt(rr);
            if (ctl.resid[it] <= ctl.thr[it]) {
              ctl.flag[it] = a.skip_verification ? 2 : 1;
            } else {
              const double be = g / ctl.gamma[it];
              const double den = dl - be * g / ctl.alpha[it];
              if (!(g > 0.0) || !(den > 0.0) || !isfinite(be) || !isfinite(den)) {
                ctl.status[it] = kBreakdown;
                ctl.active[it] = 0;
              } else {
                ctl.beta[it] = be;
                ctl.alpha[it] = g / den;
                ctl.gamma[it] = g;
                ctl.delta[it] = dl;
                ctl.restart[it] = 0;
              }
            }
          }
        }
      }
      __syncthreads();
    }

    bool verify = false, settle = false;
#pragma unroll
    for (int it = 0; it < KP; ++it) {
      verify = verify || (ctl.active[it] && ctl.flag[it] == 1);
      settle = settle || (ctl.active[it] && ctl.flag[it] == 2);
    }
    if (verify) {
      // True residual of the items at the threshold; it becomes their u (in the buffer
      // the next iteration reads) in case they restart.
      double v[1][IV], s[IV];
      bool mine[IV], any_mine = false;
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        mine[j] = on(j) && ctl.flag[item0 + j] == 1;
        any_mine = any_mine || mine[j];
        s[j] = ctl.scale[item0 + j];
      }
      if (any_mine) {
        FG_ROWS_BEGIN
        double t[IV];
        true_residual(r, ri, s, t);
        T uo[IV], d[IV], tr_[IV], un[IV];
        Load<T, IV>(Uc + ri, uo);
        load_d(r, d);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          tr_[j] = t[j];
        divide(r, tr_, d, un);
#pragma unroll
        for (int j = 0; j < IV; ++j)
          if (mine[j])
            v[0][j] += t[j] * t[j];
          else
            un[j] = uo[j];
        Store<T, IV>(Uc + ri, un);
        FG_ROWS_END
      }
      if (!GridReduce<KP, IV, 1, false>(a, gs, v, sm, epoch, buf, tr, 2))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        if (ctl.active[it] && ctl.flag[it] == 1) {
          const double trr = sm.result[it];
          if (!isfinite(trr)) {
            ctl.status[it] = kNonfinite;
            ctl.active[it] = 0;
            ctl.flag[it] = 0;
          } else {
            ctl.resid[it] = sqrt(trr);
            ctl.flag[it] = ctl.resid[it] <= ctl.thr[it] ? 2 : 3;
          }
        }
      }
      __syncthreads();
    }
    if (verify || settle) {
      // Accepted items scale x back; restarted items take m = A u / d of their true
      // residual and the scalars of a fresh start.
      if (!restart_phase(true))
        return;
    }
  }

  // Iteration budget exhausted: report the true residual and scale the iterate back.
  bool any = false;
#pragma unroll
  for (int it = 0; it < KP; ++it)
    any = any || ctl.active[it];
  if (any) {
    {
      double v[1][IV], s[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        s[j] = ctl.scale[item0 + j];
      }
      FG_ROWS_BEGIN
      double t[IV];
      true_residual(r, ri, s, t);
      (void)ri;
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (on(j))
          v[0][j] += t[j] * t[j];
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
            ctl.gamma[it] = trr;
          }
        }
      }
      __syncthreads();
    }
    {
      double v[1][IV], s[IV];
#pragma unroll
      for (int j = 0; j < IV; ++j) {
        v[0][j] = 0.0;
        s[j] = ctl.scale[item0 + j];
      }
      FG_ROWS_BEGIN
      T xv[IV];
      Load<T, IV>(X + ri, xv);
#pragma unroll
      for (int j = 0; j < IV; ++j)
        if (on(j)) {
          xv[j] = xv[j] * s[j];
          if (!isfinite(xv[j]))
            v[0][j] += 1.0;
        }
      Store<T, IV>(X + ri, xv);
      FG_ROWS_END
      if (!GridReduce<KP, IV, 1, false>(a, gs, v, sm, epoch, buf, tr, 3))
        return;
      if (threadIdx.x < KP) {
        const int it = threadIdx.x;
        if (ctl.active[it]) {
          if (sm.result[it] != 0.0) {
            ctl.status[it] = kNonfinite;
          } else {
            ctl.resid[it] = sqrt(ctl.gamma[it]) * ctl.scale[it];
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

template <int KP, int IV>
__global__ void __launch_bounds__(kPcgThreads, 2) Pcg1rKernel(PcgArgs a)
{
  Pcg1rBody<KP, IV>(a, GridShape{static_cast<int>(gridDim.x), static_cast<int>(blockIdx.x)});
}

} // namespace
} // namespace fg
