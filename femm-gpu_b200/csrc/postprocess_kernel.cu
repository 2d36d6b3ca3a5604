// postprocess_kernel.cu -- device form of the frozen postprocess: per-(CTA, item) partial
// sums of the weighted-stress force and torque (ForceKernel), and the smoothed radial
// air-gap B of every (item, probe) from the probe corners' recipes (ProbeKernel).
//
// The probe arithmetic uses explicitly rounded operations (no fused multiply-add) in the
// host smoothing's order, so the samples equal the host form's bit for bit; the sharp-corner
// fallback's |B| uses the device hypot.
#include "postprocess.h"

namespace fg
{
namespace
{

constexpr int kThreads = 256;
constexpr int kSms = 148;
constexpr int kMaxCtas = 3 * kSms;
constexpr int kPerThread = 8; // elements per thread of the force reduction, at least
constexpr double kInvTwoMu0 = 1.0 / (2.0 * 4.0e-7 * 3.141592653589793238462643383279502884);

// Sum over the block in a fixed order: warp trees, then warp 0 over the warp totals.
__device__ double BlockSum(double v, double *scratch)
{
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0)
    scratch[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < kThreads / 32 ? scratch[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1)
      t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t; // valid in thread 0
}

// Nodal B of one probe corner, in the host smoothing's operation order.  Term indices are
// loaded ahead of the values they address (two dependent hops per batch of terms, not two per
// term); the accumulation order stays the host's.
__device__ void Corner(const PostprocessDevice &p, const CornerStencil &c, const double *a,
                       const double *b1, const double *b2, double *nbx, double *nby)
{
  constexpr int kBatch = 8;
  double x = 0.0, y = 0.0;
  if (c.kind == 0 || c.kind == 3) {
    double largest = 0.0;
    for (int t0 = c.first; t0 < c.first + c.count; t0 += kBatch) {
      int e[kBatch];
      double v1[kBatch], v2[kBatch];
#pragma unroll
      for (int j = 0; j < kBatch; ++j)
        e[j] = t0 + j < c.first + c.count ? p.term_elem[t0 + j] : -1;
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        v1[j] = e[j] >= 0 ? b1[e[j]] : 0.0;
        v2[j] = e[j] >= 0 ? b2[e[j]] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        if (e[j] < 0)
          break;
        if (c.kind == 0) {
          const double w = p.term_w[t0 + j];
          x = __dadd_rn(x, __dmul_rn(w, v1[j]));
          y = __dadd_rn(y, __dmul_rn(w, v2[j]));
        } else {
          largest = fmax(largest, hypot(v1[j], v2[j]));
        }
      }
    }
    if (c.kind == 0) {
      x = __ddiv_rn(x, c.wsum);
      y = __ddiv_rn(y, c.wsum);
    } else {
      const double o1 = b1[c.element], o2 = b2[c.element];
      const double own = hypot(o1, o2);
      x = own > 0.0 ? __ddiv_rn(__dmul_rn(largest, o1), own) : 0.0;
      y = own > 0.0 ? __ddiv_rn(__dmul_rn(largest, o2), own) : 0.0;
    }
  } else if (c.kind == 1) {
    const double an = a[c.node];
    for (int t = c.first; t < c.first + c.count; ++t) {
      const int e = p.term_elem[t];
      const double tx = p.term_tx[t], ty = p.term_ty[t], w = p.term_w[t];
      const double bt = __dadd_rn(__dmul_rn(b1[e], tx), __dmul_rn(b2[e], ty));
      const double bn = __ddiv_rn(__dsub_rn(a[p.term_node[t]], an), p.term_len[t]);
      x = __dadd_rn(x, __dmul_rn(w, __dadd_rn(__dmul_rn(tx, bt), __dmul_rn(ty, bn))));
      y = __dadd_rn(y, __dmul_rn(w, __dsub_rn(__dmul_rn(ty, bt), __dmul_rn(tx, bn))));
    }
    x = __ddiv_rn(x, c.wsum);
    y = __ddiv_rn(y, c.wsum);
  } else {
    x = b1[c.element];
    y = b2[c.element];
  }
  *nbx = x;
  *nby = y;
}

// Force / torque partial sums: CTA (blockIdx.x, item blockIdx.y) over a contiguous element
// range.  Each thread takes its elements three at a time and issues all 21 loads of a group
// before using any, so that a warp keeps enough bytes in flight to cover the HBM latency.
__global__ void __launch_bounds__(kThreads, 3) ForceKernel(PostprocessDevice p)
{
  __shared__ double scratch[kThreads / 32];
  constexpr int G = 3;
  const int item = blockIdx.y;
  const int64_t chunk = (static_cast<int64_t>(p.E) + p.ctas - 1) / p.ctas;
  const int64_t first = chunk * blockIdx.x;
  const int64_t last = min(first + chunk, static_cast<int64_t>(p.E));
  const double *b1 = p.b1 + static_cast<int64_t>(item) * p.E;
  const double *b2 = p.b2 + static_cast<int64_t>(item) * p.E;
  double fx = 0.0, fy = 0.0, tq = 0.0;
  for (int64_t base = first + threadIdx.x; base < last; base += G * kThreads) {
    double hx[G], hy[G], w[G], cx[G], cy[G], bx[G], by[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const int64_t e = base + g * kThreads;
      const bool in = e < last;
      hx[g] = in ? p.hx[e] : 0.0;
      hy[g] = in ? p.hy[e] : 0.0;
      w[g] = in ? p.weight[e] : 0.0;
      cx[g] = in ? p.cx[e] : 0.0;
      cy[g] = in ? p.cy[e] : 0.0;
      bx[g] = in ? __ldcs(b1 + e) : 0.0;
      by[g] = in ? __ldcs(b2 + e) : 0.0;
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const double fxd = ((bx[g] * bx[g] - by[g] * by[g]) * hx[g] + 2.0 * bx[g] * by[g] * hy[g]) * kInvTwoMu0;
      const double fyd = (2.0 * bx[g] * by[g] * hx[g] + (by[g] * by[g] - bx[g] * bx[g]) * hy[g]) * kInvTwoMu0;
      fx += w[g] * fxd;
      fy += w[g] * fyd;
      tq += w[g] * (cx[g] * fyd - cy[g] * fxd);
    }
  }
  fx = BlockSum(fx, scratch);
  fy = BlockSum(fy, scratch);
  tq = BlockSum(tq, scratch);
  if (threadIdx.x == 0) {
    double *q = p.partials + (static_cast<int64_t>(blockIdx.x) * p.items + item) * 3;
    q[0] = fx;
    q[1] = fy;
    q[2] = tq;
  }
}

// Air-gap samples: four lanes per (item, probe), lanes 0-2 one corner each; lane 0
// combines the corners in the host's order.
__global__ void __launch_bounds__(kThreads) ProbeKernel(PostprocessDevice p)
{
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  const int64_t sample = t >> 2;
  const int l = static_cast<int>(t & 3);
  const bool live = sample < static_cast<int64_t>(p.probes) * p.items;
  double nbx = 0.0, nby = 0.0;
  int item = 0, k = 0;
  if (live) {
    item = static_cast<int>(sample / p.probes);
    k = static_cast<int>(sample % p.probes);
    if (l < 3)
      Corner(p, p.corners[3 * k + l], p.a + static_cast<int64_t>(item) * p.N,
             p.b1 + static_cast<int64_t>(item) * p.E, p.b2 + static_cast<int64_t>(item) * p.E, &nbx, &nby);
  }
  double cx[3], cy[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    cx[j] = __shfl_sync(0xffffffffu, nbx, (threadIdx.x & ~3) + j);
    cy[j] = __shfl_sync(0xffffffffu, nby, (threadIdx.x & ~3) + j);
  }
  if (!live || l != 0)
    return;
  const double *pr = p.probe + 5 * k;
  double bx = 0.0, by = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    bx = __dadd_rn(bx, __dmul_rn(pr[j], cx[j]));
    by = __dadd_rn(by, __dmul_rn(pr[j], cy[j]));
  }
  p.radial[sample] = __dadd_rn(__dmul_rn(bx, pr[3]), __dmul_rn(by, pr[4]));
}

} // namespace

int PostprocessCtas(int32_t E, int32_t items)
{
  // One wave: at most three resident CTAs per SM over all (range, item) CTAs, and at least
  // kPerThread elements per thread.
  const int64_t by_size = (static_cast<int64_t>(E) + kPerThread * kThreads - 1) / (kPerThread * kThreads);
  const int64_t by_wave = (3 * kSms) / (items > 0 ? items : 1);
  int64_t want = by_size > by_wave ? by_wave : by_size;
  return static_cast<int>(want < 1 ? 1 : (want > kMaxCtas ? kMaxCtas : want));
}

cudaError_t LaunchPostprocess(const PostprocessDevice &p, cudaStream_t stream)
{
  if (p.items < 1 || p.items > 65535)
    return cudaErrorInvalidValue;
  ForceKernel<<<dim3(static_cast<unsigned>(p.ctas), static_cast<unsigned>(p.items)), kThreads, 0, stream>>>(p);
  const int64_t lanes = 4 * static_cast<int64_t>(p.probes) * p.items;
  if (lanes > 0)
    ProbeKernel<<<static_cast<unsigned>((lanes + kThreads - 1) / kThreads), kThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

} // namespace fg
