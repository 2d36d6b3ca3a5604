// postprocess_kernel.cu -- device form of the frozen postprocess: per-(CTA, item) partial
// sums of the weighted-stress force and torque, and the smoothed radial air-gap B of every
// (item, probe) from the probe corners' recipes, in one launch.
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
constexpr int kMaxCtas = 148 * 2;
constexpr double kTwoMu0 = 2.0 * 4.0e-7 * 3.141592653589793238462643383279502884;

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

// Nodal B of one probe corner, in the host smoothing's operation order.
__device__ void Corner(const PostprocessDevice &p, const CornerStencil &c, const double *a,
                       const double *b1, const double *b2, double *nbx, double *nby)
{
  double x = 0.0, y = 0.0;
  if (c.kind == 0) {
    for (int t = c.first; t < c.first + c.count; ++t) {
      const int e = p.term_elem[t];
      x = __dadd_rn(x, __dmul_rn(p.term_w[t], b1[e]));
      y = __dadd_rn(y, __dmul_rn(p.term_w[t], b2[e]));
    }
    x = __ddiv_rn(x, c.wsum);
    y = __ddiv_rn(y, c.wsum);
  } else if (c.kind == 1) {
    for (int t = c.first; t < c.first + c.count; ++t) {
      const int e = p.term_elem[t];
      const double tx = p.term_tx[t], ty = p.term_ty[t], w = p.term_w[t];
      const double bt = __dadd_rn(__dmul_rn(b1[e], tx), __dmul_rn(b2[e], ty));
      const double bn = __ddiv_rn(__dsub_rn(a[p.term_node[t]], a[c.node]), p.term_len[t]);
      x = __dadd_rn(x, __dmul_rn(w, __dadd_rn(__dmul_rn(tx, bt), __dmul_rn(ty, bn))));
      y = __dadd_rn(y, __dmul_rn(w, __dsub_rn(__dmul_rn(ty, bt), __dmul_rn(tx, bn))));
    }
    x = __ddiv_rn(x, c.wsum);
    y = __ddiv_rn(y, c.wsum);
  } else if (c.kind == 2) {
    x = b1[c.element];
    y = b2[c.element];
  } else {
    double largest = 0.0;
    for (int t = c.first; t < c.first + c.count; ++t) {
      const int e = p.term_elem[t];
      largest = fmax(largest, hypot(b1[e], b2[e]));
    }
    const double own = hypot(b1[c.element], b2[c.element]);
    x = own > 0.0 ? __ddiv_rn(__dmul_rn(largest, b1[c.element]), own) : 0.0;
    y = own > 0.0 ? __ddiv_rn(__dmul_rn(largest, b2[c.element]), own) : 0.0;
  }
  *nbx = x;
  *nby = y;
}

__global__ void __launch_bounds__(kThreads) PostprocessKernel(PostprocessDevice p)
{
  __shared__ double scratch[kThreads / 32];
  if (static_cast<int>(blockIdx.x) < p.ctas) {
    // Contiguous element range of this CTA for item blockIdx.y.
    const int item = blockIdx.y;
    const int64_t chunk = (static_cast<int64_t>(p.E) + p.ctas - 1) / p.ctas;
    const int64_t first = chunk * blockIdx.x;
    const int64_t last = min(first + chunk, static_cast<int64_t>(p.E));
    const double *b1 = p.b1 + static_cast<int64_t>(item) * p.E;
    const double *b2 = p.b2 + static_cast<int64_t>(item) * p.E;
    double fx = 0.0, fy = 0.0, tq = 0.0;
    for (int64_t e = first + threadIdx.x; e < last; e += kThreads) {
      const double hx = p.hx[e], hy = p.hy[e];
      const double bx = __ldcs(b1 + e), by = __ldcs(b2 + e);
      const double fxd = ((bx * bx - by * by) * hx + 2.0 * bx * by * hy) / kTwoMu0;
      const double fyd = (2.0 * bx * by * hx + (by * by - bx * bx) * hy) / kTwoMu0;
      const double w = p.weight[e];
      fx += w * fxd;
      fy += w * fyd;
      tq += w * (p.cx[e] * fyd - p.cy[e] * fxd);
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
    return;
  }
  // Probe blocks (blockIdx.y == 0 only): one thread per (item, probe).
  if (blockIdx.y != 0)
    return;
  const int64_t t = static_cast<int64_t>(blockIdx.x - p.ctas) * kThreads + threadIdx.x;
  if (t >= static_cast<int64_t>(p.probes) * p.items)
    return;
  const int item = static_cast<int>(t / p.probes), k = static_cast<int>(t % p.probes);
  const double *a = p.a + static_cast<int64_t>(item) * p.N;
  const double *b1 = p.b1 + static_cast<int64_t>(item) * p.E;
  const double *b2 = p.b2 + static_cast<int64_t>(item) * p.E;
  const double *pr = p.probe + 5 * k;
  double bx = 0.0, by = 0.0;
  for (int l = 0; l < 3; ++l) {
    double nbx, nby;
    Corner(p, p.corners[3 * k + l], a, b1, b2, &nbx, &nby);
    bx = __dadd_rn(bx, __dmul_rn(pr[l], nbx));
    by = __dadd_rn(by, __dmul_rn(pr[l], nby));
  }
  p.radial[t] = __dadd_rn(__dmul_rn(bx, pr[3]), __dmul_rn(by, pr[4]));
}

} // namespace

int PostprocessCtas(int32_t E)
{
  const int64_t want = (static_cast<int64_t>(E) + 4 * kThreads - 1) / (4 * kThreads);
  return static_cast<int>(want < 1 ? 1 : (want > kMaxCtas ? kMaxCtas : want));
}

cudaError_t LaunchPostprocess(const PostprocessDevice &p, cudaStream_t stream)
{
  const int64_t samples = static_cast<int64_t>(p.probes) * p.items;
  const int64_t blocks = p.ctas + (samples + kThreads - 1) / kThreads;
  if (p.items < 1 || p.items > 65535)
    return cudaErrorInvalidValue;
  PostprocessKernel<<<dim3(static_cast<unsigned>(blocks), static_cast<unsigned>(p.items)), kThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

} // namespace fg
