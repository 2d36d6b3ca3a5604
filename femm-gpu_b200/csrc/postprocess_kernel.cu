// postprocess_kernel.cu -- device form of the frozen postprocess: per-CTA partial sums of the
// weighted-stress force and torque for every item, and the gather of the element B and
// nodal A values that the air-gap probes' smoothing reads, in one launch.
#include "postprocess.h"

namespace fg
{
namespace
{

constexpr int kThreads = 256;
constexpr int kMaxCtas = 148 * 4;
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

__global__ void __launch_bounds__(kThreads) PostprocessKernel(PostprocessDevice p)
{
  __shared__ double scratch[kThreads / 32];
  if (static_cast<int>(blockIdx.x) < p.ctas) {
    // Contiguous element range of this CTA; every item in turn (the geometry stays in L1/L2).
    const int64_t chunk = (static_cast<int64_t>(p.E) + p.ctas - 1) / p.ctas;
    const int64_t first = chunk * blockIdx.x;
    const int64_t last = min(first + chunk, static_cast<int64_t>(p.E));
    for (int item = 0; item < p.items; ++item) {
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
    }
    return;
  }
  const int64_t per_item = 2 * static_cast<int64_t>(p.gather_e) + p.gather_n;
  const int64_t t = static_cast<int64_t>(blockIdx.x - p.ctas) * kThreads + threadIdx.x;
  if (t >= per_item * p.items)
    return;
  const int64_t item = t / per_item, j = t - item * per_item;
  double v;
  if (j < p.gather_e)
    v = p.b1[item * p.E + p.gather_elements[j]];
  else if (j < 2 * p.gather_e)
    v = p.b2[item * p.E + p.gather_elements[j - p.gather_e]];
  else
    v = p.a[item * p.N + p.gather_nodes[j - 2 * p.gather_e]];
  p.gathered[t] = v;
}

} // namespace

int PostprocessCtas(int32_t E)
{
  const int64_t want = (static_cast<int64_t>(E) + 4 * kThreads - 1) / (4 * kThreads);
  return static_cast<int>(want < 1 ? 1 : (want > kMaxCtas ? kMaxCtas : want));
}

cudaError_t LaunchPostprocess(const PostprocessDevice &p, cudaStream_t stream)
{
  const int64_t gathers = (2 * static_cast<int64_t>(p.gather_e) + p.gather_n) * p.items;
  const int64_t blocks = p.ctas + (gathers + kThreads - 1) / kThreads;
  PostprocessKernel<<<static_cast<unsigned>(blocks), kThreads, 0, stream>>>(p);
  return cudaGetLastError();
}

} // namespace fg
