// precond.cu -- block-Jacobi preconditioner set-up.
//
// Semantics of the reference's BuildBlockInverse (gpu_solver/src/solvers/
// block_jacobi_preconditioner.cu:72-167): for each contiguous block of BS rows of each
// item's operator, the principal block is scaled by D^-1/2, factored by Cholesky and
// inverted column by column; a block with a non-positive or subnormal reciprocal
// diagonal, an asymmetric or non-finite entry, a failed pivot or a non-finite inverse is
// stored as NaN in its first entry (the PCG then uses the diagonal for its rows) and
// counted.  The reference factors with one thread per block; here lane c of a BS-lane
// group finishes column c of the factor after lane c has formed the pivot, which keeps
// each entry's operation order, and lane c then solves for column c of the inverse.
//
// Layout: item-interleaved like every batch array, entry (i, j) of block b at
// [(b * BS + j) * BS + i][KP] -- the PCG's lanes for consecutive rows and items read
// consecutive addresses for a fixed j.
#include "kernels.cuh"

#include <cfloat>
#include <cmath>

namespace fg
{
namespace
{

constexpr int kThreads = 64;

struct BlockArgs {
  int n, n_pad, groups, kp;
  const int32_t *slice_off, *row_len, *sell_col;
  const double *values;
  int value_item;
  const double *diag;
  int diag_item;
  double *out64;
  float *out32;
  int32_t *fallbacks;
};

template <int BS> __global__ void __launch_bounds__(kThreads) BlockInverseKernel(BlockArgs a)
{
  constexpr int P = kThreads / BS; // blocks factored per CTA
  __shared__ double F[P][BS][BS + 1];
  __shared__ double X[P][BS][BS + 1]; // X[g][c] = column c of the inverse
  __shared__ double sc[P][BS];
  __shared__ int bad[P];
  const int g = threadIdx.x / BS, l = threadIdx.x % BS;
  const long long pair = static_cast<long long>(blockIdx.x) * P + g;
  const int blocks = a.n_pad / BS;
  const bool valid = pair < static_cast<long long>(blocks) * a.groups;
  const int blk = valid ? static_cast<int>(pair / a.groups) : 0;
  const int item = valid ? static_cast<int>(pair % a.groups) : 0;
  const int first = blk * BS;
  const int width = valid ? max(0, min(BS, a.n - first)) : 0;
  const int vs = a.value_item ? a.kp : 1, vi = a.value_item ? item : 0;
  const int ds = a.diag_item ? a.kp : 1, di = a.diag_item ? item : 0;

  double d = 1.0;
  if (l < width)
    d = a.diag[static_cast<size_t>(first + l) * ds + di];
  sc[g][l] = l < width ? sqrt(d) : 1.0;
  for (int c = 0; c < BS; ++c)
    F[g][l][c] = 0.0;
  if (l == 0)
    bad[g] = 0;
  __syncthreads();
  if (l < width) {
    const int r = first + l;
    const int len = a.row_len[r];
    const size_t base = static_cast<size_t>(a.slice_off[r >> 5]) + (r & 31);
    for (int w = 0; w < len; ++w) {
      const size_t pos = base + 32 * static_cast<size_t>(w);
      const int c = a.sell_col[pos] - first;
      if (c >= 0 && c < width)
        F[g][l][c] += a.values[pos * vs + vi] / sc[g][l] / sc[g][c];
    }
  }
  __syncthreads();
  if (l < width) {
    const double reciprocal = 1.0 / d;
    bool b = !isfinite(reciprocal) || reciprocal < DBL_MIN;
    for (int c = 0; c <= l; ++c) {
      const double x = F[g][l][c], y = F[g][c][l];
      if (!isfinite(x) || !isfinite(y) || fabs(x - y) > 1e-12 * fmax(1.0, fmax(fabs(x), fabs(y))))
        b = true;
    }
    if (b)
      atomicOr(&bad[g], 1);
  }
  __syncthreads();
  for (int c = 0; c < BS; ++c) {
    if (c < width && !bad[g] && l == c) {
      double pivot = F[g][c][c];
      for (int k = 0; k < c; ++k)
        pivot -= F[g][c][k] * F[g][c][k];
      if (!(pivot > 0.0) || !isfinite(pivot))
        bad[g] = 1;
      else
        F[g][c][c] = sqrt(pivot);
    }
    __syncthreads();
    if (c < width && !bad[g] && l > c && l < width) {
      double v = F[g][l][c];
      for (int k = 0; k < c; ++k)
        v -= F[g][l][k] * F[g][c][k];
      F[g][l][c] = v / F[g][c][c];
    }
    __syncthreads();
  }
  if (l < width && !bad[g]) {
    double *x = X[g][l];
    for (int row = 0; row < width; ++row) {
      double v = row == l ? 1.0 : 0.0;
      for (int k = 0; k < row; ++k)
        v -= F[g][row][k] * x[k];
      x[row] = v / F[g][row][row];
    }
    for (int row = width - 1; row >= 0; --row) {
      double v = x[row];
      for (int k = row + 1; k < width; ++k)
        v -= F[g][k][row] * x[k];
      x[row] = v / F[g][row][row];
    }
    bool b = false;
    for (int row = 0; row < width; ++row) {
      x[row] = x[row] / sc[g][row] / sc[g][l];
      b = b || !isfinite(x[row]);
    }
    if (b)
      atomicOr(&bad[g], 1);
  }
  __syncthreads();
  if (!valid)
    return;
  const bool b = bad[g] != 0;
  if (b && l == 0 && a.fallbacks)
    atomicAdd(a.fallbacks, 1);
  for (int row = 0; row < BS; ++row) {
    const double v = b ? (row == 0 && l == 0 ? NAN : 0.0)
                       : (row < width && l < width ? X[g][l][row] : 0.0);
    const size_t o = (static_cast<size_t>(first + l) * BS + row) * vs + vi;
    if (a.out64)
      a.out64[o] = v;
    else
      a.out32[o] = static_cast<float>(v);
  }
}

} // namespace

cudaError_t LaunchBlockInverse(const DevicePlan &p, int kp, int items, int bs, const double *values,
                               int value_item, const double *diag, int diag_item, double *out64,
                               float *out32, int32_t *fallbacks, cudaStream_t stream)
{
  BlockArgs a{};
  a.n = p.n;
  a.n_pad = p.n_pad;
  a.groups = value_item ? items : 1;
  a.kp = kp;
  a.slice_off = p.slice_off;
  a.row_len = p.row_len;
  a.sell_col = p.sell_col;
  a.values = values;
  a.value_item = value_item;
  a.diag = diag;
  a.diag_item = diag_item;
  a.out64 = out64;
  a.out32 = out32;
  a.fallbacks = fallbacks;
  if ((bs != 8 && bs != 32) || (!out64 && !out32) || items < 1 || p.n_pad % bs != 0)
    return cudaErrorInvalidValue;
  const long long pairs = static_cast<long long>(p.n_pad / bs) * a.groups;
  const long long per = kThreads / bs;
  const unsigned grid = static_cast<unsigned>((pairs + per - 1) / per);
  if (bs == 8)
    BlockInverseKernel<8><<<grid, kThreads, 0, stream>>>(a);
  else
    BlockInverseKernel<32><<<grid, kThreads, 0, stream>>>(a);
  return cudaGetLastError();
}

} // namespace fg
