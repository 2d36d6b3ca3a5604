// pcg.cu -- kernel selection and the cooperative launch of the batched PCG
// (kernel template in pcg_kernel.cuh; instantiations in pcg_f64*.cu / pcg_f32*.cu).
#include "kernels.cuh"

#include <atomic>
#include <cstdlib>
#include <cstring>

namespace fg
{

const void *PcgKernelF64(int kp);
const void *PcgKernelF32(int kp);
const void *PcgKernelF64Block(int kp, int bs);
const void *PcgKernelF32Block(int kp, int bs);
const void *MultiPcgKernelF64(int kp);
const void *PcgKernelF64OneReduction(int kp);
const void *PcgKernelF64Wide(int kp);

namespace
{

constexpr int kPcgThreads = 512;
constexpr int kPcgWarps = kPcgThreads / 32;

const void *SelectKernel(int kp, int precision, int bs, bool one_reduction = false)
{
  if (one_reduction)
    return precision == 0 && bs == 0 ? PcgKernelF64OneReduction(kp) : nullptr;
  if (bs == 0)
    return precision == 0 ? PcgKernelF64(kp) : PcgKernelF32(kp);
  return precision == 0 ? PcgKernelF64Block(kp, bs) : PcgKernelF32Block(kp, bs);
}

int ItemsPerThread(int kp, int precision)
{
  if (precision == 0)
    return kp >= 2 ? 2 : 1;
  return kp >= 4 ? 4 : (kp >= 2 ? 2 : 1);
}

// Dynamic shared memory of the block-Jacobi staging buffer: U rows x KP items per warp.
size_t StagingBytes(int kp, int precision, int bs)
{
  if (bs == 0)
    return 0;
  const int rows_per_warp = 32 * ItemsPerThread(kp, precision) / kp;
  const int u = bs > rows_per_warp ? bs : rows_per_warp;
  return static_cast<size_t>(kPcgWarps) * u * kp * (precision == 0 ? 8 : 4);
}

// Co-resident CTAs of one kernel shape (at most `cap` per SM), 0 on failure.
int KernelGrid(const void *kernel, size_t smem, int threads = kPcgThreads, int cap = 2)
{
  int device = 0, sms = 0, per_sm = 0;
  if (!kernel || cudaGetDevice(&device) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return 0;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess)
    return 0;
  return sms * (per_sm < cap ? per_sm : cap);
}

// Dynamic shared memory a launch may use for staging plus the column cache: two CTAs of
// 512 threads per SM must stay resident (228 KB per SM, about 12 KB static per CTA).
constexpr size_t kColumnCacheBudget = 104 * 1024;

// FG_PCG_VALUE_RING=0 in the environment turns the cp.async value ring off (for A/B timing).
bool ValueRingEnabled()
{
  static const bool enabled = [] {
    const char *v = std::getenv("FG_PCG_VALUE_RING");
    return !(v && v[0] == '0');
  }();
  return enabled;
}

// The column cache is off unless FG_PCG_COL_CACHE=1: beside the value ring its shared
// memory shrinks L1 and costs the update phase more than the cached indices save
// (measured on the 251k-node batch of 8: 69.9 us per CG iteration without, 73.2 with).
bool ColumnCacheEnabled()
{
  static const bool enabled = [] {
    const char *v = std::getenv("FG_PCG_COL_CACHE");
    return v && v[0] == '1';
  }();
  return enabled;
}

// FG_PCG_BLOCK=1024 selects the 1024-thread CTAs where a plan's autotuner has not chosen
// (read at every launch).
bool WideBlocksEnabled()
{
  const char *v = std::getenv("FG_PCG_BLOCK");
  return v && std::strcmp(v, "1024") == 0;
}

} // namespace

namespace
{
std::atomic<long long> g_wait_limit_ns{kDefaultWaitLimitNs};
} // namespace

long long PcgWaitLimitNs() { return g_wait_limit_ns.load(std::memory_order_relaxed); }

long long SetPcgWaitLimitNs(long long ns)
{
  return g_wait_limit_ns.exchange(ns > 0 ? ns : kDefaultWaitLimitNs, std::memory_order_relaxed);
}

bool PcgSupported(int kp, int precision, int block_size)
{
  return SelectKernel(kp, precision, block_size) != nullptr;
}

// Grid of the Jacobi kernels for kp items (the same for both precisions, so FP64 and
// FP32 launches of one batch reduce over the same partition); block-Jacobi launches use
// at most this many CTAs.
int PcgMaxGrid(int kp)
{
  int grid = 0;
  for (int precision = 0; precision < 2; ++precision) {
    const int g = KernelGrid(SelectKernel(kp, precision, 0), 0);
    if (g <= 0)
      return 0;
    grid = precision == 0 ? g : (g < grid ? g : grid);
  }
  return grid;
}

size_t PcgPartialsDoubles(int grid, bool one_reduction)
{
  return static_cast<size_t>(2) * (one_reduction ? 96 : 64) * static_cast<size_t>(grid);
}

cudaError_t LaunchPcg(PcgArgs args, int *grid_out, int *block_out, cudaStream_t stream)
{
  const int bs = args.blocks ? args.block_size : 0;
  args.block_size = bs;
  const void *kernel = SelectKernel(args.kp, args.precision, bs, args.one_reduction != 0);
  if (args.one_reduction && (!args.t0 || !args.t1))
    return cudaErrorInvalidValue;
  if (!kernel)
    return cudaErrorInvalidValue;
  size_t smem = StagingBytes(args.kp, args.precision, bs);
  int max_grid = PcgMaxGrid(args.kp);
  const int own = KernelGrid(kernel, smem);
  if (own < max_grid)
    max_grid = own;
  if (max_grid <= 0)
    return cudaErrorInvalidConfiguration;
  const int iv = ItemsPerThread(args.kp, args.precision);
  const int rows_per_warp = 32 * iv / args.kp;
  const int warp_slices = args.n_pad / rows_per_warp;
  int grid = (warp_slices + kPcgWarps - 1) / kPcgWarps; // row groups of kPcgWarps warps
  if (grid > max_grid)
    grid = max_grid;
  if (grid < 1)
    grid = 1;
  // Wide CTAs (FP64 Jacobi): the same row groups two to a CTA of 1024 threads, one CTA per
  // SM -- the same rows, order and partial sums, so the same bits.
  const bool want_wide = args.block_request == 0 ? WideBlocksEnabled() : args.block_request == 1;
  const void *wide_kernel = want_wide && args.precision == 0 && bs == 0 && !args.one_reduction && grid % 2 == 0
                                ? PcgKernelF64Wide(args.kp)
                                : nullptr;
  const bool wide = wide_kernel && KernelGrid(wide_kernel, 0, 2 * kPcgThreads, 1) >= grid / 2;
  const int threads = wide ? 2 * kPcgThreads : kPcgThreads, warps = threads / 32;
  const int ctas = wide ? grid / 2 : grid, cap = wide ? 1 : 2;
  const size_t budget = wide ? 200 * 1024 : kColumnCacheBudget;
  if (wide)
    kernel = wide_kernel;
  // Value ring (16-byte item vectors, per-item operators): 2 stages x kRingEntries entries x
  // 32 lanes x 16 bytes per warp, after the block-Jacobi staging buffer.
  args.value_ring = 0;
  args.value_ring_offset = 0;
  const bool want_ring = args.ring_request == 0 ? ValueRingEnabled() : args.ring_request == 1;
  const bool ring_shape = (args.precision == 0 ? 8 : 4) * iv == 16 && args.value_item && want_ring;
  if (ring_shape) {
    const size_t offset = (smem + 15) / 16 * 16;
    const size_t total = offset + static_cast<size_t>(warps) * 2 * kRingEntries * 32 * 16;
    if (total <= budget && KernelGrid(kernel, total, threads, cap) >= ctas) {
      args.value_ring = 1;
      args.value_ring_offset = static_cast<int32_t>(offset);
      smem = total;
    }
  }
  // Column-index cache: the largest slice range any CTA's rows touch, if it fits in the
  // shared memory that still leaves the grid co-resident.
  args.col_cache = 0;
  args.col_cache_offset = 0;
  const bool want_cache = args.col_cache_request == 0 ? ColumnCacheEnabled() : args.col_cache_request == 1;
  if (args.host_slice_off && want_cache) {
    size_t most = 0;
    for (int g = 0; g < ctas; ++g) {
      const long long w0 = static_cast<long long>(warp_slices) * g / ctas;
      const long long w1 = static_cast<long long>(warp_slices) * (g + 1) / ctas;
      if (w1 <= w0)
        continue;
      const long long s0 = (w0 * rows_per_warp) >> 5, s1 = (w1 * rows_per_warp - 1) >> 5;
      const size_t p = static_cast<size_t>(args.host_slice_off[s1 + 1] - args.host_slice_off[s0]);
      most = p > most ? p : most;
    }
    const size_t offset = (smem + 15) / 16 * 16;
    const size_t total = offset + most * sizeof(int32_t);
    if (total <= budget && KernelGrid(kernel, total, threads, cap) >= ctas) {
      args.col_cache = 1;
      args.col_cache_offset = static_cast<int32_t>(offset);
      smem = total;
    }
  }
  cudaError_t e = cudaMemsetAsync(args.barrier, 0, sizeof(unsigned), stream);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(args.error, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess)
    return e;
  void *params[] = {&args};
  e = cudaLaunchCooperativeKernel(kernel, dim3(ctas), dim3(threads), params, smem, stream);
  if (grid_out)
    *grid_out = ctas;
  if (block_out)
    *block_out = threads;
  return e;
}

size_t MultiPcgRingBytes(int kp)
{
  // The value ring carries 16-byte item vectors: FP64 with two items per thread.
  const int iv = ItemsPerThread(kp, 0);
  if (8 * iv != 16 || !ValueRingEnabled())
    return 0;
  return static_cast<size_t>(kPcgWarps) * 2 * kRingEntries * 32 * 16;
}

int MultiPcgMaxGrid(int kp)
{
  const void *kernel = MultiPcgKernelF64(kp);
  return kernel ? KernelGrid(kernel, MultiPcgRingBytes(kp)) : 0;
}

cudaError_t LaunchMultiPcg(PcgGroups t, int kp, int ctas, cudaStream_t stream)
{
  const void *kernel = MultiPcgKernelF64(kp);
  const int max_grid = MultiPcgMaxGrid(kp);
  if (!kernel || ctas < 1 || ctas > max_grid)
    return cudaErrorInvalidConfiguration;
  void *params[] = {&t};
  return cudaLaunchCooperativeKernel(kernel, dim3(ctas), dim3(kPcgThreads), params, MultiPcgRingBytes(kp),
                                     stream);
}

} // namespace fg
