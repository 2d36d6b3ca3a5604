// noalloc_pcg.cu -- fg_csr_pcg_noalloc: the deterministic PCG on a caller's CSR system
// without any memory allocation.
//
// Who needs it: callers that may not allocate GPU memory at the point of the solve --
// code running under a memory pool that owns the whole device, real-time loops that
// forbid allocator calls, plug-in hosts that hand out only their own buffers.  They pass
// the CSR system and the solution buffer in device memory they already own; everything
// else the solve needs lives in one file-scope device array of fixed size, so the call
// makes no cudaMalloc / cudaFree and uses no allocating library routine.
//
// Limits: at most kNoallocMaxRows rows and kNoallocMaxPositions SELL-32 slots (the CSR
// entries after padding every 32-row slice to its longest row).  Larger systems are
// rejected with FG_INVALID_ARGUMENT before any work is queued.
//
// Sharing: every call on a device uses the same array, which keeps the previous call's
// contents; the set-up kernel rewrites everything the solve reads and the launch clears
// the barrier counter and error flag, so stale contents never leak into a result.  Calls
// that overlap on the GPU (from different host threads or on different streams) race on
// the array and must be serialised by the caller.
//
// Set-up: the array's host-side name is only a stand-in for the device symbol, so the
// first call on each device -- with that device current -- resolves the device address
// with cudaGetSymbolAddress and caches it; make that first call before any stream
// capture begins.
//
// Host waits: every call synchronises `stream` -- once after the set-up kernel, to read
// what it found wrong with the system, and again after the solve, to read its status before
// x is written -- so it returns only when x and info are final.
#include "femm_gpu.h"
#include "common.h"
#include "kernels.cuh"

#include <cmath>
#include <cstdint>
#include <limits>
#include <mutex>

namespace fg
{
namespace
{

constexpr int kNoallocMaxRows = FG_NOALLOC_MAX_ROWS;
constexpr int kNoallocMaxPositions = FG_NOALLOC_MAX_POSITIONS;
constexpr int kNoallocMaxSlices = kNoallocMaxRows / 32;
constexpr int kNoallocMaxGrid = 1024; // PCG CTAs the partial-sum area can hold
constexpr int kPrepThreads = 1024;

// Byte offsets of the regions inside the scratch array (each 256-byte aligned).
constexpr size_t Align(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffSliceOff = 0;
constexpr size_t kOffRowLen = kOffSliceOff + Align(sizeof(int32_t) * (kNoallocMaxSlices + 1));
constexpr size_t kOffCol = kOffRowLen + Align(sizeof(int32_t) * kNoallocMaxRows);
constexpr size_t kOffVal = kOffCol + Align(sizeof(int32_t) * kNoallocMaxPositions);
constexpr size_t kVec = Align(sizeof(double) * kNoallocMaxRows);
constexpr size_t kOffDiag = kOffVal + Align(sizeof(double) * kNoallocMaxPositions);
constexpr size_t kOffInvd = kOffDiag + kVec;
constexpr size_t kOffB = kOffInvd + kVec;
constexpr size_t kOffX = kOffB + kVec;
constexpr size_t kOffR = kOffX + kVec;
constexpr size_t kOffZ = kOffR + kVec;
constexpr size_t kOffP0 = kOffZ + kVec;
constexpr size_t kOffP1 = kOffP0 + kVec;
constexpr size_t kOffQ = kOffP1 + kVec;
constexpr size_t kOffPartials = kOffQ + kVec;
constexpr size_t kOffControl = kOffPartials + Align(sizeof(double) * 2 * 64 * kNoallocMaxGrid);
constexpr size_t kScratchBytes = kOffControl + 256;

// Control block: [0] barrier counter, [1] PCG error flag, [2] set-up error, [3] SELL slots
// used, [4] inverse diagonal usable; doubles from byte 64: PCG info (status, iterations,
// residual).
struct Control {
  unsigned int barrier;
  int32_t pcg_error;
  int32_t setup_error;
  int32_t positions;
  int32_t usable;
  int32_t pad[11];
  double info[3];
};
static_assert(sizeof(Control) <= 256, "control block");

// The only memory this entry point touches besides the caller's buffers.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Set-up error codes (Control::setup_error).
enum : int32_t { kSetupOk = 0, kSetupBadOffsets = 1, kSetupBadColumn = 2, kSetupNonfinite = 3, kSetupTooLarge = 4 };

// One block: CSR -> SELL-32 inside the scratch array, diagonal / inverse / RHS copies.
__global__ void __launch_bounds__(kPrepThreads)
    PrepareKernel(int n, const int32_t *__restrict__ ro, const int32_t *__restrict__ col,
                  const double *__restrict__ val, const double *__restrict__ diag,
                  const double *__restrict__ rhs, unsigned char *__restrict__ scratch)
{
  __shared__ int32_t width[kNoallocMaxSlices];
  __shared__ int32_t err;
  int32_t *slice_off = reinterpret_cast<int32_t *>(scratch + kOffSliceOff);
  int32_t *row_len = reinterpret_cast<int32_t *>(scratch + kOffRowLen);
  int32_t *sell_col = reinterpret_cast<int32_t *>(scratch + kOffCol);
  double *sell_val = reinterpret_cast<double *>(scratch + kOffVal);
  double *d = reinterpret_cast<double *>(scratch + kOffDiag);
  double *inv = reinterpret_cast<double *>(scratch + kOffInvd);
  double *b = reinterpret_cast<double *>(scratch + kOffB);
  Control *ctl = reinterpret_cast<Control *>(scratch + kOffControl);
  const int n_pad = (n + 31) / 32 * 32, slices = n_pad / 32;
  if (threadIdx.x == 0)
    err = kSetupOk;
  for (int s = threadIdx.x; s < slices; s += blockDim.x)
    width[s] = 0;
  __syncthreads();
  if (threadIdx.x == 0 && ro[0] != 0)
    err = kSetupBadOffsets;
  for (int r = threadIdx.x; r < n_pad; r += blockDim.x) {
    int len = 0;
    if (r < n) {
      len = ro[r + 1] - ro[r];
      if (len < 0)
        atomicExch(&err, kSetupBadOffsets);
    }
    row_len[r] = len > 0 ? len : 0;
    if (len > 0)
      atomicMax(&width[r >> 5], len);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long total = 0;
    for (int s = 0; s < slices; ++s) {
      slice_off[s] = static_cast<int32_t>(total < kNoallocMaxPositions ? total : kNoallocMaxPositions);
      total += 32LL * width[s];
    }
    slice_off[slices] = static_cast<int32_t>(total < kNoallocMaxPositions ? total : kNoallocMaxPositions);
    if (total > kNoallocMaxPositions && err == kSetupOk)
      err = kSetupTooLarge;
    ctl->positions = static_cast<int32_t>(total < kNoallocMaxPositions ? total : kNoallocMaxPositions);
  }
  __syncthreads();
  if (err != kSetupOk) {
    if (threadIdx.x == 0) {
      ctl->setup_error = err;
      ctl->usable = 0;
    }
    return;
  }
  // Scatter every row into its slice; padding slots repeat the row index with value 0.
  int usable = 1;
  for (int r = threadIdx.x; r < n_pad; r += blockDim.x) {
    const int s = r >> 5, lane = r & 31, w_max = width[s];
    const size_t base = static_cast<size_t>(slice_off[s]) + lane;
    const int len = row_len[r];
    for (int w = 0; w < w_max; ++w) {
      const size_t pos = base + 32 * static_cast<size_t>(w);
      if (w < len) {
        const int c = col[ro[r] + w];
        const double v = val[ro[r] + w];
        if (c < 0 || c >= n)
          atomicExch(&err, kSetupBadColumn);
        if (!isfinite(v))
          atomicExch(&err, kSetupNonfinite);
        sell_col[pos] = (c >= 0 && c < n) ? c : r;
        sell_val[pos] = v;
      } else {
        sell_col[pos] = r < n ? r : 0;
        sell_val[pos] = 0.0;
      }
    }
    if (r < n) {
      const double dv = diag[r], iv = 1.0 / dv;
      if (!isfinite(dv))
        atomicExch(&err, kSetupNonfinite);
      // Usable inverse: finite, positive and normal (BuildJacobiInverseDiagonal's rule).
      const bool good = isfinite(dv) && dv > 0.0 && isfinite(iv) && iv >= 2.2250738585072014e-308;
      usable = usable && good;
      d[r] = dv;
      inv[r] = good ? iv : 0.0;
      b[r] = rhs[r];
    } else {
      d[r] = 1.0;
      inv[r] = 0.0;
      b[r] = 0.0;
    }
  }
  const int all_usable = __syncthreads_and(usable);
  if (threadIdx.x == 0) {
    ctl->setup_error = err;
    ctl->usable = all_usable;
  }
}

std::mutex g_address_mutex;
constexpr int kMaxDevices = 64;
void *g_address[kMaxDevices] = {};

// Device address of the scratch array on the current device (resolved once per device).
Status ScratchAddress(unsigned char **out)
{
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
    cudaGetLastError();
    return Status::kGpuUnavailable;
  }
  std::lock_guard<std::mutex> lock(g_address_mutex);
  if (!g_address[device]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) {
      cudaGetLastError();
      return Status::kGpuUnavailable;
    }
    g_address[device] = ptr;
  }
  *out = static_cast<unsigned char *>(g_address[device]);
  return Status::kOk;
}

Status NoallocPcg(int32_t n, const int32_t *ro, const int32_t *col, const double *val,
                  const double *diag, const double *rhs, double tol, int32_t maxit, double *x,
                  fg_linear_info *info, cudaStream_t stream)
{
  if (!info)
    return Status::kInvalidArgument;
  *info = fg_linear_info{ToInt(Status::kInvalidArgument), 0, std::numeric_limits<double>::infinity()};
  if (n <= 0 || n > kNoallocMaxRows || !ro || !col || !val || !diag || !rhs || !x)
    return Status::kInvalidArgument;
  if (!(tol > 0.0) || !(tol < 1.0) || !std::isfinite(tol) || maxit < 0)
    return Status::kOk; // the solve itself reports INVALID_ARGUMENT, as GpuCsrSolver does
  unsigned char *scratch = nullptr;
  Status s = ScratchAddress(&scratch);
  if (s != Status::kOk)
    return s;
  const int grid_cap = PcgMaxGrid(1);
  if (grid_cap <= 0)
    return Status::kGpuUnavailable;
  if (grid_cap > kNoallocMaxGrid)
    return Status::kUnsupportedFeature;
  PrepareKernel<<<1, kPrepThreads, 0, stream>>>(n, ro, col, val, diag, rhs, scratch);
  if (cudaGetLastError() != cudaSuccess)
    return Status::kInternalError;
  Control control{};
  if (cudaMemcpyAsync(&control, scratch + kOffControl, sizeof(Control), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return Status::kInternalError;
  if (control.setup_error != kSetupOk)
    return Status::kInvalidArgument;
  const int n_pad = (n + 31) / 32 * 32;
  PcgArgs a{};
  a.n = n;
  a.n_pad = n_pad;
  a.slices = n_pad / 32;
  a.kp = 1;
  a.items = 1;
  a.slice_off = reinterpret_cast<const int32_t *>(scratch + kOffSliceOff);
  a.row_len = reinterpret_cast<const int32_t *>(scratch + kOffRowLen);
  a.sell_col = reinterpret_cast<const int32_t *>(scratch + kOffCol);
  a.values = reinterpret_cast<const double *>(scratch + kOffVal);
  a.value_stride = 1;
  a.value_item = 1;
  a.diag = reinterpret_cast<const double *>(scratch + kOffDiag);
  a.invd = reinterpret_cast<const double *>(scratch + kOffInvd);
  a.diag_stride = 1;
  a.diag_item = 1;
  a.use_inverse = control.usable;
  a.b = reinterpret_cast<const double *>(scratch + kOffB);
  a.x = reinterpret_cast<double *>(scratch + kOffX);
  a.r = reinterpret_cast<double *>(scratch + kOffR);
  a.z = reinterpret_cast<double *>(scratch + kOffZ);
  a.p0 = reinterpret_cast<double *>(scratch + kOffP0);
  a.p1 = reinterpret_cast<double *>(scratch + kOffP1);
  a.q = reinterpret_cast<double *>(scratch + kOffQ);
  a.partials = reinterpret_cast<double *>(scratch + kOffPartials);
  Control *dctl = reinterpret_cast<Control *>(scratch + kOffControl);
  a.barrier = &dctl->barrier;
  a.error = &dctl->pcg_error;
  a.info = dctl->info;
  a.tolerance = tol;
  a.max_iterations = maxit;
  a.active_mask = 1u;
  a.timeout_ns = 5000000000LL;
  a.trace = nullptr;
  if (LaunchPcg(a, nullptr, nullptr, stream) != cudaSuccess) {
    cudaGetLastError();
    return Status::kInternalError;
  }
  // The solve's status first: x is written only when the kernel finished without an error
  // (a grid-barrier wait that ran out leaves x untouched and reports INTERNAL_ERROR).
  if (cudaMemcpyAsync(&control, scratch + kOffControl, sizeof(Control), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    info->status = ToInt(Status::kInternalError);
    return Status::kInternalError;
  }
  if (control.pcg_error != 0) {
    info->status = ToInt(Status::kInternalError);
    return Status::kInternalError;
  }
  if (cudaMemcpyAsync(x, scratch + kOffX, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    info->status = ToInt(Status::kInternalError);
    return Status::kInternalError;
  }
  info->status = static_cast<int32_t>(control.info[0]);
  info->iterations = static_cast<int32_t>(control.info[1]);
  info->residual_l2 = control.info[2];
  return Status::kOk;
}

} // namespace
} // namespace fg

extern "C" int fg_csr_pcg_noalloc(int32_t n, const int32_t *row_offsets, const int32_t *columns,
                                  const double *values, const double *diagonal, const double *rhs,
                                  double relative_tolerance, int32_t max_iterations, double *x,
                                  fg_linear_info *info, void *stream)
{
  return fg::ToInt(fg::NoallocPcg(n, row_offsets, columns, values, diagonal, rhs,
                                  relative_tolerance, max_iterations, x, info,
                                  static_cast<cudaStream_t>(stream)));
}
