// common.h -- status codes, CUDA error handling and device buffers for libfemmgpu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>

namespace fg
{

// Status numbering of gpu_solver/src/core/types.h:11-28.
enum class Status : int {
  kOk = 0,
  kInputIo = 1,
  kInvalidArgument = 2,
  kUnsupportedFeature = 3,
  kMeshInvalid = 4,
  kBoundaryInvalid = 5,
  kGpuUnavailable = 6,
  kGpuAllocationFailed = 7,
  kAssemblyFailed = 8,
  kLinearSolveNotConverged = 9,
  kLinearSolveBreakdown = 10,
  kNumericalNonfinite = 11,
  kOutputIo = 12,
  kInternalError = 13,
  kNonlinearSolveNotConverged = 14,
  kInvalidMaterial = 15,
};

const char *StatusName(Status status);

inline int ToInt(Status s) { return static_cast<int>(s); }

// Device memory owned by one plan.  Grows only; never shrinks until the plan dies.
template <typename T> class DeviceArray
{
public:
  DeviceArray() = default;
  DeviceArray(const DeviceArray &) = delete;
  DeviceArray &operator=(const DeviceArray &) = delete;
  DeviceArray(DeviceArray &&other) noexcept { swap(other); }
  DeviceArray &operator=(DeviceArray &&other) noexcept
  {
    swap(other);
    return *this;
  }
  ~DeviceArray() { reset(); }

  Status ensure(size_t count)
  {
    if (count <= capacity_)
      return Status::kOk;
    reset();
    void *p = nullptr;
    if (cudaMalloc(&p, (count > 0 ? count : 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      return Status::kGpuAllocationFailed;
    }
    ptr_ = static_cast<T *>(p);
    capacity_ = count;
    return Status::kOk;
  }
  Status upload(const T *host, size_t count, cudaStream_t stream = nullptr)
  {
    Status s = ensure(count);
    if (s != Status::kOk)
      return s;
    if (count == 0)
      return Status::kOk;
    return cudaMemcpyAsync(ptr_, host, count * sizeof(T), cudaMemcpyHostToDevice, stream) ==
                   cudaSuccess
               ? Status::kOk
               : Status::kInternalError;
  }
  void reset()
  {
    if (ptr_)
      cudaFree(ptr_);
    ptr_ = nullptr;
    capacity_ = 0;
  }
  T *get() const { return ptr_; }
  size_t capacity() const { return capacity_; }
  size_t bytes() const { return capacity_ * sizeof(T); }

private:
  void swap(DeviceArray &o)
  {
    std::swap(ptr_, o.ptr_);
    std::swap(capacity_, o.capacity_);
  }
  T *ptr_ = nullptr;
  size_t capacity_ = 0;
};

// Pinned host staging.
template <typename T> class PinnedArray
{
public:
  PinnedArray() = default;
  PinnedArray(const PinnedArray &) = delete;
  PinnedArray &operator=(const PinnedArray &) = delete;
  ~PinnedArray() { reset(); }
  Status ensure(size_t count)
  {
    if (count <= capacity_)
      return Status::kOk;
    reset();
    void *p = nullptr;
    if (cudaMallocHost(&p, (count > 0 ? count : 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      return Status::kGpuAllocationFailed;
    }
    ptr_ = static_cast<T *>(p);
    capacity_ = count;
    return Status::kOk;
  }
  void reset()
  {
    if (ptr_)
      cudaFreeHost(ptr_);
    ptr_ = nullptr;
    capacity_ = 0;
  }
  T *get() const { return ptr_; }

private:
  T *ptr_ = nullptr;
  size_t capacity_ = 0;
};

#define FG_CUDA_OK(expr) ((expr) == cudaSuccess)

} // namespace fg
