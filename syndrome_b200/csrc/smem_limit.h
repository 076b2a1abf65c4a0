// Dynamic shared-memory limit of a kernel (host side).
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

namespace syn {

// Raises kernel fn's dynamic shared-memory limit on the current device to the most the
// device allows (once per kernel and device).  The limit is a process-wide attribute
// of the kernel: setting it to what one launch needs would race with a concurrent
// launch of the same kernel (another thread, another decoder, another batch size)
// that needs more, and that launch would fail.
inline cudaError_t allow_max_dynamic_smem(const void* fn) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, dev})) return cudaSuccess;
  int optin = 0;
  cudaFuncAttributes attr{};
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess ||
      (e = cudaFuncGetAttributes(&attr, fn)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)attr.sharedSizeBytes)) != cudaSuccess)
    return e;
  done.insert({fn, dev});
  return cudaSuccess;
}

}  // namespace syn
