// Per-device one-time setup of kernel attributes.  Attributes set with
// cudaFuncSetAttribute belong to the current device's context, so a process
// that uses several GPUs sets them once on each.  The attribute is set before
// the device is marked, so a thread racing the first call sets it twice at
// worst (the call is idempotent).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

namespace tb {

template <typename F>
void once_per_device(std::atomic<uint64_t> &done, F &&set) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = -1;
  }
  const uint64_t bit = (dev >= 0 && dev < 64) ? (uint64_t(1) << dev) : 0;
  if (bit != 0 && (done.load(std::memory_order_acquire) & bit) != 0) return;
  set();
  if (bit != 0) done.fetch_or(bit, std::memory_order_release);
}

}  // namespace tb
