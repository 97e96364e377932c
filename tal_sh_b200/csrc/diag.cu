// Launch bookkeeping and CUDA error capture shared by the kernel modules.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "common.h"

namespace tb {
namespace {
std::atomic<unsigned long long> g_launches{0};
std::mutex g_err_mu;
char g_last_err[256] = "";
}  // namespace

void note_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void note_cuda_error(const char *what, int code) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  std::snprintf(g_last_err, sizeof(g_last_err), "%s: %s (%d)", what,
                cudaGetErrorString((cudaError_t)code), code);
}

void note_error_text(const char *msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  std::snprintf(g_last_err, sizeof(g_last_err), "%s", msg);
}

int current_sm_count() {
  static std::atomic<int> cache[64];  // zero-initialised: 0 = not probed yet
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); dev = 0; }
  if (dev < 0 || dev >= 64) return 148;
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
      cudaGetLastError();
      v = 148;
    }
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

int check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return TALSH_SUCCESS;
  note_cuda_error(what, (int)e);
  return TALSH_FAILURE;
}
}  // namespace tb

extern "C" unsigned long long tcKernelLaunchCount(void) { return tb::g_launches.load(); }

extern "C" const char *tcLastErrorString(void) { return tb::g_last_err; }
