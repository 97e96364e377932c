// Tensor contraction for callers that must not allocate device memory.
//
// tcTensorContract takes its scratch (the gather-GEMM offset tables, and the
// partial sums of a full contraction) from the caller, who normally gets it
// from cudaMalloc or a pool.  Some callers cannot: code running inside a
// memory pool's own allocation callback or a custom allocator, a host that
// has handed the whole device budget to another runtime, or a real-time
// driver loop where a cudaMalloc (an implicit device synchronisation) is not
// allowed.  tcTensorContractNoAlloc serves them with a fixed scratch array
// compiled into this library: every GPU that loads the library holds
// kNoAllocScratchBytes of it until the process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "common.h"

namespace tb {
size_t contract_scratch_bytes(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                              const int *ldims, int rrank, const int *rdims);
int contract_launch(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                    const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                    const void *R, double alpha_re, double alpha_im, int conj_bits,
                    int accumulative, void *scratch, size_t scratch_bytes, void *stream);

namespace {

constexpr size_t kNoAllocScratchBytes = TC_CONTRACT_NOALLOC_SCRATCH_BYTES;

// The scratch itself.  Host code must never pass this name to a kernel: on the
// host it is only a stand-in; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_contract_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void *g_scratch_dev[kMaxDevices] = {};  // device address of g_contract_scratch, per device

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does the lookup) and kept for the
// life of the process: a device reset after that first call is not supported,
// since the module would be reloaded at another address.
int scratch_address(void **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    note_cuda_error("tcTensorContractNoAlloc: cudaGetDevice", (int)e);
    return TALSH_FAILURE;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    note_error_text("tcTensorContractNoAlloc: device ordinal beyond the supported 64");
    return TALSH_LIMIT_EXCEEDED;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (g_scratch_dev[dev] == nullptr) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_contract_scratch);
    if (e != cudaSuccess || p == nullptr) {
      note_cuda_error("tcTensorContractNoAlloc: cudaGetSymbolAddress", (int)e);
      return TALSH_FAILURE;
    }
    g_scratch_dev[dev] = p;
  }
  *out = g_scratch_dev[dev];
  return TALSH_SUCCESS;
}

}  // namespace
}  // namespace tb

extern "C" size_t tcTensorContractNoAllocMaxScratch(void) { return tb::kNoAllocScratchBytes; }

extern "C" int tcTensorContractNoAlloc(int data_kind, const int *cptrn, int drank,
                                       const int *ddims, int lrank, const int *ldims, int rrank,
                                       const int *rdims, void *D, const void *L, const void *R,
                                       double alpha_re, double alpha_im, int conj_bits,
                                       int accumulative, void *stream) {
  // The scratch need is a function of the shapes only; reject what does not fit
  // before touching the device.
  const size_t need = tb::contract_scratch_bytes(data_kind, cptrn, drank, ddims, lrank, ldims,
                                                 rrank, rdims);
  if (need > tb::kNoAllocScratchBytes) {
    char msg[200];
    std::snprintf(msg, sizeof(msg),
                  "tcTensorContractNoAlloc: shape needs %zu bytes of scratch, above the fixed "
                  "%zu-byte array; use tcTensorContract with caller scratch",
                  need, tb::kNoAllocScratchBytes);
    tb::note_error_text(msg);
    return TALSH_LIMIT_EXCEEDED;
  }
  void *scratch = nullptr;
  if (need > 0) {
    const int rc = tb::scratch_address(&scratch);
    if (rc != TALSH_SUCCESS) return rc;
  }
  // Every table entry and partial sum is written by the launch before it is
  // read, so nothing in the array has to start at zero.
  return tb::contract_launch(data_kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims, D, L, R,
                             alpha_re, alpha_im, conj_bits, accumulative, scratch,
                             tb::kNoAllocScratchBytes, stream);
}
