// Shared definitions of the talsh-b200 core (host and device code).
#pragma once

#include <cstddef>
#include <cstdint>

#include "talsh.h"
#include "talsh_b200.h"

namespace tb {

constexpr int kMaxRank = MAX_TENSOR_RANK;

inline int kind_size(int kind) {
  switch (kind) {
    case R4: return 4;
    case R8: return 8;
    case C4: return 8;
    case C8: return 16;
    default: return 0;
  }
}
inline bool kind_is_complex(int kind) { return kind == C4 || kind == C8; }
// True when p is aligned to the element size of kind (the kernels move whole
// elements with vector accesses; a complex(8) body must be 16-byte aligned).
inline bool elem_aligned(int kind, const void *p) {
  const int es = kind_size(kind);
  return es > 0 && (reinterpret_cast<uintptr_t>(p) % (uintptr_t)es) == 0;
}

// Flops of a contraction in digital form: 2 M N K H (real) or 8 M N K H
// (complex), M and N the extents of the free indices of L and of R, K the
// contracted extent, H the extent of the hyper indices (in D, L and R), counted
// once.  Without hyper indices this is the reference's 2 ll lr lc
// (tensor_algebra_cpu.F90:4096-4101).
inline double contract_flops(int kind, const int *cptrn, int lrank, const int *ldims, int rrank,
                             const int *rdims) {
  double f = kind_is_complex(kind) ? 8.0 : 2.0;
  for (int i = 0; i < lrank; ++i) f *= (double)ldims[i];
  for (int j = 0; j < rrank; ++j) {
    const int p = cptrn[lrank + j];
    bool hyper = false;
    for (int i = 0; p > 0 && i < lrank; ++i) hyper = hyper || cptrn[i] == p;
    if (p > 0 && !hyper) f *= (double)rdims[j];
  }
  return f;
}

// Real approximant of a complex scale factor that keeps the modulus and the
// sign of the real part (reference cmplx8_to_real8, tensor_algebra_cpu.F90:430-445).
double cmplx8_to_real8(double re, double im);

// Bookkeeping shared by the CUDA translation units.
void note_launch(unsigned n = 1);
void note_cuda_error(const char *what, int code);
void note_error_text(const char *msg);  // sets the text tcLastErrorString returns
int check_launch(const char *what);  // 0 or TALSH_FAILURE after a kernel launch
// SM count of the current device, cached per device (thread-safe).
int current_sm_count();

// Batched contractions for host-side schedulers: `get` returns device scratch
// of scratch_bytes and sets *stage to a pinned host block of stage_bytes that
// stays untouched until the launch's upload has run (nullptr refuses: the
// call returns TRY_LATER).
using BatchScratchFn = void *(*)(void *ctx, size_t scratch_bytes, size_t stage_bytes, void **stage);
int batch_launch_with(int ntasks, const tcContractTask *tasks, BatchScratchFn get, void *ctx, void *stream);
// A batch's scratch is at most batch_fixed_scratch() plus the sum of
// batch_task_scratch_bound over its tasks.
size_t batch_task_scratch_bound(const tcContractTask &task);
size_t batch_fixed_scratch();

}  // namespace tb
