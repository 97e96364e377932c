// Tensor slicing and insertion (tcTensorSlice / tcTensorInsert): copies between
// a dense column-major tensor and a rectangular sub-block of another one.
//
// Reference: talshTensorSlice / talshTensorInsert (talshc.cpp:4008-4268,
// :4269-4528) run only on the CPU there (tensor_block_slice_dlf_r8
// tensor_algebra_cpu.F90:6900-6974, tensor_block_insert_dlf_r8 :7216-7290,
// slice = slice*beta + tensor*alpha with alpha = 1, beta = 1 when
// accumulative else 0); its GPU entry points gpu_tensor_block_slice/insert are
// unimplemented stubs (tensor_algebra_gpu_nvidia.cu:4788-4804).
//
// Layout: leading dimensions that the slice covers completely fuse with the
// first partially covered one into one contiguous run (the same bytes in both
// tensors); the remaining slice dimensions index runs ("rows").  A warp copies
// one row when runs are long; short runs are copied element by element.
// Pure data movement (memory-bound): 2 * slice volume * element size bytes,
// 3 * ... when accumulating.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.h"

namespace tb {
namespace {

constexpr int kSliceThreads = 256;

struct SliceParams {
  int nrow;                       // row dimensions after the run
  int64_t run;                    // contiguous elements per row
  int64_t rows;                   // number of rows
  int64_t base;                   // full-tensor offset of the slice origin
  int64_t rext[kMaxRank];         // slice extents of the row dimensions
  int64_t rstr[kMaxRank];         // full-tensor strides of the row dimensions
};

template <typename T> __device__ __forceinline__ T vadd(T a, T b) { return a + b; }
template <> __device__ __forceinline__ float2 vadd<float2>(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
template <> __device__ __forceinline__ double2 vadd<double2>(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}

__device__ __forceinline__ int64_t row_offset(const SliceParams &p, int64_t r) {
  int64_t off = p.base;
  for (int d = 0; d < p.nrow; ++d) {
    const int64_t q = r / p.rext[d];
    off += (r - q * p.rext[d]) * p.rstr[d];
    r = q;
  }
  return off;
}

// INSERT = false: slice[e] (+)= full[map(e)]; true: full[map(e)] (+)= slice[e].
template <typename T, bool INSERT, bool ACC>
__device__ __forceinline__ void move(const T *src, T *dst, int64_t full_off, int64_t slice_off) {
  const int64_t si = INSERT ? slice_off : full_off, di = INSERT ? full_off : slice_off;
  const T v = src[si];
  dst[di] = ACC ? vadd(dst[di], v) : v;
}

// One warp per row (runs of 16 elements or more).
template <typename T, bool INSERT, bool ACC>
__global__ void __launch_bounds__(kSliceThreads) slice_rows_kernel(const T *__restrict__ src, T *dst,
                                                                   const SliceParams p) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (kSliceThreads / 32);
  for (int64_t r = (int64_t)blockIdx.x * (kSliceThreads / 32) + (threadIdx.x >> 5); r < p.rows; r += warps) {
    const int64_t f = row_offset(p, r), s = r * p.run;
    for (int64_t c = lane; c < p.run; c += 32) move<T, INSERT, ACC>(src, dst, f + c, s + c);
  }
}

// One thread per element (short runs).
template <typename T, bool INSERT, bool ACC>
__global__ void __launch_bounds__(kSliceThreads) slice_elems_kernel(const T *__restrict__ src, T *dst,
                                                                    const SliceParams p) {
  const int64_t total = p.rows * p.run;
  const int64_t step = (int64_t)gridDim.x * kSliceThreads;
  for (int64_t e = (int64_t)blockIdx.x * kSliceThreads + threadIdx.x; e < total; e += step) {
    const int64_t r = e / p.run, c = e - r * p.run;
    move<T, INSERT, ACC>(src, dst, row_offset(p, r) + c, e);
  }
}

template <typename T, bool INSERT, bool ACC>
int launch(const void *src, void *dst, const SliceParams &p, cudaStream_t st) {
  const int64_t cap = (int64_t)current_sm_count() * 8;
  if (p.run >= 16) {
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((p.rows + 7) / 8, cap));
    slice_rows_kernel<T, INSERT, ACC><<<(unsigned)blocks, kSliceThreads, 0, st>>>((const T *)src, (T *)dst, p);
  } else {
    const int64_t total = p.rows * p.run;
    const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((total + kSliceThreads - 1) / kSliceThreads, cap));
    slice_elems_kernel<T, INSERT, ACC><<<(unsigned)blocks, kSliceThreads, 0, st>>>((const T *)src, (T *)dst, p);
  }
  note_launch();
  return check_launch(INSERT ? "tensor insert" : "tensor slice");
}

template <typename T>
int dispatch(bool insert, bool acc, const void *src, void *dst, const SliceParams &p, cudaStream_t st) {
  if (insert) return acc ? launch<T, true, true>(src, dst, p, st) : launch<T, true, false>(src, dst, p, st);
  return acc ? launch<T, false, true>(src, dst, p, st) : launch<T, false, false>(src, dst, p, st);
}

int slice_op(bool insert, int kind, int rank, const int *full_dims, const int *slice_dims, const int *offsets,
             const void *src, void *dst, int accumulative, void *stream) {
  if (kind_size(kind) == 0 || rank < 1 || rank > kMaxRank || full_dims == nullptr || slice_dims == nullptr ||
      offsets == nullptr || src == nullptr || dst == nullptr)
    return TALSH_INVALID_ARGS;
  if (!elem_aligned(kind, src) || !elem_aligned(kind, dst)) return TALSH_INVALID_ARGS;
  for (int i = 0; i < rank; ++i)
    if (full_dims[i] <= 0 || slice_dims[i] <= 0 || offsets[i] < 0 || offsets[i] + (int64_t)slice_dims[i] > full_dims[i])
      return TALSH_INVALID_ARGS;
  SliceParams p;
  std::memset(&p, 0, sizeof(p));
  // Run: leading fully covered dimensions plus the first partial one.
  int64_t stride = 1, base = 0;
  int d = 0;
  p.run = 1;
  while (d < rank) {
    base += (int64_t)offsets[d] * stride;
    p.run *= slice_dims[d];
    const bool full = slice_dims[d] == full_dims[d];
    stride *= full_dims[d];
    ++d;
    if (!full) break;
  }
  p.rows = 1;
  for (; d < rank; ++d) {
    base += (int64_t)offsets[d] * stride;
    if (slice_dims[d] > 1) {
      p.rext[p.nrow] = slice_dims[d];
      p.rstr[p.nrow] = stride;
      p.nrow++;
      p.rows *= slice_dims[d];
    }
    stride *= full_dims[d];
  }
  p.base = base;
  const bool acc = accumulative != 0;
  cudaStream_t st = (cudaStream_t)stream;
  switch (kind) {
    case R4: return dispatch<float>(insert, acc, src, dst, p, st);
    case R8: return dispatch<double>(insert, acc, src, dst, p, st);
    case C4: return dispatch<float2>(insert, acc, src, dst, p, st);
    default: return dispatch<double2>(insert, acc, src, dst, p, st);
  }
}

}  // namespace
}  // namespace tb

extern "C" int tcTensorSlice(int data_kind, int rank, const int *full_dims, const int *slice_dims,
                             const int *offsets, const void *full, void *slice, int accumulative, void *stream) {
  return tb::slice_op(false, data_kind, rank, full_dims, slice_dims, offsets, full, slice, accumulative, stream);
}

extern "C" int tcTensorInsert(int data_kind, int rank, const int *full_dims, const int *slice_dims,
                              const int *offsets, const void *slice, void *full, int accumulative, void *stream) {
  return tb::slice_op(true, data_kind, rank, full_dims, slice_dims, offsets, slice, full, accumulative, stream);
}
