// Element-wise kernels: init, scale and the 1-norm reduction.
//
// Scale follows tensor_block_scale (reference tensor_algebra_cpu.F90:1821-1890):
// real kinds multiply by cmplx8_to_real8(alpha) in their own precision, complex
// kinds by alpha with the textbook complex product; every product and sum is
// rounded on its own (no FMA), so results are bit-exact with the CPU rules.
// The 1-norm accumulates |x| in double with a fixed two-pass partition (the
// partition depends only on the volume), so it is run-to-run deterministic.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.h"

namespace tb {
namespace {

constexpr int kThreads = 256;

template <typename T> struct ScaleOp;
template <> struct ScaleOp<float> {
  __device__ static float apply(float x, double sr, double) { return __fmul_rn(x, (float)sr); }
  __device__ static double absd(float x) { return (double)fabsf(x); }
};
template <> struct ScaleOp<double> {
  __device__ static double apply(double x, double sr, double) { return __dmul_rn(x, sr); }
  __device__ static double absd(double x) { return fabs(x); }
};
template <> struct ScaleOp<float2> {
  __device__ static float2 apply(float2 x, double sr, double si) {
    const float ar = (float)sr, ai = (float)si;
    return make_float2(__fsub_rn(__fmul_rn(x.x, ar), __fmul_rn(x.y, ai)),
                       __fadd_rn(__fmul_rn(x.x, ai), __fmul_rn(x.y, ar)));
  }
  __device__ static double absd(float2 x) { return (double)hypotf(x.x, x.y); }
};
template <> struct ScaleOp<double2> {
  __device__ static double2 apply(double2 x, double sr, double si) {
    return make_double2(__dsub_rn(__dmul_rn(x.x, sr), __dmul_rn(x.y, si)),
                        __dadd_rn(__dmul_rn(x.x, si), __dmul_rn(x.y, sr)));
  }
  __device__ static double absd(double2 x) { return hypot(x.x, x.y); }
};

template <typename T>
__global__ void __launch_bounds__(kThreads) init_kernel(T *dst, int64_t vol, T val) {
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < vol; i += stride) dst[i] = val;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) scale_kernel(T *dst, int64_t vol, double sr, double si) {
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < vol; i += stride)
    dst[i] = ScaleOp<T>::apply(dst[i], sr, si);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block sum in a fixed order: per-warp shuffle trees, then warp 0 over the warp sums.
__device__ double block_sum(double v) {
  __shared__ double ws[kThreads / 32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = (lane < kThreads / 32) ? ws[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;  // valid in thread 0
}

// Pass 1: block b sums the contiguous chunk [b*chunk, min((b+1)*chunk, vol)).
template <typename T>
__global__ void __launch_bounds__(kThreads) norm1_partial_kernel(const T *__restrict__ src,
                                                                 int64_t vol, int64_t chunk,
                                                                 double *partial) {
  const int64_t beg = (int64_t)blockIdx.x * chunk;
  const int64_t end = min(vol, beg + chunk);
  double acc = 0.0;
  for (int64_t i = beg + threadIdx.x; i < end; i += kThreads) acc += ScaleOp<T>::absd(src[i]);
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Pass 2: one block folds the partials in a fixed order.
__global__ void __launch_bounds__(kThreads) norm1_final_kernel(const double *partial, int n,
                                                               double *result) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += kThreads) acc += partial[i];
  const double s = block_sum(acc);
  if (threadIdx.x == 0) *result = s;
}

int grid_for(int64_t n) {
  const int64_t g = (n + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

// Number of norm partial blocks: a function of the volume only.
int norm1_blocks(size_t vol) {
  const size_t per = 16384;
  size_t b = (vol + per - 1) / per;
  if (b < 1) b = 1;
  if (b > 2048) b = 2048;
  return (int)b;
}

}  // namespace

double cmplx8_to_real8(double re, double im) {
  if (re != 0.0) return std::hypot(re, im) * (re > 0.0 ? 1.0 : -1.0);
  return im;
}

}  // namespace tb

using namespace tb;

extern "C" int tcTensorInit(int data_kind, size_t vol, void *dst, double val_re, double val_im,
                            void *stream) {
  if (kind_size(data_kind) == 0 || (dst == nullptr && vol > 0)) return TALSH_INVALID_ARGS;
  if (vol > 0 && !elem_aligned(data_kind, dst)) return TALSH_INVALID_ARGS;
  if (vol == 0) return TALSH_SUCCESS;
  cudaStream_t st = (cudaStream_t)stream;
  const int grid = grid_for((int64_t)vol);
  switch (data_kind) {
    case R4: init_kernel<float><<<grid, kThreads, 0, st>>>((float *)dst, vol, (float)val_re); break;
    case R8: init_kernel<double><<<grid, kThreads, 0, st>>>((double *)dst, vol, val_re); break;
    case C4:
      init_kernel<float2><<<grid, kThreads, 0, st>>>((float2 *)dst, vol,
                                                     make_float2((float)val_re, (float)val_im));
      break;
    case C8:
      init_kernel<double2><<<grid, kThreads, 0, st>>>((double2 *)dst, vol, make_double2(val_re, val_im));
      break;
  }
  note_launch();
  return check_launch("init_kernel");
}

extern "C" int tcTensorScale(int data_kind, size_t vol, void *dst, double alpha_re,
                             double alpha_im, void *stream) {
  if (kind_size(data_kind) == 0 || (dst == nullptr && vol > 0)) return TALSH_INVALID_ARGS;
  if (vol > 0 && !elem_aligned(data_kind, dst)) return TALSH_INVALID_ARGS;
  if (vol == 0) return TALSH_SUCCESS;
  cudaStream_t st = (cudaStream_t)stream;
  const int grid = grid_for((int64_t)vol);
  double sr = alpha_re, si = alpha_im;
  if (!kind_is_complex(data_kind)) { sr = cmplx8_to_real8(alpha_re, alpha_im); si = 0.0; }
  switch (data_kind) {
    case R4: scale_kernel<float><<<grid, kThreads, 0, st>>>((float *)dst, vol, sr, si); break;
    case R8: scale_kernel<double><<<grid, kThreads, 0, st>>>((double *)dst, vol, sr, si); break;
    case C4: scale_kernel<float2><<<grid, kThreads, 0, st>>>((float2 *)dst, vol, sr, si); break;
    case C8: scale_kernel<double2><<<grid, kThreads, 0, st>>>((double2 *)dst, vol, sr, si); break;
  }
  note_launch();
  return check_launch("scale_kernel");
}

extern "C" size_t tcTensorNorm1Scratch(size_t vol) { return (size_t)norm1_blocks(vol) * sizeof(double); }

namespace tb {
// Shared by the public entry point and by callers that bring their own scratch.
int norm1_launch(int data_kind, size_t vol, const void *src, double *result_dev, double *partial,
                 cudaStream_t st) {
  const int nb = norm1_blocks(vol);
  const int64_t chunk = (int64_t)((vol + nb - 1) / nb);
  switch (data_kind) {
    case R4: norm1_partial_kernel<float><<<nb, kThreads, 0, st>>>((const float *)src, vol, chunk, partial); break;
    case R8: norm1_partial_kernel<double><<<nb, kThreads, 0, st>>>((const double *)src, vol, chunk, partial); break;
    case C4: norm1_partial_kernel<float2><<<nb, kThreads, 0, st>>>((const float2 *)src, vol, chunk, partial); break;
    case C8: norm1_partial_kernel<double2><<<nb, kThreads, 0, st>>>((const double2 *)src, vol, chunk, partial); break;
    default: return TALSH_INVALID_ARGS;
  }
  note_launch();
  norm1_final_kernel<<<1, kThreads, 0, st>>>(partial, nb, result_dev);
  note_launch();
  return check_launch("norm1_kernels");
}
}  // namespace tb

extern "C" int tcTensorNorm1(int data_kind, size_t vol, const void *src, double *result_dev,
                             void *scratch, size_t scratch_bytes, void *stream) {
  if (vol > 0 && src != nullptr && !elem_aligned(data_kind, src)) return TALSH_INVALID_ARGS;
  if (kind_size(data_kind) == 0 || result_dev == nullptr || (src == nullptr && vol > 0))
    return TALSH_INVALID_ARGS;
  if (vol == 0) return TALSH_INVALID_ARGS;
  if (scratch == nullptr || scratch_bytes < tcTensorNorm1Scratch(vol)) return TALSH_INVALID_ARGS;
  return norm1_launch(data_kind, vol, src, result_dev, (double *)scratch, (cudaStream_t)stream);
}
