// Split-precision R8 tensor contraction on the 5th-generation tensor cores.
//
// D = beta*D + alpha * sum_k A[m,k] B[k,n] in FP64 accuracy from exact int8
// products (the Ozaki scheme with integer slices):
//  1. L and R are permuted into row-major matrices A (M x K) and Bt (N x K)
//     by the transpose kernel (k fastest, the same k order on both sides).
//  2. Each row of A is scaled by a power of two 2^-e so that |x| < 1 and cut
//     into S slices of 7 bits: x = sum_s a_s 2^(-7 s) + r, a_s in [-127, 127],
//     |r| < 2^(-7 S).  Every step is exact in FP64 (scaling by 2^k, truncation
//     and subtraction of the truncated part).  Bt likewise per row (column of B).
//  3. For every anti-diagonal g = s + t (2 <= g <= S + 1) the products
//     P_g = sum_{s+t=g} A_s Bt_t^T are exact int8 x int8 -> int32 sums.  One
//     CTA keeps the S accumulators P_2 .. P_{S+1} of a 128 x 64 tile in tensor
//     memory (S x 64 columns) and issues tcgen05.mma kind::i8 for all slice
//     pairs of each 64-byte K block; shared-memory operands use the
//     no-swizzle K-major canonical layout (8-row x 16-byte core matrices).
//  4. The epilogue reads the accumulators (tcgen05.ld) and forms
//     C = 2^(e_m + f_n) * sum_g 2^(-7 g) P_g in FP64, then D = alpha*C (+ D).
// Slice pairs with s + t > S + 1 are dropped; with S = 6 the relative error
// against an FP64 contraction is about sqrt(K) * 2^-46 for random data.
// The int32 sums are exact while (S) * K * 127^2 < 2^31; longer contractions
// are split into K chunks that accumulate into D.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "common.h"
#include "device_once.h"
#include "split_complex.h"

namespace tb {
int contract_validate(int kind, const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                      int rrank, const int *rdims);
int permute_launch_o2n(int kind, int rank, const int *dims, const int *o2n, const void *src, void *dst,
                       cudaStream_t st);
size_t contract_tables_bytes(int64_t M, int64_t N, int64_t K);
int contract_build_tables(const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                          int rrank, const int *rdims, void *tables, cudaStream_t st, int64_t &M,
                          int64_t &N, int64_t &K, const int64_t **mD, const int64_t **nD);

namespace {

constexpr int kOzBM = 128;        // tile rows (m), the UMMA M
constexpr int kOzBN = 64;         // tile columns (n), the UMMA N
constexpr int kOzBK = 64;         // K bytes per stage (two UMMA K steps of 32)
constexpr int kOzThreads = 128;   // four warps: loads, MMA issue (thread 0), epilogue
constexpr int kOzStages = 2;
constexpr int kOzMaxSlices = 7;
constexpr uint32_t kSpinLimit = 1u << 22;  // bounded mbarrier waits (seconds at most)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: no swizzle, K-major.  Core matrices are
// 8 rows x 16 bytes (128 contiguous bytes); lbo = byte distance between the
// two 16-byte K halves of an MMA, sbo = byte distance between 8-row groups.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Shared-memory matrix descriptor, 32-byte swizzle, K-major: rows of 32 bytes
// (one UMMA K step of int8) as written by a TMA box of {32 bytes, rows} with
// CU_TENSOR_MAP_SWIZZLE_32B; 8-row groups 256 bytes apart.
__device__ __forceinline__ uint64_t make_desc_sw32(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46) |
         (6ull << 61);
}
// The same for CU_TENSOR_MAP_SWIZZLE_64B tiles (64-byte rows, 8-row groups
// 512 bytes apart).  A K step inside the 64-byte row starts 32 bytes further:
// the swizzle is a function of the absolute shared address, so advancing the
// start address selects the second half of every row.
__device__ __forceinline__ uint64_t make_desc_sw64(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46) |
         (4ull << 61);
}

// Instruction descriptor of kind::i8: int32 accumulator, signed A and B, both
// K-major, M = 128, N = 64.
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kOzBN >> 3) << 17) |
                              ((uint32_t)(kOzBM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescI8), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false (and the error flag set) when the phase never completes.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err,
                                          uint32_t limit = kSpinLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}

// Count of CTAs that gave up a bounded wait, per device (as the reference's
// gpu_error_count, tensor_algebra_gpu_nvidia.cu:189, counts kernel errors);
// read on the host by gpu_get_error_count.
__device__ int g_device_errors = 0;

// Marks the CTA aborted; the first marker counts the CTA in g_device_errors.
__device__ __forceinline__ void raise_abort(int *abort_flag) {
  if (atomicExch(abort_flag, 1) == 0) atomicAdd(&g_device_errors, 1);
}

__device__ __forceinline__ void cp16(uint32_t s, const void *g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g));
}

// Tiled slice layout (the one the warp-specialised GEMM reads): 128-row x
// 64-byte tiles, the S slices of one (row tile, K box) adjacent, and every
// tile stored as the shared-memory image of a 64-byte-swizzled load -- the
// 16-byte chunk c of tile row i sits at chunk c ^ ((i >> 1) & 3), the layout
// make_desc_sw64 describes.  One contiguous bulk copy then moves the slices of
// a box into a stage.  kb: byte offset in the row; nbox: 64-byte boxes per row.
__device__ __forceinline__ int64_t tiled_off(int64_t r, int64_t kb, int s, int S, int64_t nbox) {
  const int64_t tile = ((r >> 7) * nbox + (kb >> 6)) * S + s;
  const int i = (int)(r & 127);
  const int c = (int)((kb >> 4) & 3) ^ ((i >> 1) & 3);
  return tile * 8192 + i * 64 + c * 16 + (kb & 15);
}

// Row split: one CTA per (padded) row; 256 threads.
__global__ void __launch_bounds__(256) oz_split_rows(const double *__restrict__ X, int64_t rows,
                                                     int64_t K, int64_t rows_p, int64_t Kp, int S,
                                                     int8_t *__restrict__ slices, int32_t *expo, int tiled) {
  const int64_t r = blockIdx.x;
  const int tid = threadIdx.x;
  __shared__ double red[8];
  __shared__ int e_sh;
  const double *x = X + r * K;
  double mx = 0.0;
  if (r < rows)
    for (int64_t k = tid; k < K; k += 256) mx = fmax(mx, fabs(x[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0) red[tid >> 5] = mx;
  __syncthreads();
  if (tid == 0) {
    double m = 0.0;
    for (int w = 0; w < 8; ++w) m = fmax(m, red[w]);
    // m = f * 2^e with f in [0.5, 1): scaled entries lie in (-1, 1).
    e_sh = (m > 0.0) ? ilogb(m) + 1 : 0;
    expo[r] = e_sh;
  }
  __syncthreads();
  const int e = e_sh;
  const int64_t plane = rows_p * Kp;
  for (int64_t k = tid; k < Kp; k += 256) {
    double v = (r < rows && k < K) ? scalbn(x[k], -e) : 0.0;
    for (int s = 0; s < S; ++s) {
      const double y = v * 128.0;  // |y| < 128
      const double t = trunc(y);   // in [-127, 127]
      slices[tiled ? tiled_off(r, k, s, S, Kp >> 6) : s * plane + r * Kp + k] = (int8_t)(int)t;
      v = y - t;                   // exact remainder, |v| < 1
    }
  }
}

// ---------------------------------------------------------------------------
// Split forms.  The scheme above with the slices stored as int8 digits
// (kFormInt8, exact int32 accumulation) or as floating-point slices on the
// bf16, tf32 and e4m3 tensor-core kinds with fp32 accumulation:
//   x 2^-e = sum_s y_s 2^(-b s) + r,   y_s = round_X(r_s 2^(b s)),
//   r_{s+1} = r_s - y_s 2^(-b s)  (exact in FP64),
// b = the significant bits of X (bf16 8, tf32 11, e4m3 4).  The slice pairs
// with s + t <= S - 1 (0-based) are multiplied, each diagonal g = s + t in its
// own fp32 accumulator (every bf16/tf32/e4m3 product is exact in fp32; the
// accumulation rounds), and recombined in FP64 with weights 2^(-b g).  The
// error is that of the fp32 accumulation plus the dropped pairs (about
// 2^(-b S)), stated per result by the callers.
// ---------------------------------------------------------------------------
enum : int { kFormInt8 = 0, kFormBF16 = 1, kFormTF32 = 2, kFormFP8 = 3 };

__host__ __device__ constexpr int form_esize(int form) { return form == kFormTF32 ? 4 : (form == kFormBF16 ? 2 : 1); }
__host__ __device__ constexpr int form_bits(int form) {
  return form == kFormBF16 ? 8 : (form == kFormTF32 ? 11 : (form == kFormFP8 ? 4 : 7));
}

// Rounds a double of magnitude below about 2 to the slice type; returns the
// slice's storage bits and its exact value.
template <int FORM>
__device__ __forceinline__ uint32_t round_slice(double t, double &val) {
  if constexpr (FORM == kFormBF16) {
    const __nv_bfloat16 h = __float2bfloat16_rn((float)t);
    val = (double)__bfloat162float(h);
    return (uint32_t)__bfloat16_as_ushort(h);
  } else if constexpr (FORM == kFormTF32) {
    // round to 10 stored mantissa bits (ties away from zero); the tensor core
    // reads only the upper 19 bits of a tf32 operand, so the lower 13 are zero
    uint32_t u = __float_as_uint((float)t);
    u = (u + 0x1000u) & ~0x1FFFu;
    val = (double)__uint_as_float(u);
    return u;
  } else {
    const __nv_fp8_storage_t q = __nv_cvt_float_to_fp8((float)t, __NV_SATFINITE, __NV_E4M3);
    const __half_raw hr = __nv_cvt_fp8_to_halfraw(q, __NV_E4M3);
    val = (double)__half2float(__half(hr));
    return (uint32_t)q;
  }
}

// Row split into floating-point slices: one CTA per (padded) row; 256 threads.
// slices: [S][rows_p][Kp] elements of the form's type, or the tiled layout
// (tiled_off) when tiled != 0.
template <int FORM>
__global__ void __launch_bounds__(256) split_rows_float(const double *__restrict__ X, int64_t rows, int64_t K,
                                                        int64_t rows_p, int64_t Kp, int S,
                                                        unsigned char *__restrict__ slices, int32_t *expo,
                                                        int tiled) {
  constexpr int ES = form_esize(FORM);
  constexpr int B = form_bits(FORM);
  const int64_t r = blockIdx.x;
  const int tid = threadIdx.x;
  __shared__ double red[8];
  __shared__ int e_sh;
  const double *x = X + r * K;
  double mx = 0.0;
  if (r < rows)
    for (int64_t k = tid; k < K; k += 256) mx = fmax(mx, fabs(x[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0) red[tid >> 5] = mx;
  __syncthreads();
  if (tid == 0) {
    double m = 0.0;
    for (int w = 0; w < 8; ++w) m = fmax(m, red[w]);
    e_sh = (m > 0.0) ? ilogb(m) + 1 : 0;
    expo[r] = e_sh;
  }
  __syncthreads();
  const int e = e_sh;
  const int64_t plane = rows_p * Kp;
  for (int64_t k = tid; k < Kp; k += 256) {
    double v = (r < rows && k < K) ? scalbn(x[k], -e) : 0.0;  // |v| < 1
    for (int s = 0; s < S; ++s) {
      double y;
      const uint32_t bits = round_slice<FORM>(scalbn(v, B * s), y);
      unsigned char *dst = slices + (tiled ? tiled_off(r, k * ES, s, S, (Kp * ES) >> 6)
                                           : (s * plane + r * Kp + k) * ES);
      if constexpr (ES == 4) *reinterpret_cast<uint32_t *>(dst) = bits;
      else if constexpr (ES == 2) *reinterpret_cast<uint16_t *>(dst) = (uint16_t)bits;
      else *dst = (unsigned char)bits;
      v -= scalbn(y, -B * s);  // exact: y is v 2^(B s) rounded to fewer bits
    }
  }
}

struct OzArgs {
  const int8_t *A;   // [S][Mp][Kp]
  const int8_t *B;   // [S][Np][Kp]
  int64_t Mp, Np, Kp;
  int64_t kb0, kb1;  // K-block range [kb0, kb1) of this launch (64-byte blocks)
  int S;
  const int32_t *ea, *eb;
  double *D;
  const int64_t *mD, *nD;
  int64_t M, N;
  double alpha;
  int beta;
  int *err;
  uint32_t tmem_cols;  // S x 64 columns of int32 accumulators, rounded up to a power of two
};

// Shared layout of one stage: S A-tiles (128 rows x 64 B) then S B-tiles (64 rows x 64 B),
// each in the canonical K-major layout: offset(row, c) = c*(rows*16) + (row/8)*128 + (row%8)*16
// for the 16-byte chunk c in 0..3.
constexpr int kATileBytes = kOzBM * kOzBK;
constexpr int kBTileBytes = kOzBN * kOzBK;

__global__ void __launch_bounds__(kOzThreads, 1) oz_gemm_kernel(const OzArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar[kOzStages];
  __shared__ uint32_t tmem_base_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = a.S;
  const int stage_bytes = S * (kATileBytes + kBTileBytes);
  const int64_t tm = blockIdx.x, tn = blockIdx.y;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_sh)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < kOzStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t tmem = tmem_base_sh;
  const uint32_t sbase = smem_u32(smem);

  auto load_stage = [&](int st, int64_t kb) {
    const uint32_t sst = sbase + (uint32_t)(st * stage_bytes);
    for (int s = 0; s < S; ++s) {
      const int8_t *ga = a.A + (int64_t)s * a.Mp * a.Kp + (tm * kOzBM) * a.Kp + kb * kOzBK;
      const uint32_t sa = sst + (uint32_t)(s * kATileBytes);
      for (int i = tid; i < kOzBM * 4; i += kOzThreads) {  // 128 rows x 4 chunks
        const int row = i >> 2, c = i & 3;
        cp16(sa + c * (kOzBM * 16) + (row >> 3) * 128 + (row & 7) * 16, ga + (int64_t)row * a.Kp + c * 16);
      }
      const int8_t *gb = a.B + (int64_t)s * a.Np * a.Kp + (tn * kOzBN) * a.Kp + kb * kOzBK;
      const uint32_t sb = sst + (uint32_t)(S * kATileBytes + s * kBTileBytes);
      for (int i = tid; i < kOzBN * 4; i += kOzThreads) {  // 64 rows x 4 chunks
        const int row = i >> 2, c = i & 3;
        cp16(sb + c * (kOzBN * 16) + (row >> 3) * 128 + (row & 7) * 16, gb + (int64_t)row * a.Kp + c * 16);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };

  const int64_t nkb = a.kb1 - a.kb0;
  bool ok = true;
  load_stage(0, a.kb0);
  for (int64_t it = 0; it < nkb; ++it) {
    const int st = (int)(it & 1);
    if (it + 1 < nkb) {
      // The other stage was read by the MMAs of iteration it - 1.
      if (it >= 1 && ok) ok = mbar_wait(&mbar[st ^ 1], (uint32_t)(((it - 1) >> 1) & 1), a.err);
      load_stage(st ^ 1, a.kb0 + it + 1);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0 && ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::);
      const uint32_t sst = sbase + (uint32_t)(st * stage_bytes);
      for (int g = 2; g <= S + 1; ++g) {
        const uint32_t dcol = tmem + (uint32_t)((g - 2) * kOzBN);
        for (int s = 1; s < g; ++s) {
          const int t = g - s;
          const uint32_t sa = sst + (uint32_t)((s - 1) * kATileBytes);
          const uint32_t sb = sst + (uint32_t)(S * kATileBytes + (t - 1) * kBTileBytes);
#pragma unroll
          for (int j = 0; j < 2; ++j) {  // two K steps of 32 bytes: chunks 2j, 2j+1
            const uint64_t ad = make_desc(sa + j * 2 * (kOzBM * 16), kOzBM * 16, 128);
            const uint64_t bd = make_desc(sb + j * 2 * (kOzBN * 16), kOzBN * 16, 128);
            mma_i8(dcol, ad, bd, (it > 0 || s > 1 || j > 0) ? 1u : 0u);
          }
        }
      }
      mma_commit(&mbar[st]);
    }
  }
  // All MMAs are done once the last commit has arrived (completion is in order).
  if (nkb > 0 && ok) ok = mbar_wait(&mbar[(nkb - 1) & 1], (uint32_t)(((nkb - 1) >> 1) & 1), a.err);
  ok = __syncthreads_and(ok) != 0;  // block-uniform: tcgen05.ld below is warp-collective
  asm volatile("tcgen05.fence::after_thread_sync;" ::);

  if (ok) {
    // Epilogue: warp w owns TMEM lanes (tile rows) 32w .. 32w + 31.
    const int64_t m = tm * kOzBM + warp * 32 + lane;
    const bool mrow = m < a.M;
    const int em = mrow ? a.ea[m] : 0;
    const int64_t dm = mrow ? a.mD[m] : 0;
    for (int c = 0; c < kOzBN / 16; ++c) {
      double acc[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[i] = 0.0;
      for (int g = 2; g <= S + 1; ++g) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((g - 2) * kOzBN + c * 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
              "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
              "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const double w = scalbn(1.0, -7 * g);
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[i] += (double)(int32_t)v[i] * w;
      }
      if (mrow) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int64_t n = tn * kOzBN + c * 16 + i;
          if (n < a.N) {
            double *p = a.D + dm + a.nD[n];
            const double val = a.alpha * scalbn(acc[i], em + a.eb[n]);
            *p = a.beta ? (*p + val) : val;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
}

// ---------------------------------------------------------------------------
// Warp-specialised mainloop (single CTA per 128 x 128 tile).  Warp 0: one
// thread fills each stage with bulk copies of the tiled slice layout (64-byte
// x 128-row swizzled tiles: two UMMA K steps per box, the slices of a box
// adjacent, one copy per operand and box).  Warp 1: one thread issues the MMAs
// of a stage once its copies have landed and commits them to the stage's
// "empty" barrier; warp 1 also owns the tensor memory.  Warps 2-5: epilogue,
// TMEM lane quadrant (warp % 4).  The pair kernel further down reads the same
// boxes through 2-D tensor maps over the plain slice layout.
// ---------------------------------------------------------------------------
constexpr int kOzWsThreads = 192;
constexpr int kWsBK = 32;                    // K bytes of one UMMA K step
constexpr int kWsBox = 64;                   // K bytes per TMA box row: two UMMA K steps
constexpr int kWsATile = kOzBM * kWsBox;     // 8 KB
constexpr int kWsGroupM = 4;                 // m tiles per raster group (L2 reuse of A and B)

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t sdst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          sdst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Contiguous global -> shared bulk copy completing on an mbarrier (16-byte
// aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_load(uint32_t sdst, const void *gsrc, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(sdst),
      "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

struct OzWsArgs {
  const unsigned char *At, *Bt;  // tiled slices (tiled_off)
  int64_t nbox;                  // 64-byte K boxes per slice row
  uint32_t spin_limit;  // iterations of every bounded mbarrier wait
  int stall_test;       // 1: the producer issues no copies, so the MMA warp's first wait runs out
  int64_t Mp, Np;
  int tiles_m, tiles_n;
  int group_m;  // m tiles per raster group
  int64_t kb0, kb1;
  int S, nst;
  const int32_t *ea, *eb;
  double *D;
  const int64_t *mD, *nD;
  int64_t M, N;
  double alpha;
  int beta;
  int *err;
  uint32_t tmem_cols;
};

constexpr int kWsBN = 128;                    // tile columns of the pass kernel (UMMA N)
constexpr int kWsBTile128 = kWsBN * kWsBox;   // 8 KB
constexpr int kWsDiagPerPass = 3;             // accumulators per pass: 3 x 128 TMEM columns
// Instruction descriptors, M = 128, N = 128, K-major A and B: accumulator
// format (bits 4-5: 1 F32, 2 S32), A/B formats (bits 7-9, 10-12: signed int8
// 1; bf16 1 and tf32 2 of kind::f16/tf32; e4m3 0 of kind::f8f6f4).
constexpr uint32_t kIdescMN128 = ((uint32_t)(kWsBN >> 3) << 17) | ((uint32_t)(kOzBM >> 4) << 24);
// M = 256 (a CTA pair, cta_group::2), N = 256.
constexpr uint32_t kIdescPair = ((uint32_t)(256 >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);
template <int FORM> struct FormMma;
template <> struct FormMma<kFormInt8> {
  static constexpr uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | kIdescMN128;
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
  }
  static constexpr uint32_t idesc_pair = (2u << 4) | (1u << 7) | (1u << 10) | kIdescPair;
  __device__ static void mma_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc_pair), "r"(acc));
  }
};
template <> struct FormMma<kFormBF16> {
  static constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | kIdescMN128;
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
  }
  static constexpr uint32_t idesc_pair = (1u << 4) | (1u << 7) | (1u << 10) | kIdescPair;
  __device__ static void mma_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc_pair), "r"(acc));
  }
};
template <> struct FormMma<kFormTF32> {
  static constexpr uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | kIdescMN128;
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
  }
  static constexpr uint32_t idesc_pair = (1u << 4) | (2u << 7) | (2u << 10) | kIdescPair;
  __device__ static void mma_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc_pair), "r"(acc));
  }
};
template <> struct FormMma<kFormFP8> {
  static constexpr uint32_t idesc = (1u << 4) | (0u << 7) | (0u << 10) | kIdescMN128;
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
  }
  static constexpr uint32_t idesc_pair = (1u << 4) | (0u << 7) | (0u << 10) | kIdescPair;
  __device__ static void mma_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc_pair), "r"(acc));
  }
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 128 x 128 output tile.  The anti-diagonals g = 2 .. S+1 are processed in
// passes of up to three (3 x 128 int32 TMEM columns); pass p streams K once,
// with only the slices its diagonals use, and its epilogue adds the pass's
// contribution into D before the next pass reuses the accumulators.
template <int FORM>
__global__ void __launch_bounds__(kOzWsThreads, 1)
    oz_gemm_ws_kernel(const OzWsArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr int kMaxStages = 8;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], done, drained;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = a.S, nst = a.nst;
  const int slot_bytes = S * (kWsATile + kWsBTile128);  // a stage slot holds the largest pass
  const int npass = (S + kWsDiagPerPass - 1) / kWsDiagPerPass;
  int tm, tn;
  {
    const int id = blockIdx.x;
    const int per_group = a.group_m * a.tiles_n;
    const int grp = id / per_group;
    const int first_m = grp * a.group_m;
    const int gm = min(a.group_m, a.tiles_m - first_m);
    const int r = id - grp * per_group;
    tm = first_m + r % gm;
    tn = r / gm;
  }
  const int64_t nkb = a.kb1 - a.kb0;      // UMMA K steps of this launch
  const int64_t nbox = (nkb + 1) / 2;      // 64-byte TMA boxes covering them
  auto pass_g0 = [&](int p) { return 2 + p * kWsDiagPerPass; };
  auto pass_g1 = [&](int p) { return min(S + 1, pass_g0(p) + kWsDiagPerPass - 1); };

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_sh)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < nst; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&done, 1);
    mbar_init(&drained, 128);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t tmem = tmem_base_sh;
  const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;  // swizzled tiles need aligned bases

  const uint32_t lim = a.spin_limit;
  int64_t issued_all = 0;  // warp 0 lane 0: stage-ring iterations whose copies were issued
  if (warp == 0) {
    if (lane == 0) {
      int64_t itg = 0;     // stage-ring iteration across passes
      int64_t issued = 0;  // iterations whose copies were issued
      for (int p = 0; p < npass && !*(volatile int *)&abort_sh && !a.stall_test; ++p) {
        const int smax = pass_g1(p) - 1;
        const int kper = max(1, S / smax);  // boxes per slice and stage: early passes need fewer slices
        for (int64_t it = 0; it < nbox; it += kper, ++itg) {
          const int nk = (int)min((int64_t)kper, nbox - it);
          const int st = (int)(itg % nst);
          if (itg >= nst && !mbar_wait(&empty[st], (uint32_t)(((itg / nst) - 1) & 1), a.err, lim)) {
            raise_abort(&abort_sh);
            break;
          }
          if (*(volatile int *)&abort_sh) break;
          issued = itg + 1;
          mbar_expect_tx(&full[st], (uint32_t)(nk * smax * (kWsATile + kWsBTile128)));
          const uint32_t sst = sbase + (uint32_t)(st * slot_bytes);
          for (int j = 0; j < nk; ++j) {
            // slices 0 .. smax-1 of box (tm or tn, kb0/2 + it + j) are adjacent
            const int64_t box = a.kb0 / 2 + it + j;
            const uint32_t bytes = (uint32_t)(smax * kWsATile);
            bulk_load(sst + (uint32_t)(j * smax * kWsATile),
                      a.At + ((int64_t)tm * a.nbox + box) * S * kWsATile, bytes, &full[st]);
            bulk_load(sst + (uint32_t)(S * kWsATile + j * smax * kWsBTile128),
                      a.Bt + ((int64_t)tn * a.nbox + box) * S * kWsBTile128, bytes, &full[st]);
          }
        }
      }
      issued_all = issued;
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int64_t itg = 0;
      for (int p = 0; p < npass; ++p) {
        if (p > 0 && !mbar_wait(&drained, (uint32_t)((p - 1) & 1), a.err, lim)) raise_abort(&abort_sh);
        if (*(volatile int *)&abort_sh) {
          mma_commit(&done);
          continue;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::);
        const int g0 = pass_g0(p), g1 = pass_g1(p);
        const int smax = g1 - 1;
        const int kper = max(1, S / smax);
        for (int64_t it = 0; it < nbox; it += kper, ++itg) {
          const int nk = (int)min((int64_t)kper, nbox - it);
          const int st = (int)(itg % nst);
          if (!mbar_wait(&full[st], (uint32_t)((itg / nst) & 1), a.err, lim)) {
            raise_abort(&abort_sh);
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::);
          const uint32_t sst = sbase + (uint32_t)(st * slot_bytes);
          for (int j = 0; j < nk; ++j) {
            // the two K steps of the box; the second lies past this launch's
            // K range when the range has an odd number of steps
            const int nsteps = (2 * (it + j) + 1 < nkb) ? 2 : 1;
            for (int kk = 0; kk < nsteps; ++kk) {
              for (int g = g0; g <= g1; ++g) {
                const uint32_t dcol = tmem + (uint32_t)((g - g0) * kWsBN);
                for (int s1 = 1; s1 < g; ++s1) {
                  const uint32_t sa = sst + (uint32_t)((j * smax + s1 - 1) * kWsATile + kk * kWsBK);
                  const uint32_t sb =
                      sst + (uint32_t)(S * kWsATile + (j * smax + g - s1 - 1) * kWsBTile128 + kk * kWsBK);
                  FormMma<FORM>::mma(dcol, make_desc_sw64(sa), make_desc_sw64(sb),
                                     (it > 0 || j > 0 || kk > 0 || s1 > 1) ? 1u : 0u);
                }
              }
            }
          }
          mma_commit(&empty[st]);
        }
        mma_commit(&done);  // this pass's accumulators are complete
      }
    }
  } else {
    const int q = warp & 3;
    const int64_t m = (int64_t)tm * kOzBM + q * 32 + lane;
    const bool mrow = m < a.M;
    const int em = mrow ? a.ea[m] : 0;
    const int64_t dm = mrow ? a.mD[m] : 0;
    for (int p = 0; p < npass; ++p) {
      bool ok = mbar_wait(&done, (uint32_t)(p & 1), a.err, lim);
      if (!ok) raise_abort(&abort_sh);
      ok = ok && !*(volatile int *)&abort_sh;
      ok = __all_sync(0xffffffffu, ok);
      asm volatile("tcgen05.fence::after_thread_sync;" ::);
      const int g0 = pass_g0(p), g1 = pass_g1(p);
      const bool first = (p == 0);
      if (ok) {
        const bool rd = !(first && !a.beta);  // D is read (accumulated into) in this pass
        for (int c = 0; c < kWsBN / 16; ++c) {
          // The chunk's D addresses and old values first: the 16 loads are in
          // flight together while the accumulators are read from tensor memory.
          double *ptr[16];
          double old[16];
          int esc[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int64_t n = (int64_t)tn * kWsBN + c * 16 + i;
            const bool ok = mrow && n < a.N;
            ptr[i] = ok ? a.D + dm + a.nD[n] : nullptr;
            esc[i] = ok ? em + a.eb[n] : 0;
          }
#pragma unroll
          for (int i = 0; i < 16; ++i) old[i] = (rd && ptr[i] != nullptr) ? *ptr[i] : 0.0;
          double acc[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = 0.0;
          for (int g = g0; g <= g1; ++g) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((g - g0) * kWsBN + c * 16);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                  "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            // diagonal weights: int8 digits 2^(-7 g) (1-based slices); float
            // slices 2^(-b (g - 2))
            if constexpr (FORM == kFormInt8) {
              const double w = scalbn(1.0, -7 * g);
#pragma unroll
              for (int i = 0; i < 16; ++i) acc[i] += (double)(int32_t)v[i] * w;
            } else {
              const double w = scalbn(1.0, -form_bits(FORM) * (g - 2));
#pragma unroll
              for (int i = 0; i < 16; ++i) acc[i] += (double)__uint_as_float(v[i]) * w;
            }
          }
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            if (ptr[i] == nullptr) continue;
            const double val = a.alpha * scalbn(acc[i], esc[i]);
            *ptr[i] = rd ? old[i] + val : val;
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::);
      mbar_arrive(&drained);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
  // After an abort (final once every warp has passed the barrier above), wait
  // (bounded) until the copies of the last iteration issued into each stage
  // have landed, so that none is in flight when the CTA exits.
  if (warp == 0 && lane == 0 && *(volatile int *)&abort_sh) {
    for (int st = 0; st < nst; ++st) {
      if (issued_all <= st) continue;
      const int64_t last = st + ((issued_all - 1 - st) / nst) * nst;
      mbar_wait(&full[st], (uint32_t)((last / nst) & 1), a.err, lim);
    }
  }
}

// ---------------------------------------------------------------------------
// Pair (cta_group::2) form of the warp-specialised GEMM.  Two CTAs of a
// cluster compute one 256 x 256 tile: each holds 128 rows of A and 128 rows
// of B per slice in its shared memory, and the even CTA issues MMAs of
// M = 256, N = 256 that read both CTAs' operands (each SM multiplies its own
// A rows by all of B; the B halves are exchanged between the pair), so one
// instruction does four times the work of the single-CTA form's 128 x 128.
// Every SM keeps its own rows' accumulators in its tensor memory: 2
// diagonals x 256 columns per pass, three passes for six slices.
// Synchronisation: both CTAs' copies complete on the even CTA's "full"
// barriers (the copies carry .cta_group::2); the even CTA's commits arrive on
// "empty" and "done" in both CTAs (.multicast::cluster on tcgen05.commit);
// both CTAs' epilogue threads arrive on the even CTA's "drained" barrier.
// Every wait on an mbarrier is bounded; the two cluster barriers (after the
// barrier set-up and before the tensor memory is freed) are reached by every
// thread on every path.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Shared::cluster address of the same shared variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t mapa_rank(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
// 2-D tensor copy whose completion is counted on the even CTA's barrier
// (`bar_cluster`, a shared::cluster address); no multicast.
__device__ __forceinline__ void tma_load_2d_pair(uint32_t sdst, const CUtensorMap *map, int x, int y,
                                                 uint32_t bar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(sdst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar_cluster)
      : "memory");
}
// Arrival on `bar` (same shared offset) in both CTAs of the pair once every
// previously issued MMA of this thread has completed.
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((uint16_t)3)
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}
// Waits with cluster-scope acquire (the phase may be completed by the peer CTA).
__device__ __forceinline__ bool mbar_try_cluster(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t *bar, uint32_t parity, int *err, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_cluster(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}

constexpr int kPairBN = 256;                 // tile columns of the pair (UMMA N)
constexpr int kPairDiag = 2;                 // accumulators per pass: 2 x 256 TMEM columns
constexpr int kPairBTile = 128 * kWsBox;     // 8 KB: this CTA's 128 rows of a B slice box

struct OzPairArgs {
  uint32_t spin_limit;
  int64_t Mp, Np;
  int tiles_m2, tiles_n;  // 256-row and 128-column tiles
  int group_m;            // pair tiles along m per raster group
  int64_t kb0, kb1;
  int S, nst;
  const int32_t *ea, *eb;
  double *D;
  const int64_t *mD, *nD;
  int64_t M, N;
  double alpha;
  int beta;
  int *err;
  uint32_t tmem_cols;
};

template <int FORM>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kOzWsThreads, 1)
    oz_gemm_pair_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                        const OzPairArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr int kMaxStages = 8;
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], done, drained;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_ctarank();
  const int S = a.S, nst = a.nst;
  const int slot_bytes = S * (kWsATile + kPairBTile);
  const int npass = (S + kPairDiag - 1) / kPairDiag;
  int tm, tn;  // 256-row tile of the pair, 128-column tile
  {
    const int id = blockIdx.x >> 1;
    const int per_group = a.group_m * a.tiles_n;
    const int grp = id / per_group;
    const int first_m = grp * a.group_m;
    const int gm = min(a.group_m, a.tiles_m2 - first_m);
    const int r = id - grp * per_group;
    tm = first_m + r % gm;
    tn = r / gm;
  }
  const int64_t nkb = a.kb1 - a.kb0;
  const int64_t nbox = (nkb + 1) / 2;
  auto pass_g0 = [&](int p) { return 2 + p * kPairDiag; };
  auto pass_g1 = [&](int p) { return min(S + 1, pass_g0(p) + kPairDiag - 1); };

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int i = 0; i < nst; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&done, 1);
    mbar_init(&drained, 256);  // both CTAs' epilogue threads
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::);
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&mapA) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&mapB) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  cluster_sync_all();  // the even CTA's barriers exist before the odd CTA signals them
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  const uint32_t tmem = tmem_base_sh;
  const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;
  const uint32_t lim = a.spin_limit;

  int64_t issued_all = 0;  // warp 0 lane 0: stage-ring iterations whose copies were issued
  if (warp == 0) {
    if (lane == 0) {
      int64_t itg = 0;
      for (int p = 0; p < npass && !*(volatile int *)&abort_sh; ++p) {
        const int smax = pass_g1(p) - 1;
        const int kper = max(1, S / smax);
        for (int64_t it = 0; it < nbox; it += kper, ++itg) {
          const int nk = (int)min((int64_t)kper, nbox - it);
          const int st = (int)(itg % nst);
          if (itg >= nst && !mbar_wait_cluster(&empty[st], (uint32_t)(((itg / nst) - 1) & 1), a.err, lim)) {
            raise_abort(&abort_sh);
            break;
          }
          issued_all = itg + 1;
          // the even CTA expects the bytes of both CTAs' copies of this stage
          if (rank == 0) mbar_expect_tx(&full[st], (uint32_t)(2 * nk * smax * (kWsATile + kPairBTile)));
          const uint32_t fbar = mapa_rank(smem_u32(&full[st]), 0);
          const uint32_t sst = sbase + (uint32_t)(st * slot_bytes);
          for (int j = 0; j < nk; ++j) {
            const int kx = (int)((a.kb0 + 2 * (it + j)) * kWsBK);
            for (int s = 0; s < smax; ++s) {
              const uint32_t sa = sst + (uint32_t)((j * smax + s) * kWsATile);
              const uint32_t sb = sst + (uint32_t)(S * kWsATile + (j * smax + s) * kPairBTile);
              tma_load_2d_pair(sa, &mapA, kx, (int)(s * a.Mp + tm * 256 + rank * 128), fbar);
              tma_load_2d_pair(sb, &mapB, kx, (int)(s * a.Np + tn * kPairBN + rank * 128), fbar);
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    if (rank == 0 && lane == 0) {
      int64_t itg = 0;
      for (int p = 0; p < npass; ++p) {
        if (p > 0 && !mbar_wait_cluster(&drained, (uint32_t)((p - 1) & 1), a.err, lim)) raise_abort(&abort_sh);
        if (*(volatile int *)&abort_sh) {
          mma_commit_pair(&done);
          continue;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::);
        const int g0 = pass_g0(p), g1 = pass_g1(p);
        const int smax = g1 - 1;
        const int kper = max(1, S / smax);
        for (int64_t it = 0; it < nbox; it += kper, ++itg) {
          const int nk = (int)min((int64_t)kper, nbox - it);
          const int st = (int)(itg % nst);
          if (!mbar_wait_cluster(&full[st], (uint32_t)((itg / nst) & 1), a.err, lim)) {
            raise_abort(&abort_sh);
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::);
          const uint32_t sst = sbase + (uint32_t)(st * slot_bytes);
          for (int j = 0; j < nk; ++j) {
            const int nsteps = (2 * (it + j) + 1 < nkb) ? 2 : 1;
            for (int kk = 0; kk < nsteps; ++kk) {
              for (int g = g0; g <= g1; ++g) {
                const uint32_t dcol = tmem + (uint32_t)((g - g0) * kPairBN);
                for (int s1 = 1; s1 < g; ++s1) {
                  const uint32_t sa = sst + (uint32_t)((j * smax + s1 - 1) * kWsATile + kk * kWsBK);
                  const uint32_t sb =
                      sst + (uint32_t)(S * kWsATile + (j * smax + g - s1 - 1) * kPairBTile + kk * kWsBK);
                  FormMma<FORM>::mma_pair(dcol, make_desc_sw64(sa), make_desc_sw64(sb),
                                          (it > 0 || j > 0 || kk > 0 || s1 > 1) ? 1u : 0u);
                }
              }
            }
          }
          mma_commit_pair(&empty[st]);
        }
        mma_commit_pair(&done);
      }
    }
  } else {
    const int q = warp & 3;
    const int64_t m = (int64_t)tm * 256 + rank * 128 + q * 32 + lane;
    const bool mrow = m < a.M;
    const int em = mrow ? a.ea[m] : 0;
    const int64_t dm = mrow ? a.mD[m] : 0;
    const uint32_t drained0 = mapa_rank(smem_u32(&drained), 0);
    for (int p = 0; p < npass; ++p) {
      bool ok = mbar_wait_cluster(&done, (uint32_t)(p & 1), a.err, lim);
      if (!ok) raise_abort(&abort_sh);
      ok = ok && !*(volatile int *)&abort_sh;
      ok = __all_sync(0xffffffffu, ok);
      asm volatile("tcgen05.fence::after_thread_sync;" ::);
      const int g0 = pass_g0(p), g1 = pass_g1(p);
      const bool first = (p == 0);
      if (ok) {
        const bool rd = !(first && !a.beta);
        for (int c = 0; c < kPairBN / 16; ++c) {
          double *ptr[16];
          double old[16];
          int esc[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int64_t n = (int64_t)tn * kPairBN + c * 16 + i;
            const bool okn = mrow && n < a.N;
            ptr[i] = okn ? a.D + dm + a.nD[n] : nullptr;
            esc[i] = okn ? em + a.eb[n] : 0;
          }
#pragma unroll
          for (int i = 0; i < 16; ++i) old[i] = (rd && ptr[i] != nullptr) ? *ptr[i] : 0.0;
          double acc[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[i] = 0.0;
          for (int g = g0; g <= g1; ++g) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((g - g0) * kPairBN + c * 16);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                  "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                  "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if constexpr (FORM == kFormInt8) {
              const double w = scalbn(1.0, -7 * g);
#pragma unroll
              for (int i = 0; i < 16; ++i) acc[i] += (double)(int32_t)v[i] * w;
            } else {
              const double w = scalbn(1.0, -form_bits(FORM) * (g - 2));
#pragma unroll
              for (int i = 0; i < 16; ++i) acc[i] += (double)__uint_as_float(v[i]) * w;
            }
          }
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            if (ptr[i] == nullptr) continue;
            const double val = a.alpha * scalbn(acc[i], esc[i]);
            *ptr[i] = rd ? old[i] + val : val;
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::);
      mbar_arrive_cluster(drained0);  // the pass's accumulators of this CTA have been read
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::);
  __syncthreads();
  // After an abort, the even CTA waits (bounded) for the last phase of every
  // stage it expected, so that no copy of the pair is in flight at exit.
  if (rank == 0 && warp == 0 && lane == 0 && *(volatile int *)&abort_sh) {
    for (int st = 0; st < nst; ++st) {
      if (issued_all <= st) continue;
      const int64_t last = st + ((issued_all - 1 - st) / nst) * nst;
      mbar_wait_cluster(&full[st], (uint32_t)((last / nst) & 1), a.err, lim);
    }
  }
  cluster_sync_all();  // no MMA, copy or arrival of the pair is outstanding
  asm volatile("tcgen05.fence::after_thread_sync;" ::);
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
    cudaGetLastError();
  });
  return fn;
}

// 2-D map over a [rows][Kp] int8 matrix, box 32 bytes (one UMMA K step) x
// box_rows, 64-byte swizzle (the layout make_desc_sw64 describes).
bool make_slice_map(CUtensorMap *map, const void *base, int64_t Kp, int64_t rows, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (fn == nullptr) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp};
  const cuuint32_t box[2] = {(cuuint32_t)kWsBox, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

constexpr int kOzWsSmem = 208 * 1024;  // dynamic shared bytes for the stage ring (+1 KB alignment slack)

// m tiles per raster group of the warp-specialised kernel: kWsGroupM, or
// TALSH_B200_SPLIT_GROUP_M (1..64) for tuning.
int ws_group_m() {
  static const int v = [] {
    const char *e = std::getenv("TALSH_B200_SPLIT_GROUP_M");
    const int g = e ? std::atoi(e) : 0;
    return (g >= 1 && g <= 64) ? g : kWsGroupM;
  }();
  return v;
}

// TALSH_B200_SPLIT_SIMPLE=1 selects the single-loop kernel (for tests).
bool oz_force_simple() {
  static const bool v = [] {
    const char *e = std::getenv("TALSH_B200_SPLIT_SIMPLE");
    return e && std::atoi(e) == 1;
  }();
  return v;
}

struct OzPlan {
  int64_t M, N, K, Mp, Np, Kp;
  size_t off_A64, off_B64, off_As, off_Bs, off_ea, off_eb, off_tab, off_err, total;
};

// esize: bytes per slice element; Kp (elements) makes every slice row a whole
// number of 64-byte blocks.
void oz_plan(int64_t M, int64_t N, int64_t K, int S, OzPlan &p, int esize = 1) {
  p.M = M; p.N = N; p.K = K;
  p.Mp = round_up(std::max<int64_t>(M, 1), 2 * kOzBM);  // whole 256-row tiles of the CTA-pair kernel
  p.Np = round_up(std::max<int64_t>(N, 1), 256);  // whole tiles of every kernel (the pair's are 256 wide)
  p.Kp = round_up(std::max<int64_t>(K, 1), kOzBK / esize);
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 255) & ~size_t(255); return o; };
  p.off_A64 = take((size_t)M * K * 8);
  p.off_B64 = take((size_t)N * K * 8);
  p.off_As = take((size_t)S * p.Mp * p.Kp * esize);
  p.off_Bs = take((size_t)S * p.Np * p.Kp * esize);
  p.off_ea = take((size_t)p.Mp * 4);
  p.off_eb = take((size_t)p.Np * 4);
  p.off_tab = take(contract_tables_bytes(M, N, K));
  p.off_err = take(16);
  p.total = off;
}

// O2N of an operand into (k..., own uncontracted..., unit dims...), k in the
// shared order (R's order when R leads with a contracted index and L does not
// or R is larger, else L's -- the order the tables use as well).
void operand_o2n(const int *cptrn, int lrank, const int *ldims, int rrank, const int *rdims,
                 bool left, int *o2n) {
  int64_t lvol = 1, rvol = 1;
  for (int i = 0; i < lrank; ++i) lvol *= ldims[i];
  for (int i = 0; i < rrank; ++i) rvol *= rdims[i];
  const bool l_lead_k = lrank > 0 && cptrn[0] < 0;
  const bool r_lead_k = rrank > 0 && cptrn[lrank] < 0;
  const bool k_in_r_order = r_lead_k && (!l_lead_k || rvol > lvol);
  const int rank = left ? lrank : rrank;
  const int *dims = left ? ldims : rdims;
  const int *pat = left ? cptrn : cptrn + lrank;
  int kpos[kMaxRank];
  for (int i = 0; i < rank; ++i) kpos[i] = -1;
  int nk = 0;
  if (k_in_r_order) {
    for (int j = 0; j < rrank; ++j) {
      const int v = cptrn[lrank + j];
      if (v < 0 && rdims[j] > 1) {
        const int li = -v - 1;
        kpos[left ? li : j] = nk++;
      }
    }
  } else {
    for (int i = 0; i < lrank; ++i) {
      const int v = cptrn[i];
      if (v < 0 && ldims[i] > 1) {
        const int rj = -v - 1;
        kpos[left ? i : rj] = nk++;
      }
    }
  }
  int pos = nk;
  for (int i = 0; i < rank; ++i)
    if (pat[i] > 0 && dims[i] > 1) o2n[i] = ++pos;
  for (int i = 0; i < rank; ++i) {
    if (kpos[i] >= 0) o2n[i] = kpos[i] + 1;
    else if (dims[i] <= 1) o2n[i] = ++pos;
  }
}

}  // namespace

namespace {

bool has_hyper_index(const int *cptrn, int lrank, int rrank) {
  for (int i = 0; i < lrank; ++i)
    for (int j = 0; cptrn[i] > 0 && j < rrank; ++j)
      if (cptrn[lrank + j] == cptrn[i]) return true;
  return false;
}

}  // namespace

// A split-form code: the slice count in bits 0-3 (0: the form's default, 6
// int8 digits or 3 floating-point slices), the form in bits 4-7 (kFormInt8,
// kFormBF16, kFormTF32, kFormFP8).  A plain slice count 2..7 is the int8 form.
struct FormCode {
  int form = kFormInt8, S = 6;
};
bool decode_form(int code, FormCode &f) {
  if (code < 0) return false;
  f.form = (code >> 4) & 15;
  f.S = code & 15;
  if (f.form > kFormFP8 || (code >> 8) != 0) return false;
  if (f.S == 0) f.S = (f.form == kFormInt8) ? 6 : 3;
  return f.S >= 2 && f.S <= kOzMaxSlices;
}

// Failure-detection test hook (tcTestSplitStall): the next split GEMM
// launches issue no copies and give up their first wait after 4096 polls.
std::atomic<int> g_stall_test{0};

// K elements per launch of a floating-point form (fp32 accumulation over at
// most this many products per diagonal before the FP64 sum into D): 0 = all of
// K; TALSH_B200_SPLIT_FP32_KCHUNK for tuning.
int64_t fp32_kchunk() {
  static const int64_t v = [] {
    const char *e = std::getenv("TALSH_B200_SPLIT_FP32_KCHUNK");
    const long long c = e ? std::atoll(e) : 0;
    return (int64_t)(c > 0 ? c : 0);
  }();
  return v;
}

// 0 when the form does not apply: not R8, an operand of rank 0, an invalid
// pattern or hyper-indices.
size_t contract_split_scratch(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                              const int *ldims, int rrank, const int *rdims, int slices) {
  if (kind != R8 || lrank == 0 || rrank == 0 || drank == 0) return 0;
  if (contract_validate(R8, cptrn, drank, ddims, lrank, ldims, rrank, rdims) != TALSH_SUCCESS) return 0;
  if (has_hyper_index(cptrn, lrank, rrank)) return 0;
  int64_t M = 1, N = 1, K = 1;
  for (int i = 0; i < lrank; ++i) (cptrn[i] > 0 ? M : K) *= ldims[i];
  for (int i = 0; i < rrank; ++i)
    if (cptrn[lrank + i] > 0) N *= rdims[i];
  FormCode fc;
  if (!decode_form(slices, fc)) return 0;
  OzPlan p;
  oz_plan(M, N, K, fc.S, p, form_esize(fc.form));
  return p.total;
}

namespace {

// Which GEMM runs: the CTA-pair kernel (256 x 256 tiles) when its tiles give
// every SM work (two CTAs per tile), else the single-CTA kernel (128 x 128
// tiles, four times as many); TALSH_B200_SPLIT_PAIR=1 / 0 forces one.
int split_pair_mode() {
  static const int v = [] {
    const char *e = std::getenv("TALSH_B200_SPLIT_PAIR");
    return e ? (std::atoi(e) != 0 ? 1 : 0) : -1;
  }();
  return v;
}
bool split_pair_wanted(int64_t Mp, int64_t Np) {
  const int mode = split_pair_mode();
  if (mode >= 0) return mode == 1;
  return 2 * (Mp / 256) * (Np / 256) >= current_sm_count();
}

// Stage ring of the pair kernel, plus 1 KB of alignment slack and 8 KB of
// guard after the ring (an MMA's B operand never reaches past its tile; the
// guard keeps every descriptor-addressed read inside the allocation).
constexpr int kOzPairSmem = 216 * 1024;
constexpr int kOzPairExtra = 1024 + 8192;

// The CTA-pair GEMM of one form over K-step launches [0, nkb32) in chunks of
// kc32 steps.
template <int FORM>
int launch_pair_form(const CUtensorMap &mapA, const CUtensorMap &mapB, OzPairArgs w, int64_t nkb32, int64_t kc32,
                     int accumulative, int stage_bytes, cudaStream_t st) {
  static std::atomic<uint64_t> pair_attr{0};
  once_per_device(pair_attr, [] {
    cudaFuncSetAttribute(oz_gemm_pair_kernel<FORM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kOzPairSmem + kOzPairExtra);
  });
  const int64_t ctas = 2 * (int64_t)w.tiles_m2 * w.tiles_n;
  if (ctas > 0x7fffffffLL) return TALSH_LIMIT_EXCEEDED;
  for (int64_t kb = 0; kb < nkb32; kb += kc32) {
    w.kb0 = kb;
    w.kb1 = std::min(nkb32, kb + kc32);
    w.beta = (kb == 0) ? (accumulative ? 1 : 0) : 1;
    oz_gemm_pair_kernel<FORM><<<(unsigned)ctas, kOzWsThreads, w.nst * stage_bytes + kOzPairExtra, st>>>(mapA, mapB,
                                                                                                      w);
    note_launch();
    const int rc = check_launch("oz_gemm_pair_kernel");
    if (rc != 0) return rc;
  }
  return TALSH_SUCCESS;
}

// The warp-specialised GEMM of one form over K-step launches [0, nkb32) in
// chunks of kc32 steps (32 bytes each).
template <int FORM>
int launch_ws_form(OzWsArgs w, int64_t nkb32, int64_t kc32,
                   int accumulative, int stage_bytes, cudaStream_t st) {
  static std::atomic<uint64_t> ws_attr{0};
  once_per_device(ws_attr, [] {
    cudaFuncSetAttribute(oz_gemm_ws_kernel<FORM>, cudaFuncAttributeMaxDynamicSharedMemorySize, kOzWsSmem + 1024);
  });
  const int64_t tiles = (int64_t)w.tiles_m * w.tiles_n;
  for (int64_t kb = 0; kb < nkb32; kb += kc32) {
    w.kb0 = kb;
    w.kb1 = std::min(nkb32, kb + kc32);
    w.beta = (kb == 0) ? (accumulative ? 1 : 0) : 1;
    oz_gemm_ws_kernel<FORM><<<(unsigned)tiles, kOzWsThreads, w.nst * stage_bytes + 1024, st>>>(w);
    note_launch();
    const int rc = check_launch("oz_gemm_ws_kernel");
    if (rc != 0) return rc;
  }
  return TALSH_SUCCESS;
}

}  // namespace

int contract_split_launch(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                          const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                          const void *R, double alpha_re, int accumulative, int slices, void *scratch,
                          size_t scratch_bytes, void *stream) {
  if (kind != R8) return TALSH_NOT_IMPLEMENTED;
  if (lrank == 0 || rrank == 0 || drank == 0) return TALSH_NOT_IMPLEMENTED;
  FormCode fc;
  if (!decode_form(slices, fc)) return TALSH_INVALID_ARGS;
  const int code = slices;
  slices = fc.S;
  const int es = form_esize(fc.form);
  if (D == nullptr || L == nullptr || R == nullptr || cptrn == nullptr) return TALSH_INVALID_ARGS;
  if (has_hyper_index(cptrn, lrank, rrank)) return TALSH_NOT_IMPLEMENTED;
  if (!elem_aligned(R8, D) || !elem_aligned(R8, L) || !elem_aligned(R8, R)) return TALSH_INVALID_ARGS;
  const size_t need = contract_split_scratch(kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims, code);
  if (need == 0 || scratch == nullptr || scratch_bytes < need) return TALSH_INVALID_ARGS;
  cudaStream_t st = (cudaStream_t)stream;
  char *base = (char *)scratch;
  int64_t M, N, K;
  const int64_t *mD = nullptr, *nD = nullptr;
  OzPlan p;
  {
    int64_t M0 = 1, N0 = 1, K0 = 1;
    for (int i = 0; i < lrank; ++i) (cptrn[i] > 0 ? M0 : K0) *= ldims[i];
    for (int i = 0; i < rrank; ++i)
      if (cptrn[lrank + i] > 0) N0 *= rdims[i];
    oz_plan(M0, N0, K0, slices, p, es);
  }
  int rc = contract_build_tables(cptrn, drank, ddims, lrank, ldims, rrank, rdims, base + p.off_tab, st, M, N,
                                 K, &mD, &nD);
  if (rc) return rc;
  if (M != p.M || N != p.N || K != p.K) return TALSH_NOT_IMPLEMENTED;  // hyper-indices or unit-only groups
  int o2n[kMaxRank];
  operand_o2n(cptrn, lrank, ldims, rrank, rdims, true, o2n);
  if ((rc = permute_launch_o2n(R8, lrank, ldims, o2n, L, base + p.off_A64, st)) != 0) return rc;
  operand_o2n(cptrn, lrank, ldims, rrank, rdims, false, o2n);
  if ((rc = permute_launch_o2n(R8, rrank, rdims, o2n, R, base + p.off_B64, st)) != 0) return rc;
  int8_t *As = (int8_t *)(base + p.off_As);
  int8_t *Bs = (int8_t *)(base + p.off_Bs);
  int32_t *ea = (int32_t *)(base + p.off_ea);
  int32_t *eb = (int32_t *)(base + p.off_eb);
  int *err = (int *)(base + p.off_err);
  cudaMemsetAsync(err, 0, sizeof(int), st);
  if (p.Mp > 0x7fffffffLL || p.Np > 0x7fffffffLL) return TALSH_LIMIT_EXCEEDED;
  const double *A64 = (const double *)(base + p.off_A64), *B64 = (const double *)(base + p.off_B64);
  // The warp-specialised GEMM reads the tiled layout with bulk copies; the
  // single-loop int8 kernel (TALSH_B200_SPLIT_SIMPLE=1) reads [S][rows][Kp].
  const bool simple = oz_force_simple() && fc.form == kFormInt8;
  const int64_t Kbytes = p.Kp * es;
  // The pair kernel reads [S][rows][Kp] through 2-D tensor maps (its copies
  // complete on the even CTA's barriers; the maps need 32-bit row
  // coordinates); the single-CTA kernel reads the tiled layout by bulk copies;
  // the stall test runs the single-CTA kernel.
  CUtensorMap mapA, mapB;
  std::memset(&mapA, 0, sizeof(mapA));
  std::memset(&mapB, 0, sizeof(mapB));
  const bool pair = !simple && g_stall_test.load() == 0 && split_pair_wanted(p.Mp, p.Np) &&
                    (int64_t)slices * p.Mp < 0x7fffffffLL && (int64_t)slices * p.Np < 0x7fffffffLL &&
                    make_slice_map(&mapA, As, Kbytes, slices * p.Mp, kOzBM) &&
                    make_slice_map(&mapB, Bs, Kbytes, slices * p.Np, 128);
  const int tiled = (!simple && !pair) ? 1 : 0;
  auto split_float = [&](auto kern) {
    kern<<<(unsigned)p.Mp, 256, 0, st>>>(A64, M, K, p.Mp, p.Kp, slices, (unsigned char *)As, ea, tiled);
    note_launch();
    kern<<<(unsigned)p.Np, 256, 0, st>>>(B64, N, K, p.Np, p.Kp, slices, (unsigned char *)Bs, eb, tiled);
    note_launch();
  };
  switch (fc.form) {
    case kFormBF16: split_float(split_rows_float<kFormBF16>); break;
    case kFormTF32: split_float(split_rows_float<kFormTF32>); break;
    case kFormFP8: split_float(split_rows_float<kFormFP8>); break;
    default:
      oz_split_rows<<<(unsigned)p.Mp, 256, 0, st>>>(A64, M, K, p.Mp, p.Kp, slices, As, ea, tiled);
      note_launch();
      oz_split_rows<<<(unsigned)p.Np, 256, 0, st>>>(B64, N, K, p.Np, p.Kp, slices, Bs, eb, tiled);
      note_launch();
  }
  if ((rc = check_launch("split rows")) != 0) return rc;
  // K chunks keep every int32 accumulator exact: slices * Kc * 127^2 < 2^31.
  const int64_t kc_max = ((int64_t)0x7fffffff / ((int64_t)slices * 127 * 127)) / kOzBK;
  const int64_t nkb = p.Kp / kOzBK;
  const int smem = kOzStages * slices * (kATileBytes + kBTileBytes);
  static std::atomic<uint64_t> attr_done{0};
  once_per_device(attr_done, [] {
    cudaFuncSetAttribute(oz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kOzStages * kOzMaxSlices * (kATileBytes + kBTileBytes));
  });
  OzArgs a;
  a.A = As; a.B = Bs; a.Mp = p.Mp; a.Np = p.Np; a.Kp = p.Kp; a.S = slices;
  a.ea = ea; a.eb = eb; a.D = (double *)D; a.mD = mD; a.nD = nD; a.M = M; a.N = N;
  a.alpha = alpha_re; a.err = err;
  a.tmem_cols = 32;
  while (a.tmem_cols < (uint32_t)(slices * kOzBN)) a.tmem_cols <<= 1;
  const dim3 grid((unsigned)(p.Mp / kOzBM), (unsigned)(p.Np / kOzBN));
  if (grid.y > 65535) return TALSH_LIMIT_EXCEEDED;
  // Warp-specialised TMA pipeline when the tensor maps can be encoded (the
  // slice matrices' row counts must fit the 32-bit TMA coordinates).
  const int64_t nkb32 = Kbytes / kWsBK;
  int64_t kc32 = kc_max * (kOzBK / kWsBK);  // K steps per launch
  if (fc.form != kFormInt8) {
    const int64_t kc_el = fp32_kchunk();
    kc32 = kc_el > 0 ? std::max<int64_t>(2, round_up(kc_el * es, kOzBK) / kWsBK) : nkb32;
  }
  if (pair) {
    const int stage_bytes = slices * (kWsATile + kPairBTile);
    OzPairArgs w;
    w.spin_limit = kSpinLimit;
    w.Mp = p.Mp; w.Np = p.Np; w.S = slices;
    w.nst = std::max(2, std::min(8, kOzPairSmem / stage_bytes));
    w.tiles_m2 = (int)(p.Mp / (2 * kOzBM));
    w.tiles_n = (int)(p.Np / kPairBN);
    w.group_m = std::max(1, ws_group_m() / 2);
    w.ea = ea; w.eb = eb; w.D = (double *)D; w.mD = mD; w.nD = nD; w.M = M; w.N = N;
    w.alpha = alpha_re; w.err = err;
    w.tmem_cols = 32;
    while (w.tmem_cols < (uint32_t)(std::min(slices, kPairDiag) * kPairBN)) w.tmem_cols <<= 1;
    switch (fc.form) {
      case kFormBF16: return launch_pair_form<kFormBF16>(mapA, mapB, w, nkb32, kc32, accumulative, stage_bytes, st);
      case kFormTF32: return launch_pair_form<kFormTF32>(mapA, mapB, w, nkb32, kc32, accumulative, stage_bytes, st);
      case kFormFP8: return launch_pair_form<kFormFP8>(mapA, mapB, w, nkb32, kc32, accumulative, stage_bytes, st);
      default: return launch_pair_form<kFormInt8>(mapA, mapB, w, nkb32, kc32, accumulative, stage_bytes, st);
    }
  }
  if (!tiled && fc.form != kFormInt8) return TALSH_NOT_IMPLEMENTED;  // the float forms have no simple kernel
  if (tiled) {
    const int stage_bytes = slices * (kWsATile + kWsBTile128);
    const int nst = std::max(2, std::min(8, kOzWsSmem / stage_bytes));
    const int64_t tiles = (p.Mp / kOzBM) * (p.Np / kWsBN);
    if (tiles > 0x7fffffffLL) return TALSH_LIMIT_EXCEEDED;
    OzWsArgs w;
    w.At = (const unsigned char *)As;
    w.Bt = (const unsigned char *)Bs;
    w.nbox = Kbytes / kWsBox;
    const bool stall = g_stall_test.load() != 0;
    w.spin_limit = stall ? (1u << 12) : kSpinLimit;
    w.stall_test = stall ? 1 : 0;
    w.Mp = p.Mp; w.Np = p.Np; w.S = slices; w.nst = nst;
    w.tiles_m = (int)(p.Mp / kOzBM);
    w.tiles_n = (int)(p.Np / kWsBN);
    w.group_m = ws_group_m();
    w.ea = ea; w.eb = eb; w.D = (double *)D; w.mD = mD; w.nD = nD; w.M = M; w.N = N;
    w.alpha = alpha_re; w.err = err;
    w.tmem_cols = 32;
    while (w.tmem_cols < (uint32_t)(std::min(slices, kWsDiagPerPass) * kWsBN)) w.tmem_cols <<= 1;
    switch (fc.form) {
      case kFormBF16: return launch_ws_form<kFormBF16>(w, nkb32, kc32, accumulative, stage_bytes, st);
      case kFormTF32: return launch_ws_form<kFormTF32>(w, nkb32, kc32, accumulative, stage_bytes, st);
      case kFormFP8: return launch_ws_form<kFormFP8>(w, nkb32, kc32, accumulative, stage_bytes, st);
      default: return launch_ws_form<kFormInt8>(w, nkb32, kc32, accumulative, stage_bytes, st);
    }
  }
  for (int64_t kb = 0; kb < nkb; kb += kc_max) {
    a.kb0 = kb;
    a.kb1 = std::min(nkb, kb + kc_max);
    a.beta = (kb == 0) ? (accumulative ? 1 : 0) : 1;
    oz_gemm_kernel<<<grid, kOzThreads, smem, st>>>(a);
    note_launch();
    if ((rc = check_launch("oz_gemm_kernel")) != 0) return rc;
  }
  return TALSH_SUCCESS;
}

// ---------------------------------------------------------------------------
// Complex(8) in split precision: the contraction is rewritten as one real(8)
// contraction (split_complex.h).  Scratch layout: the stacked operand Rx
// (2 x vol(R) complex elements, rounded up to 256 bytes), then the real form's
// scratch.
// ---------------------------------------------------------------------------

namespace {

size_t complex_rx_bytes(int rrank, const int *rdims) {
  size_t v = 2;
  for (int j = 0; j < rrank; ++j) v *= (size_t)rdims[j];
  return (v * 16 + 255) & ~size_t(255);
}

}  // namespace

size_t contract_split_complex_scratch(const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                                      int rrank, const int *rdims, int slices) {
  if (lrank == 0 || rrank == 0 || drank == 0) return 0;
  if (contract_validate(C8, cptrn, drank, ddims, lrank, ldims, rrank, rdims) != TALSH_SUCCESS) return 0;
  if (has_hyper_index(cptrn, lrank, rrank)) return 0;
  ComplexSplitForm f;
  if (complex_split_form(cptrn, drank, ddims, lrank, ldims, rrank, rdims, 0, f) != TALSH_SUCCESS) return 0;
  const size_t need =
      contract_split_scratch(R8, f.cptrn, f.drank, f.ddims, f.lrank, f.ldims, f.rrank, f.rdims, slices);
  return need ? complex_rx_bytes(rrank, rdims) + need : 0;
}

int contract_split_complex_launch(const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                                  int rrank, const int *rdims, void *D, const void *L, const void *R,
                                  double alpha_re, double alpha_im, int conj_bits, int accumulative, int slices,
                                  void *scratch, size_t scratch_bytes, void *stream) {
  if (lrank == 0 || rrank == 0 || drank == 0) return TALSH_NOT_IMPLEMENTED;
  FormCode fc;
  if (!decode_form(slices, fc)) return TALSH_INVALID_ARGS;
  int rc = contract_validate(C8, cptrn, drank, ddims, lrank, ldims, rrank, rdims);
  if (rc) return rc;
  if (has_hyper_index(cptrn, lrank, rrank)) return TALSH_NOT_IMPLEMENTED;
  if (D == nullptr || L == nullptr || R == nullptr || scratch == nullptr) return TALSH_INVALID_ARGS;
  if (!elem_aligned(C8, D) || !elem_aligned(C8, L) || !elem_aligned(C8, R) || !elem_aligned(C8, scratch))
    return TALSH_INVALID_ARGS;
  ComplexSplitForm f;
  if ((rc = complex_split_form(cptrn, drank, ddims, lrank, ldims, rrank, rdims, conj_bits, f)) != 0) return rc;
  const size_t rx = complex_rx_bytes(rrank, rdims);
  const size_t need =
      contract_split_scratch(R8, f.cptrn, f.drank, f.ddims, f.lrank, f.ldims, f.rrank, f.rdims, slices);
  if (need == 0 || scratch_bytes < rx + need) return TALSH_INVALID_ARGS;
  // Rx = [Y s, Y (z i) s], Y = R or conj(R), s = alpha or conj(alpha); z i s is
  // exact (a swap and a sign).
  size_t half = 1;
  for (int j = 0; j < rrank; ++j) half *= (size_t)rdims[j];
  int id[kMaxRank];
  for (int j = 0; j < rrank; ++j) id[j] = j + 1;
  const double sr = alpha_re, si = f.alpha_conj ? -alpha_im : alpha_im;
  const double zr = -f.z_im * si, zi = f.z_im * sr;
  char *rxp = (char *)scratch;
  if ((rc = tcTensorInit(C8, 2 * half, rxp, 0.0, 0.0, stream)) != TALSH_SUCCESS) return rc;
  if ((rc = tcTensorPermuteAdd(C8, rrank, rdims, id, R, rxp, sr, si, f.y_conj, stream)) != TALSH_SUCCESS)
    return rc;
  if ((rc = tcTensorPermuteAdd(C8, rrank, rdims, id, R, rxp + half * 16, zr, zi, f.y_conj, stream)) !=
      TALSH_SUCCESS)
    return rc;
  return contract_split_launch(R8, f.cptrn, f.drank, f.ddims, f.lrank, f.ldims, f.rrank, f.rdims, D, L, rxp, 1.0,
                               accumulative, slices, rxp + rx, scratch_bytes - rx, stream);
}

}  // namespace tb

namespace {
// The int8 form's documented slice argument: 0 (6) or 2..7.
bool plain_slices_ok(int slices) { return slices == 0 || (slices >= 2 && slices <= tb::kOzMaxSlices); }
int form_code(int form, int slices) {
  if (form < tb::kFormInt8 || form > tb::kFormFP8 || slices < 0 || slices > tb::kOzMaxSlices || slices == 1)
    return -1;
  return (form << 4) | slices;
}
}  // namespace

extern "C" size_t tcTensorContractSplitScratch(int data_kind, const int *cptrn, int drank,
                                               const int *ddims, int lrank, const int *ldims,
                                               int rrank, const int *rdims, int slices) {
  if (!plain_slices_ok(slices)) return 0;
  if (data_kind == C8)
    return tb::contract_split_complex_scratch(cptrn, drank, ddims, lrank, ldims, rrank, rdims, slices);
  return tb::contract_split_scratch(data_kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims, slices);
}

extern "C" int tcTensorContractSplit(int data_kind, const int *cptrn, int drank, const int *ddims,
                                     int lrank, const int *ldims, int rrank, const int *rdims, void *D,
                                     const void *L, const void *R, double alpha_re, double alpha_im,
                                     int conj_bits, int accumulative, int slices, void *scratch,
                                     size_t scratch_bytes, void *stream) {
  if (!plain_slices_ok(slices)) return TALSH_INVALID_ARGS;
  if (data_kind == C8)
    return tb::contract_split_complex_launch(cptrn, drank, ddims, lrank, ldims, rrank, rdims, D, L, R, alpha_re,
                                             alpha_im, conj_bits, accumulative, slices, scratch, scratch_bytes,
                                             stream);
  return tb::contract_split_launch(data_kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims, D, L, R,
                                   alpha_re, accumulative, slices, scratch, scratch_bytes, stream);
}

extern "C" size_t tcTensorContractSplitFormScratch(int data_kind, const int *cptrn, int drank,
                                                   const int *ddims, int lrank, const int *ldims,
                                                   int rrank, const int *rdims, int form, int slices) {
  const int code = form_code(form, slices);
  if (code < 0) return 0;
  if (data_kind == C8)
    return tb::contract_split_complex_scratch(cptrn, drank, ddims, lrank, ldims, rrank, rdims, code);
  return tb::contract_split_scratch(data_kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims, code);
}

extern "C" int tcTensorContractSplitForm(int data_kind, const int *cptrn, int drank, const int *ddims,
                                         int lrank, const int *ldims, int rrank, const int *rdims, void *D,
                                         const void *L, const void *R, double alpha_re, double alpha_im,
                                         int conj_bits, int accumulative, int form, int slices, void *scratch,
                                         size_t scratch_bytes, void *stream) {
  const int code = form_code(form, slices);
  if (code < 0) return TALSH_INVALID_ARGS;
  if (data_kind == C8)
    return tb::contract_split_complex_launch(cptrn, drank, ddims, lrank, ldims, rrank, rdims, D, L, R, alpha_re,
                                             alpha_im, conj_bits, accumulative, code, scratch, scratch_bytes,
                                             stream);
  return tb::contract_split_launch(data_kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims, D, L, R,
                                   alpha_re, accumulative, code, scratch, scratch_bytes, stream);
}

extern "C" int tcTestSplitStall(int enable) {
  tb::g_stall_test = enable ? 1 : 0;
  return TALSH_SUCCESS;
}

// Number of CTAs on the current device that gave up a bounded wait since the
// library was loaded (reference gpu_get_error_count, device_algebra.h:200,
// tensor_algebra_gpu_nvidia.cu:2315); -1 when it cannot be read.
extern "C" int gpu_get_error_count(void) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, tb::g_device_errors, sizeof(int), 0, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return v;
}
