// Tensor contraction D = beta*D + alpha * sum_contracted L*R for sm_100a.
//
// Reference semantics: tensor_block_contract (tensor_algebra_cpu.F90:3675-4358)
// and gpu_tensor_block_contract_dlf (tensor_algebra_gpu_nvidia.cu:5847-7183):
// digital pattern, conjugation bits (the D bit flips the L and R bits), real
// kinds use real(alpha), beta = 1 when accumulative else D is overwritten.
//
// Design (no transpose + GEMM + transpose): every operand stays in its own
// layout.  The contraction is viewed as C[m,n] = sum_k A[m,k] B[k,n] where
//   m runs over L's uncontracted indices (L order), n over R's uncontracted
//   indices (R order) and k over the contracted pairs,
// and three small offset tables (m -> L and D offsets, n -> R and D offsets,
// k -> L and R offsets) built on the device turn every tile load into a
// gather and the epilogue into a scatter in D's own layout.  Tile loads are
// mapped so that the operand's stride-1 index runs across the lanes.
//  * R8: warp-level DMMA (mma.sync m8n8k4 f64) on a multistage cp.async
//    pipeline, FP64 end to end.
//  * R4 / C4 / C8: register-blocked SIMT FMA kernel on the same tables.
//  * Degenerate patterns: full contraction (dot, deterministic two-pass),
//    scalar x tensor (the permute-add kernel with a device-side scale) and
//    scalar x scalar.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "common.h"
#include "device_once.h"

namespace tb {
int permute_scaled_by_device_scalar(int kind, int rank, const int *dims, const int *o2n,
                                    const void *src, void *dst, double alpha_re, double alpha_im,
                                    const void *scalar_dev, int scalar_conj, int tensor_conj,
                                    int accumulate, void *stream);
namespace {

constexpr int kMaxGR = 24;  // max indices per group (m, n or k)

struct TableParams {
  int nm, nn, nk, nh;
  int64_t M, N, K, H;
  int64_t mext[kMaxGR], mstrL[kMaxGR], mstrD[kMaxGR];
  int64_t next[kMaxGR], nstrR[kMaxGR], nstrD[kMaxGR];
  int64_t kext[kMaxGR], kstrL[kMaxGR], kstrR[kMaxGR];
  // hyper-indices (in D, L and R): one independent GEMM per combination
  int64_t hext[kMaxGR], hstrL[kMaxGR], hstrR[kMaxGR], hstrD[kMaxGR];
  int64_t *mL, *mD, *nR, *nD, *kL, *kR;
  int64_t *hL, *hR, *hD;  // used when nh > 0
};

__global__ void build_tables_kernel(const TableParams T) {
  const int64_t mnk = T.M + T.N + T.K;
  const int64_t total = mnk + (T.nh > 0 ? T.H : 0);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    if (i >= mnk) {
      int64_t r = i - mnk, a = 0, b = 0, c = 0;
      for (int d = 0; d < T.nh; ++d) {
        const int64_t x = r % T.hext[d];
        r /= T.hext[d];
        a += x * T.hstrL[d];
        b += x * T.hstrR[d];
        c += x * T.hstrD[d];
      }
      T.hL[i - mnk] = a;
      T.hR[i - mnk] = b;
      T.hD[i - mnk] = c;
    } else if (i < T.M) {
      int64_t r = i, a = 0, b = 0;
      for (int d = 0; d < T.nm; ++d) {
        const int64_t c = r % T.mext[d];
        r /= T.mext[d];
        a += c * T.mstrL[d];
        b += c * T.mstrD[d];
      }
      T.mL[i] = a;
      T.mD[i] = b;
    } else if (i < T.M + T.N) {
      int64_t r = i - T.M, a = 0, b = 0;
      for (int d = 0; d < T.nn; ++d) {
        const int64_t c = r % T.next[d];
        r /= T.next[d];
        a += c * T.nstrR[d];
        b += c * T.nstrD[d];
      }
      T.nR[i - T.M] = a;
      T.nD[i - T.M] = b;
    } else {
      int64_t r = i - T.M - T.N, a = 0, b = 0;
      for (int d = 0; d < T.nk; ++d) {
        const int64_t c = r % T.kext[d];
        r /= T.kext[d];
        a += c * T.kstrL[d];
        b += c * T.kstrR[d];
      }
      T.kL[i - T.M - T.N] = a;
      T.kR[i - T.M - T.N] = b;
    }
  }
}

struct GemmArgs {
  int M, N, K;
  int tiles_m;
  int tiles_mn;                      // tiles of one GEMM (hyper-index launches)
  int H;                             // hyper combinations (1 without hyper-indices)
  const int64_t *hL, *hR, *hD;       // per hyper combination offsets, or null
  const int64_t *mL, *mD, *nR, *nD, *kL, *kR;
  double alpha_re, alpha_im;
  int beta;       // 1: D += ..., 0: D = ...
  int a_along_m;  // A tile loads: lanes along m (else along k)
  int b_along_n;  // B tile loads: lanes along n (else along k)
  int conj_l, conj_r;
};

// Hyper-index launches: block b runs tile b mod tiles_mn of the GEMM for
// hyper combination b / tiles_mn, whose operands start at the table offsets.
template <typename T>
__device__ __forceinline__ int hyper_offsets(const GemmArgs &a, const T *&L, const T *&R, T *&D) {
  int local = (int)blockIdx.x;
  if (a.hL != nullptr) {
    const int h = local / a.tiles_mn;
    local -= h * a.tiles_mn;
    L += a.hL[h];
    R += a.hR[h];
    D += a.hD[h];
  }
  return local;
}

// ---------------------------------------------------------------- R8: DMMA
__device__ __forceinline__ void cp_async8(void *smem_ptr, const void *gptr, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_ptr);
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gptr), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int BM, int BN>
struct DmmaCfg {
  // warp tile: 32x32, or 16x16 in 32x32 CTA tiles (four warps per small tile)
  static constexpr int WM = BM <= 32 ? 16 : 32, WN = BN <= 32 ? 16 : 32;
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
  static constexpr int THREADS = WARPS_M * WARPS_N * 32;
  static constexpr int BK = 16, STAGES = 3;
  static constexpr int AP = BM + 8, BP = BN + 8;    // pitches: 2-wavefront fragment loads
  static constexpr size_t SMEM = (size_t)STAGES * BK * (AP + BP) * sizeof(double) +
                                 (size_t)(2 * BM + 2 * BN + 2 * STAGES * BK) * sizeof(int64_t);
};

// k-offset tables of the tiles in flight live in a shared ring (slot t % ST
// holds tile t's BK entries of kL and kR).  The tables of tiles 0..ST-1 are
// written before the main loop; afterwards warp 0 fetches tile t+ST's entries
// from global memory during iteration t and stores them at its end, so the
// address of a cp.async never waits for a global load.
template <int BK, int ST>
__device__ __forceinline__ void kring_init(const GemmArgs &a, int64_t *kLs, int64_t *kRs, int tid, int nt,
                                           int64_t &pf) {
  for (int i = tid; i < ST * BK; i += nt) {
    kLs[i] = i < a.K ? a.kL[i] : 0;
    kRs[i] = i < a.K ? a.kR[i] : 0;
  }
  if (tid < 2 * BK) {
    const int k = ST * BK + (tid % BK);
    pf = k < a.K ? (tid < BK ? a.kL[k] : a.kR[k]) : 0;
  }
}
template <int BK, int ST>
__device__ __forceinline__ void kring_step(const GemmArgs &a, int64_t *kLs, int64_t *kRs, int tid, int kt,
                                           int64_t &pf) {
  if (tid < 2 * BK) {
    const int j = tid % BK;
    (tid < BK ? kLs : kRs)[(kt % ST) * BK + j] = pf;
    const int64_t k = (int64_t)(kt + ST + 1) * BK + j;
    pf = k < a.K ? (tid < BK ? a.kL[k] : a.kR[k]) : 0;
  }
}

// Column swizzle of the FP64 tiles: row k stores column c at c ^ ((k >> 1) & 7)
// (a permutation inside each aligned group of 8 columns).  Tile loads whose
// lanes run along k (the operand's stride-1 index is contracted) then hit 16
// different bank pairs per half-warp instead of 2; fragment loads, which read
// 8 consecutive columns of one row, are unaffected.
__device__ __forceinline__ int kswz(int k) { return (k >> 1) & 7; }

// One BM x BN tile of a gather-GEMM (shared by the single-contraction kernel and
// the batched one).
template <int BM, int BN>
__device__ __forceinline__ void dmma_tile(const double *__restrict__ L, const double *__restrict__ R,
                                          double *D, const GemmArgs &a, int tile_m, int tile_n,
                                          unsigned char *smem) {
  using C = DmmaCfg<BM, BN>;
  constexpr int BK = C::BK, ST = C::STAGES, AP = C::AP, BP = C::BP, NT = C::THREADS;
  double *As = reinterpret_cast<double *>(smem);
  double *Bs = As + ST * BK * AP;
  int64_t *mLs = reinterpret_cast<int64_t *>(Bs + ST * BK * BP);
  int64_t *mDs = mLs + BM;
  int64_t *nRs = mDs + BM;
  int64_t *nDs = nRs + BN;
  int64_t *kLs = nDs + BN;
  int64_t *kRs = kLs + ST * BK;
  int64_t pf = 0;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = tile_m * BM, n0 = tile_n * BN;
  for (int i = tid; i < BM; i += NT) {
    const int m = m0 + i;
    mLs[i] = m < a.M ? a.mL[m] : 0;
    mDs[i] = m < a.M ? a.mD[m] : 0;
  }
  for (int i = tid; i < BN; i += NT) {
    const int n = n0 + i;
    nRs[i] = n < a.N ? a.nR[n] : 0;
    nDs[i] = n < a.N ? a.nD[n] : 0;
  }
  kring_init<BK, ST>(a, kLs, kRs, tid, NT, pf);
  __syncthreads();

  const int numK = (a.K + BK - 1) / BK;
  auto load_tile = [&](int kt, int s) {
    double *as = As + s * BK * AP;
    double *bs = Bs + s * BK * BP;
#pragma unroll
    for (int i = 0; i < (BM * BK) / NT; ++i) {
      const int idx = tid + i * NT;
      const int ml = a.a_along_m ? (idx % BM) : (idx / BK);
      const int kl = a.a_along_m ? (idx / BM) : (idx % BK);
      const int m = m0 + ml, k = kt * BK + kl;
      const bool v = (m < a.M) && (k < a.K);
      const double *src = v ? (L + mLs[ml] + kLs[s * BK + kl]) : L;
      cp_async8(as + kl * AP + (ml ^ kswz(kl)), src, v);
    }
#pragma unroll
    for (int i = 0; i < (BN * BK) / NT; ++i) {
      const int idx = tid + i * NT;
      const int nl = a.b_along_n ? (idx % BN) : (idx / BK);
      const int kl = a.b_along_n ? (idx / BN) : (idx % BK);
      const int n = n0 + nl, k = kt * BK + kl;
      const bool v = (n < a.N) && (k < a.K);
      const double *src = v ? (R + nRs[nl] + kRs[s * BK + kl]) : R;
      cp_async8(bs + kl * BP + (nl ^ kswz(kl)), src, v);
    }
  };

  constexpr int FM = C::WM / 8, FN = C::WN / 8;
  double acc[FM][FN][2];
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int wm0 = (warp % C::WARPS_M) * C::WM, wn0 = (warp / C::WARPS_M) * C::WN;
  const int fr = lane >> 2, fc = lane & 3;

#pragma unroll
  for (int s = 0; s < ST - 1; ++s) {
    if (s < numK) load_tile(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < numK; ++kt) {
    cp_async_wait<ST - 2>();
    __syncthreads();
    const int pre = kt + ST - 1;
    if (pre < numK) load_tile(pre, pre % ST);
    cp_async_commit();
    const double *as = As + (kt % ST) * BK * AP;
    const double *bs = Bs + (kt % ST) * BK * BP;
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      double af[FM], bf[FN];
      const int sw = kswz(ks * 4 + fc);
#pragma unroll
      for (int i = 0; i < FM; ++i) af[i] = as[(ks * 4 + fc) * AP + wm0 + i * 8 + (fr ^ sw)];
#pragma unroll
      for (int j = 0; j < FN; ++j) bf[j] = bs[(ks * 4 + fc) * BP + wn0 + j * 8 + (fr ^ sw)];
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    kring_step<BK, ST>(a, kLs, kRs, tid, kt, pf);
  }
  cp_async_wait<0>();

  const double alpha = a.alpha_re;
#pragma unroll
  for (int i = 0; i < FM; ++i) {
    const int ml = wm0 + i * 8 + fr;
    if (m0 + ml >= a.M) continue;
#pragma unroll
    for (int j = 0; j < FN; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int nl = wn0 + j * 8 + fc * 2 + h;
        if (n0 + nl >= a.N) continue;
        double *p = D + mDs[ml] + nDs[nl];
        *p = a.beta ? fma(alpha, acc[i][j][h], *p) : alpha * acc[i][j][h];
      }
    }
  }
}

// Complex-double tile on the FP64 tensor pipe: complex elements stay
// interleaved in shared memory (one 16-byte cp.async per element, one 128-bit
// load per fragment element), and
// C_re += A_re B_re - A_im B_im, C_im += A_re B_im + A_im B_re run as four
// DMMA products.  Row pitches of BM + 2 elements put the four k-rows of a
// fragment load in different bank groups.
// Warp tiles are 32 x 16 (16 x 16 in 32x32 CTA tiles): two accumulator sets
// (real, imaginary) per fragment.
template <int BM, int BN>
struct ZmmaCfg {
  static constexpr int WM = BM <= 32 ? 16 : 32, WN = 16;
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / WN;
  static constexpr int THREADS = WARPS_M * WARPS_N * 32;
  static constexpr int BK = 16, STAGES = BM <= 32 ? 2 : 3;  // two stages keep five small CTAs per SM
  static constexpr int AP = BM + 2, BP = BN + 2;           // in complex elements
  static constexpr size_t SMEM = (size_t)STAGES * BK * (AP + BP) * sizeof(double2) +
                                 (size_t)(2 * BM + 2 * BN + 2 * STAGES * BK) * sizeof(int64_t);
};

__device__ __forceinline__ void cp_async16(void *smem_ptr, const void *gptr, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_ptr);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gptr), "r"(n));
}


template <int BM, int BN>
__device__ __forceinline__ void zmma_tile(const double2 *__restrict__ L, const double2 *__restrict__ R,
                                          double2 *D, const GemmArgs &a, int tile_m, int tile_n,
                                          unsigned char *smem) {
  using C = ZmmaCfg<BM, BN>;
  constexpr int BK = C::BK, ST = C::STAGES, AP = C::AP, BP = C::BP, NT = C::THREADS;
  double2 *As = reinterpret_cast<double2 *>(smem);
  double2 *Bs = As + ST * BK * AP;
  int64_t *mLs = reinterpret_cast<int64_t *>(Bs + ST * BK * BP);
  int64_t *mDs = mLs + BM;
  int64_t *nRs = mDs + BM;
  int64_t *nDs = nRs + BN;
  int64_t *kLs = nDs + BN;
  int64_t *kRs = kLs + ST * BK;
  int64_t pf = 0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = tile_m * BM, n0 = tile_n * BN;
  for (int i = tid; i < BM; i += NT) {
    const int m = m0 + i;
    mLs[i] = m < a.M ? a.mL[m] : 0;
    mDs[i] = m < a.M ? a.mD[m] : 0;
  }
  for (int i = tid; i < BN; i += NT) {
    const int n = n0 + i;
    nRs[i] = n < a.N ? a.nR[n] : 0;
    nDs[i] = n < a.N ? a.nD[n] : 0;
  }
  kring_init<BK, ST>(a, kLs, kRs, tid, NT, pf);
  __syncthreads();
  const int numK = (a.K + BK - 1) / BK;
  auto load_tile = [&](int kt, int s) {
#pragma unroll
    for (int i = 0; i < (BM * BK) / NT; ++i) {
      const int idx = tid + i * NT;
      const int ml = a.a_along_m ? (idx % BM) : (idx / BK);
      const int kl = a.a_along_m ? (idx / BM) : (idx % BK);
      const int m = m0 + ml, k = kt * BK + kl;
      const bool v = (m < a.M) && (k < a.K);
      const double2 *src = v ? (L + mLs[ml] + kLs[s * BK + kl]) : L;
      cp_async16(As + (s * BK + kl) * AP + ml, src, v);
    }
#pragma unroll
    for (int i = 0; i < (BN * BK) / NT; ++i) {
      const int idx = tid + i * NT;
      const int nl = a.b_along_n ? (idx % BN) : (idx / BK);
      const int kl = a.b_along_n ? (idx / BN) : (idx % BK);
      const int n = n0 + nl, k = kt * BK + kl;
      const bool v = (n < a.N) && (k < a.K);
      const double2 *src = v ? (R + nRs[nl] + kRs[s * BK + kl]) : R;
      cp_async16(Bs + (s * BK + kl) * BP + nl, src, v);
    }
  };
  constexpr int FM = C::WM / 8, FN = C::WN / 8;
  double cr[FM][FN][2], ci[FM][FN][2];
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
  const int wm0 = (warp % C::WARPS_M) * C::WM, wn0 = (warp / C::WARPS_M) * C::WN;
  const int fr = lane >> 2, fc = lane & 3;
  const double sl = a.conj_l ? -1.0 : 1.0, sr = a.conj_r ? -1.0 : 1.0;
#pragma unroll
  for (int s = 0; s < ST - 1; ++s) {
    if (s < numK) load_tile(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < numK; ++kt) {
    cp_async_wait<ST - 2>();
    __syncthreads();
    const int pre = kt + ST - 1;
    if (pre < numK) load_tile(pre, pre % ST);
    cp_async_commit();
    const int so = (kt % ST);
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      double ar[FM], ai[FM], nai[FM], br[FN], bi[FN];
#pragma unroll
      for (int i = 0; i < FM; ++i) {
        const double2 v = As[(so * BK + ks * 4 + fc) * AP + wm0 + i * 8 + fr];
        ar[i] = v.x;
        ai[i] = sl * v.y;
        nai[i] = -ai[i];
      }
#pragma unroll
      for (int j = 0; j < FN; ++j) {
        const double2 v = Bs[(so * BK + ks * 4 + fc) * BP + wn0 + j * 8 + fr];
        br[j] = v.x;
        bi[j] = sr * v.y;
      }
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) {
          dmma_8x8x4(cr[i][j][0], cr[i][j][1], ar[i], br[j]);
          dmma_8x8x4(cr[i][j][0], cr[i][j][1], nai[i], bi[j]);
          dmma_8x8x4(ci[i][j][0], ci[i][j][1], ar[i], bi[j]);
          dmma_8x8x4(ci[i][j][0], ci[i][j][1], ai[i], br[j]);
        }
    }
    kring_step<BK, ST>(a, kLs, kRs, tid, kt, pf);
  }
  cp_async_wait<0>();
  const double alr = a.alpha_re, ali = a.alpha_im;
#pragma unroll
  for (int i = 0; i < FM; ++i) {
    const int ml = wm0 + i * 8 + fr;
    if (m0 + ml >= a.M) continue;
#pragma unroll
    for (int j = 0; j < FN; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int nl = wn0 + j * 8 + fc * 2 + h;
        if (n0 + nl >= a.N) continue;
        double2 *p = D + mDs[ml] + nDs[nl];
        const double vr = cr[i][j][h] * alr - ci[i][j][h] * ali;
        const double vi = cr[i][j][h] * ali + ci[i][j][h] * alr;
        if (a.beta) {
          const double2 d = *p;
          *p = make_double2(d.x + vr, d.y + vi);
        } else {
          *p = make_double2(vr, vi);
        }
      }
    }
  }
}

template <int BM, int BN>
__global__ void __launch_bounds__(ZmmaCfg<BM, BN>::THREADS)
    zgemm_gather_kernel(const double2 *__restrict__ L, const double2 *__restrict__ R, double2 *D,
                        const GemmArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const double2 *Lp = L, *Rp = R;
  double2 *Dp = D;
  const int local = hyper_offsets(a, Lp, Rp, Dp);
  zmma_tile<BM, BN>(Lp, Rp, Dp, a, local % a.tiles_m, local / a.tiles_m, smem);
}

template <int BM, int BN>
__global__ void __launch_bounds__(DmmaCfg<BM, BN>::THREADS)
    dgemm_gather_kernel(const double *__restrict__ L, const double *__restrict__ R, double *D,
                        const GemmArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const double *Lp = L, *Rp = R;
  double *Dp = D;
  const int local = hyper_offsets(a, Lp, Rp, Dp);
  dmma_tile<BM, BN>(Lp, Rp, Dp, a, local % a.tiles_m, local / a.tiles_m, smem);
}

// ------------------------------------------------- R4 / C4 / C8: SIMT FMA
template <typename T> struct Num;
template <> struct Num<float> {
  using A = float;
  __device__ static A zero() { return 0.f; }
  __device__ static A load(const float &x, bool) { return x; }
  __device__ static void fma_acc(A &c, A x, A y) { c = fmaf(x, y, c); }
  __device__ static float out(A acc, float d, double ar, double, int beta) {
    const float v = acc * (float)ar;
    return beta ? d + v : v;
  }
};
template <> struct Num<double> {
  using A = double;
  __device__ static A zero() { return 0.0; }
  __device__ static A load(const double &x, bool) { return x; }
  __device__ static void fma_acc(A &c, A x, A y) { c = fma(x, y, c); }
  __device__ static double out(A acc, double d, double ar, double, int beta) {
    return beta ? fma(ar, acc, d) : ar * acc;
  }
};
template <> struct Num<float2> {
  using A = float2;
  __device__ static A zero() { return make_float2(0.f, 0.f); }
  __device__ static A load(const float2 &x, bool cj) { return cj ? make_float2(x.x, -x.y) : x; }
  __device__ static void fma_acc(A &c, A x, A y) {
    c.x = fmaf(x.x, y.x, c.x); c.x = fmaf(-x.y, y.y, c.x);
    c.y = fmaf(x.x, y.y, c.y); c.y = fmaf(x.y, y.x, c.y);
  }
  __device__ static float2 out(A acc, float2 d, double ar, double ai, int beta) {
    const float vr = acc.x * (float)ar - acc.y * (float)ai, vi = acc.x * (float)ai + acc.y * (float)ar;
    return beta ? make_float2(d.x + vr, d.y + vi) : make_float2(vr, vi);
  }
};
template <> struct Num<double2> {
  using A = double2;
  __device__ static A zero() { return make_double2(0.0, 0.0); }
  __device__ static A load(const double2 &x, bool cj) { return cj ? make_double2(x.x, -x.y) : x; }
  __device__ static void fma_acc(A &c, A x, A y) {
    c.x = fma(x.x, y.x, c.x); c.x = fma(-x.y, y.y, c.x);
    c.y = fma(x.x, y.y, c.y); c.y = fma(x.y, y.x, c.y);
  }
  __device__ static double2 out(A acc, double2 d, double ar, double ai, int beta) {
    const double vr = acc.x * ar - acc.y * ai, vi = acc.x * ai + acc.y * ar;
    return beta ? make_double2(d.x + vr, d.y + vi) : make_double2(vr, vi);
  }
};

constexpr int kSBM = 64, kSBN = 64, kSBK = 16, kSThreads = 256;

template <typename T>
__device__ __forceinline__ void simt_tile(const T *__restrict__ L, const T *__restrict__ R, T *D,
                                          const GemmArgs &a, int tile_m, int tile_n) {
  using A = typename Num<T>::A;
  __shared__ A As[kSBK][kSBM + 1];
  __shared__ A Bs[kSBK][kSBN + 1];
  __shared__ int64_t mLs[kSBM], mDs[kSBM], nRs[kSBN], nDs[kSBN];
  const int tid = threadIdx.x;
  const int m0 = tile_m * kSBM, n0 = tile_n * kSBN;
  for (int i = tid; i < kSBM; i += kSThreads) {
    const int m = m0 + i;
    mLs[i] = m < a.M ? a.mL[m] : 0;
    mDs[i] = m < a.M ? a.mD[m] : 0;
  }
  for (int i = tid; i < kSBN; i += kSThreads) {
    const int n = n0 + i;
    nRs[i] = n < a.N ? a.nR[n] : 0;
    nDs[i] = n < a.N ? a.nD[n] : 0;
  }
  const int tr = tid % 16, tc = tid / 16;  // 16 x 16 threads, 4 x 4 outputs each
  A acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = Num<T>::zero();
  __syncthreads();
  for (int k0 = 0; k0 < a.K; k0 += kSBK) {
#pragma unroll
    for (int i = 0; i < (kSBM * kSBK) / kSThreads; ++i) {
      const int idx = tid + i * kSThreads;
      const int ml = a.a_along_m ? (idx % kSBM) : (idx / kSBK);
      const int kl = a.a_along_m ? (idx / kSBM) : (idx % kSBK);
      const int m = m0 + ml, k = k0 + kl;
      As[kl][ml] = (m < a.M && k < a.K) ? Num<T>::load(L[mLs[ml] + a.kL[k]], a.conj_l) : Num<T>::zero();
    }
#pragma unroll
    for (int i = 0; i < (kSBN * kSBK) / kSThreads; ++i) {
      const int idx = tid + i * kSThreads;
      const int nl = a.b_along_n ? (idx % kSBN) : (idx / kSBK);
      const int kl = a.b_along_n ? (idx / kSBN) : (idx % kSBK);
      const int n = n0 + nl, k = k0 + kl;
      Bs[kl][nl] = (n < a.N && k < a.K) ? Num<T>::load(R[nRs[nl] + a.kR[k]], a.conj_r) : Num<T>::zero();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kSBK; ++kk) {
      A av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[kk][tr + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[kk][tc + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) Num<T>::fma_acc(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int ml = tr + 16 * i;
    if (m0 + ml >= a.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int nl = tc + 16 * j;
      if (n0 + nl >= a.N) continue;
      T *p = D + mDs[ml] + nDs[nl];
      *p = Num<T>::out(acc[i][j], a.beta ? *p : T(), a.alpha_re, a.alpha_im, a.beta);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kSThreads)
    gemm_gather_simt_kernel(const T *__restrict__ L, const T *__restrict__ R, T *D, const GemmArgs a) {
  const T *Lp = L, *Rp = R;
  T *Dp = D;
  const int local = hyper_offsets(a, Lp, Rp, Dp);
  simt_tile<T>(Lp, Rp, Dp, a, local % a.tiles_m, local / a.tiles_m);
}

// ------------------------------------------------------ full contraction
constexpr int kDotThreads = 256;

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return v;
}
__device__ double2 block_sum2(double2 v) {
  __shared__ double2 ws[kDotThreads / 32];
  v = warp_sum2(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  double2 r = make_double2(0.0, 0.0);
  if (warp == 0) {
    r = (lane < kDotThreads / 32) ? ws[lane] : make_double2(0.0, 0.0);
    r = warp_sum2(r);
  }
  return r;
}

template <typename T> __device__ __forceinline__ double2 as_c(const T &x, bool cj);
template <> __device__ __forceinline__ double2 as_c<float>(const float &x, bool) { return make_double2(x, 0.0); }
template <> __device__ __forceinline__ double2 as_c<double>(const double &x, bool) { return make_double2(x, 0.0); }
template <> __device__ __forceinline__ double2 as_c<float2>(const float2 &x, bool cj) { return make_double2(x.x, cj ? -x.y : x.y); }
template <> __device__ __forceinline__ double2 as_c<double2>(const double2 &x, bool cj) { return make_double2(x.x, cj ? -x.y : x.y); }

template <typename T> __device__ __forceinline__ void store_c(T *p, double2 v);
template <> __device__ __forceinline__ void store_c<float>(float *p, double2 v) { *p = (float)v.x; }
template <> __device__ __forceinline__ void store_c<double>(double *p, double2 v) { *p = v.x; }
template <> __device__ __forceinline__ void store_c<float2>(float2 *p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ void store_c<double2>(double2 *p, double2 v) { *p = v; }

template <typename T>
__global__ void __launch_bounds__(kDotThreads)
    dot_partial_kernel(const T *__restrict__ L, const T *__restrict__ R, const int64_t *kL,
                       const int64_t *kR, int64_t K, int64_t chunk, int cl, int cr, double2 *part) {
  const int64_t beg = (int64_t)blockIdx.x * chunk, end = min(K, beg + chunk);
  double2 acc = make_double2(0.0, 0.0);
  for (int64_t k = beg + threadIdx.x; k < end; k += kDotThreads) {
    const double2 x = as_c<T>(L[kL[k]], cl), y = as_c<T>(R[kR[k]], cr);
    acc.x += x.x * y.x - x.y * y.y;
    acc.y += x.x * y.y + x.y * y.x;
  }
  const double2 s = block_sum2(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

template <typename T>
__global__ void __launch_bounds__(kDotThreads)
    dot_final_kernel(const double2 *part, int n, T *D, double ar, double ai, int beta) {
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < n; i += kDotThreads) { acc.x += part[i].x; acc.y += part[i].y; }
  const double2 s = block_sum2(acc);
  if (threadIdx.x == 0) {
    double2 v = make_double2(s.x * ar - s.y * ai, s.x * ai + s.y * ar);
    if (beta) {
      const double2 d = as_c<T>(*D, false);
      v.x += d.x;
      v.y += d.y;
    }
    store_c<T>(D, v);
  }
}

// scalar x scalar: d = (beta ? d : 0) + (l*r)*alpha in complex(8) arithmetic.
template <typename T>
__global__ void scalar_mul_kernel(const T *L, const T *R, T *D, double ar, double ai, int cl,
                                  int cr, int beta) {
  const double2 l = as_c<T>(*L, cl), r = as_c<T>(*R, cr);
  const double2 p = make_double2(l.x * r.x - l.y * r.y, l.x * r.y + l.y * r.x);
  double2 v = make_double2(p.x * ar - p.y * ai, p.x * ai + p.y * ar);
  if (beta) {
    const double2 d = as_c<T>(*D, false);
    v.x = d.x + v.x;
    v.y = d.y + v.y;
  }
  store_c<T>(D, v);
}

int dot_blocks(int64_t K) {
  int64_t b = (K + 16383) / 16384;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 1024));
}

struct Analysis {
  TableParams T;
  bool a_along_m = true, b_along_n = true;
  int hyper = 0;
};

int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// Splits the pattern into m / n / k index groups with their strides.
int analyze(const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims, int rrank,
            const int *rdims, Analysis &an) {
  TableParams &T = an.T;
  std::memset(&T, 0, sizeof(T));
  int64_t dstr[kMaxRank], lstr[kMaxRank], rstr[kMaxRank];
  int64_t s = 1;
  for (int i = 0; i < drank; ++i) { dstr[i] = s; s *= ddims[i]; }
  s = 1;
  for (int i = 0; i < lrank; ++i) { lstr[i] = s; s *= ldims[i]; }
  s = 1;
  for (int i = 0; i < rrank; ++i) { rstr[i] = s; s *= rdims[i]; }
  // Validation in the manner of the GPU path (reference :5934-5966).
  int dseen[kMaxRank] = {0}, lseen[kMaxRank] = {0}, rseen[kMaxRank] = {0};
  for (int i = 0; i < lrank; ++i) {
    const int j = cptrn[i];
    if (j > 0) {
      if (j > drank || ddims[j - 1] != ldims[i]) return TALSH_INVALID_ARGS;
      dseen[j - 1]++;
    } else if (j < 0) {
      if (-j > rrank || rdims[-j - 1] != ldims[i] || cptrn[lrank - j - 1] != -(i + 1)) return TALSH_INVALID_ARGS;
      if (rseen[-j - 1]++) return TALSH_INVALID_ARGS;
    } else {
      return TALSH_INVALID_ARGS;
    }
  }
  for (int i = 0; i < rrank; ++i) {
    const int j = cptrn[lrank + i];
    if (j > 0) {
      if (j > drank || ddims[j - 1] != rdims[i]) return TALSH_INVALID_ARGS;
      dseen[j - 1]++;
    } else if (j < 0) {
      if (-j > lrank || ldims[-j - 1] != rdims[i] || cptrn[-j - 1] != -(i + 1)) return TALSH_INVALID_ARGS;
      if (lseen[-j - 1]++) return TALSH_INVALID_ARGS;
    } else {
      return TALSH_INVALID_ARGS;
    }
  }
  for (int i = 0; i < drank; ++i) {
    if (dseen[i] == 2) an.hyper++;
    else if (dseen[i] != 1) return TALSH_INVALID_ARGS;
  }
  // h: indices in D, L and R, in L order (reference nhu groups,
  // tensor_algebra_cpu.F90:5829-5839).
  T.H = 1;
  for (int i = 0; i < lrank; ++i) {
    const int j = cptrn[i];
    if (j <= 0 || dseen[j - 1] != 2 || ldims[i] == 1) continue;
    int r = 0;
    while (r < rrank && cptrn[lrank + r] != j) ++r;
    if (r == rrank) return TALSH_INVALID_ARGS;
    if (T.nh >= kMaxGR) return TALSH_LIMIT_EXCEEDED;
    T.hext[T.nh] = ldims[i]; T.hstrL[T.nh] = lstr[i]; T.hstrR[T.nh] = rstr[r]; T.hstrD[T.nh] = dstr[j - 1];
    T.H *= ldims[i]; T.nh++;
  }
  int64_t lvol = 1, rvol = 1;
  for (int i = 0; i < lrank; ++i) lvol *= ldims[i];
  for (int i = 0; i < rrank; ++i) rvol *= rdims[i];
  // m: L uncontracted in L order; n: R uncontracted in R order.
  T.M = T.N = T.K = 1;
  for (int i = 0; i < lrank; ++i) {
    if (cptrn[i] > 0 && dseen[cptrn[i] - 1] == 1 && ldims[i] > 1) {
      if (T.nm >= kMaxGR) return TALSH_LIMIT_EXCEEDED;
      T.mext[T.nm] = ldims[i]; T.mstrL[T.nm] = lstr[i]; T.mstrD[T.nm] = dstr[cptrn[i] - 1];
      T.M *= ldims[i]; T.nm++;
    }
  }
  for (int i = 0; i < rrank; ++i) {
    if (cptrn[lrank + i] > 0 && dseen[cptrn[lrank + i] - 1] == 1 && rdims[i] > 1) {
      if (T.nn >= kMaxGR) return TALSH_LIMIT_EXCEEDED;
      T.next[T.nn] = rdims[i]; T.nstrR[T.nn] = rstr[i]; T.nstrD[T.nn] = dstr[cptrn[lrank + i] - 1];
      T.N *= rdims[i]; T.nn++;
    }
  }
  // k: follow R's order when R's leading index is contracted and L's is not
  // (or R is the larger operand), otherwise L's order.
  const bool l_lead_k = lrank > 0 && cptrn[0] < 0;
  const bool r_lead_k = rrank > 0 && cptrn[lrank] < 0;
  const bool k_in_r_order = r_lead_k && (!l_lead_k || rvol > lvol);
  if (k_in_r_order) {
    for (int i = 0; i < rrank; ++i) {
      const int j = cptrn[lrank + i];
      if (j < 0 && rdims[i] > 1) {
        if (T.nk >= kMaxGR) return TALSH_LIMIT_EXCEEDED;
        T.kext[T.nk] = rdims[i]; T.kstrR[T.nk] = rstr[i]; T.kstrL[T.nk] = lstr[-j - 1];
        T.K *= rdims[i]; T.nk++;
      }
    }
  } else {
    for (int i = 0; i < lrank; ++i) {
      const int j = cptrn[i];
      if (j < 0 && ldims[i] > 1) {
        if (T.nk >= kMaxGR) return TALSH_LIMIT_EXCEEDED;
        T.kext[T.nk] = ldims[i]; T.kstrL[T.nk] = lstr[i]; T.kstrR[T.nk] = rstr[-j - 1];
        T.K *= ldims[i]; T.nk++;
      }
    }
  }
  // Lane mapping for the tile loads: along the operand's stride-1 group.
  an.a_along_m = T.nm > 0 && (T.nk == 0 || T.mstrL[0] <= T.kstrL[0]);
  an.b_along_n = T.nn > 0 && (T.nk == 0 || T.nstrR[0] <= T.kstrR[0]);
  return TALSH_SUCCESS;
}

size_t table_bytes(const TableParams &T) {
  return (size_t)align_up(8 * (2 * T.M + 2 * T.N + 2 * T.K + (T.nh > 0 ? 3 * T.H : 0)), 256);
}

// Grid of a gather-GEMM launch: tiles of one GEMM times hyper combinations.
int gemm_grid(GemmArgs &ga, int bm, int bn, int64_t *blocks) {
  ga.tiles_m = (ga.M + bm - 1) / bm;
  const int64_t per = (int64_t)ga.tiles_m * ((ga.N + bn - 1) / bn);
  const int64_t all = per * std::max(ga.H, 1);
  if (per > 0x7fffffffLL || all > 0x7fffffffLL) return TALSH_LIMIT_EXCEEDED;
  ga.tiles_mn = (int)per;
  *blocks = all;
  return TALSH_SUCCESS;
}

int sm_count_dev() { return current_sm_count(); }

template <int BM, int BN>
int launch_dmma(const double *L, const double *R, double *D, GemmArgs ga, cudaStream_t st) {
  using C = DmmaCfg<BM, BN>;
  static std::atomic<uint64_t> attr_set{0};
  once_per_device(attr_set, [] {
    cudaFuncSetAttribute(dgemm_gather_kernel<BM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)C::SMEM);
  });
  int64_t tiles = 0;
  if (gemm_grid(ga, BM, BN, &tiles)) return TALSH_LIMIT_EXCEEDED;
  dgemm_gather_kernel<BM, BN><<<(unsigned)tiles, C::THREADS, C::SMEM, st>>>(L, R, D, ga);
  note_launch();
  return check_launch("dgemm_gather_kernel");
}

template <int BM, int BN>
int launch_zmma(const double2 *L, const double2 *R, double2 *D, GemmArgs ga, cudaStream_t st) {
  using Z = ZmmaCfg<BM, BN>;
  static std::atomic<uint64_t> attr_set{0};
  once_per_device(attr_set, [] {
    cudaFuncSetAttribute(zgemm_gather_kernel<BM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Z::SMEM);
  });
  int64_t tiles = 0;
  if (gemm_grid(ga, BM, BN, &tiles)) return TALSH_LIMIT_EXCEEDED;
  zgemm_gather_kernel<BM, BN><<<(unsigned)tiles, Z::THREADS, Z::SMEM, st>>>(L, R, D, ga);
  note_launch();
  return check_launch("zgemm_gather_kernel");
}

template <typename T>
int launch_simt(const void *L, const void *R, void *D, GemmArgs ga, cudaStream_t st) {
  int64_t tiles = 0;
  if (gemm_grid(ga, kSBM, kSBN, &tiles)) return TALSH_LIMIT_EXCEEDED;
  gemm_gather_simt_kernel<T><<<(unsigned)tiles, kSThreads, 0, st>>>((const T *)L, (const T *)R,
                                                                     (T *)D, ga);
  note_launch();
  return check_launch("gemm_gather_simt_kernel");
}

template <typename T>
int launch_dot(const void *L, const void *R, void *D, const int64_t *kL, const int64_t *kR,
               int64_t K, int cl, int cr, double ar, double ai, int beta, double2 *part,
               cudaStream_t st) {
  const int nb = dot_blocks(K);
  const int64_t chunk = (K + nb - 1) / nb;
  dot_partial_kernel<T><<<nb, kDotThreads, 0, st>>>((const T *)L, (const T *)R, kL, kR, K, chunk, cl, cr, part);
  note_launch();
  dot_final_kernel<T><<<1, kDotThreads, 0, st>>>(part, nb, (T *)D, ar, ai, beta);
  note_launch();
  return check_launch("dot_kernels");
}

template <typename T>
int launch_scalar(const void *L, const void *R, void *D, double ar, double ai, int cl, int cr,
                  int beta, cudaStream_t st) {
  scalar_mul_kernel<T><<<1, 1, 0, st>>>((const T *)L, (const T *)R, (T *)D, ar, ai, cl, cr, beta);
  note_launch();
  return check_launch("scalar_mul_kernel");
}

// Operands must be aligned to their element size (16 bytes for C8): the
// kernels move whole elements with vector loads and stores.
bool elements_aligned(int kind, const void *D, const void *L, const void *R) {
  const uintptr_t m = (uintptr_t)kind_size(kind) - 1;
  return ((reinterpret_cast<uintptr_t>(D) | reinterpret_cast<uintptr_t>(L) | reinterpret_cast<uintptr_t>(R)) & m) == 0;
}

// Shape / kind checks shared by the scratch query and the launch.
int check_args(int kind, const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
               int rrank, const int *rdims) {
  if (kind_size(kind) == 0) return TALSH_INVALID_ARGS;
  if (drank < 0 || lrank < 0 || rrank < 0 || drank > kMaxRank || lrank > kMaxRank || rrank > kMaxRank)
    return TALSH_INVALID_ARGS;
  if ((lrank + rrank > 0 && cptrn == nullptr) || (drank > 0 && ddims == nullptr) ||
      (lrank > 0 && ldims == nullptr) || (rrank > 0 && rdims == nullptr))
    return TALSH_INVALID_ARGS;
  for (int i = 0; i < drank; ++i) if (ddims[i] <= 0) return TALSH_INVALID_ARGS;
  for (int i = 0; i < lrank; ++i) if (ldims[i] <= 0) return TALSH_INVALID_ARGS;
  for (int i = 0; i < rrank; ++i) if (rdims[i] <= 0) return TALSH_INVALID_ARGS;
  return TALSH_SUCCESS;
}

}  // namespace

// Scratch bytes needed by tcTensorContract for this shape (0 when none).
size_t contract_scratch_bytes(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                              const int *ldims, int rrank, const int *rdims) {
  if (check_args(kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims)) return 0;
  if (lrank == 0 || rrank == 0) return 0;
  Analysis an;
  if (analyze(cptrn, drank, ddims, lrank, ldims, rrank, rdims, an)) return 0;
  size_t b = table_bytes(an.T);
  if (drank == 0) b += (size_t)dot_blocks(an.T.K) * sizeof(double2);
  return b;
}

// The argument checks of contract_launch without launching anything.
int contract_validate(int kind, const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                      int rrank, const int *rdims) {
  int rc = check_args(kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims);
  if (rc) return rc;
  if (lrank == 0 && rrank == 0) return drank == 0 ? TALSH_SUCCESS : TALSH_INVALID_ARGS;
  if (lrank == 0 || rrank == 0) {
    const int trank = lrank ? lrank : rrank;
    const int *tdims = lrank ? ldims : rdims;
    const int *tptrn = lrank ? cptrn : cptrn + lrank;
    if (trank != drank) return TALSH_INVALID_ARGS;
    for (int i = 0; i < trank; ++i)
      if (tptrn[i] < 1 || tptrn[i] > drank || ddims[tptrn[i] - 1] != tdims[i]) return TALSH_INVALID_ARGS;
    return TALSH_SUCCESS;
  }
  Analysis an;
  if ((rc = analyze(cptrn, drank, ddims, lrank, ldims, rrank, rdims, an)) != 0) return rc;
  if (an.T.M > 0x7fffffffLL || an.T.N > 0x7fffffffLL || an.T.K > 0x7fffffffLL || an.T.H > 0x7fffffffLL)
    return TALSH_LIMIT_EXCEEDED;
  return TALSH_SUCCESS;
}

int contract_launch(int kind, const int *cptrn, int drank, const int *ddims, int lrank,
                    const int *ldims, int rrank, const int *rdims, void *D, const void *L,
                    const void *R, double alpha_re, double alpha_im, int conj_bits,
                    int accumulative, void *scratch, size_t scratch_bytes, void *stream) {
  int rc = check_args(kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims);
  if (rc) return rc;
  if (D == nullptr || L == nullptr || R == nullptr) return TALSH_INVALID_ARGS;
  if (!elements_aligned(kind, D, L, R)) return TALSH_INVALID_ARGS;
  const bool cplx = kind_is_complex(kind);
  int cl = 0, cr = 0;
  if (cplx) {
    int cb = conj_bits & 7;
    if (cb & 1) cb ^= 7;  // a conjugated destination conjugates both inputs instead
    cl = (cb >> 1) & 1;
    cr = (cb >> 2) & 1;
  }
  const double ar = alpha_re, ai = cplx ? alpha_im : 0.0;
  const int beta = accumulative ? 1 : 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (lrank == 0 && rrank == 0) {
    if (drank != 0) return TALSH_INVALID_ARGS;
    switch (kind) {
      case R4: return launch_scalar<float>(L, R, D, alpha_re, alpha_im, cl, cr, beta, st);
      case R8: return launch_scalar<double>(L, R, D, alpha_re, alpha_im, cl, cr, beta, st);
      case C4: return launch_scalar<float2>(L, R, D, alpha_re, alpha_im, cl, cr, beta, st);
      default: return launch_scalar<double2>(L, R, D, alpha_re, alpha_im, cl, cr, beta, st);
    }
  }
  if (lrank == 0 || rrank == 0) {
    // scalar x tensor: D (+)= permute(T) * (s * alpha), the reference's ADD_TENSOR case.
    const int trank = lrank ? lrank : rrank;
    const int *tdims = lrank ? ldims : rdims;
    const int *tptrn = lrank ? cptrn : cptrn + lrank;
    if (trank != drank) return TALSH_INVALID_ARGS;
    for (int i = 0; i < trank; ++i)
      if (tptrn[i] < 1 || tptrn[i] > drank || ddims[tptrn[i] - 1] != tdims[i]) return TALSH_INVALID_ARGS;
    return permute_scaled_by_device_scalar(kind, trank, tdims, tptrn, lrank ? L : R, D, alpha_re,
                                           alpha_im, lrank ? R : L, lrank ? cr : cl,
                                           lrank ? cl : cr, beta, stream);
  }
  Analysis an;
  if ((rc = analyze(cptrn, drank, ddims, lrank, ldims, rrank, rdims, an)) != 0) return rc;
  TableParams T = an.T;
  const size_t need = table_bytes(T) + (drank == 0 ? (size_t)dot_blocks(T.K) * sizeof(double2) : 0);
  if (scratch == nullptr || scratch_bytes < need) return TALSH_INVALID_ARGS;
  if (T.M > 0x7fffffffLL || T.N > 0x7fffffffLL || T.K > 0x7fffffffLL || T.H > 0x7fffffffLL)
    return TALSH_LIMIT_EXCEEDED;
  int64_t *base = (int64_t *)scratch;
  T.mL = base; T.mD = T.mL + T.M; T.nR = T.mD + T.M; T.nD = T.nR + T.N; T.kL = T.nD + T.N; T.kR = T.kL + T.K;
  if (T.nh > 0) {
    T.hL = T.kR + T.K; T.hR = T.hL + T.H; T.hD = T.hR + T.H;
  }
  {
    const int64_t total = T.M + T.N + T.K + (T.nh > 0 ? T.H : 0);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 4096));
    build_tables_kernel<<<grid, 256, 0, st>>>(T);
    note_launch();
    if ((rc = check_launch("build_tables_kernel")) != 0) return rc;
  }
  if (drank == 0) {
    double2 *part = (double2 *)((char *)scratch + table_bytes(T));
    switch (kind) {
      case R4: return launch_dot<float>(L, R, D, T.kL, T.kR, T.K, cl, cr, ar, ai, beta, part, st);
      case R8: return launch_dot<double>(L, R, D, T.kL, T.kR, T.K, cl, cr, ar, ai, beta, part, st);
      case C4: return launch_dot<float2>(L, R, D, T.kL, T.kR, T.K, cl, cr, ar, ai, beta, part, st);
      default: return launch_dot<double2>(L, R, D, T.kL, T.kR, T.K, cl, cr, ar, ai, beta, part, st);
    }
  }
  GemmArgs ga;
  std::memset(&ga, 0, sizeof(ga));
  ga.M = (int)T.M; ga.N = (int)T.N; ga.K = (int)T.K;
  ga.mL = T.mL; ga.mD = T.mD; ga.nR = T.nR; ga.nD = T.nD; ga.kL = T.kL; ga.kR = T.kR;
  ga.alpha_re = ar; ga.alpha_im = ai; ga.beta = beta;
  ga.a_along_m = an.a_along_m ? 1 : 0;
  ga.b_along_n = an.b_along_n ? 1 : 0;
  ga.conj_l = cl; ga.conj_r = cr;
  ga.H = (int)T.H;
  if (T.nh > 0) {
    ga.hL = T.hL; ga.hR = T.hR; ga.hD = T.hD;
  }
  switch (kind) {
    case R8: {
      const int64_t big_tiles = ((T.M + 127) / 128) * ((T.N + 127) / 128) * T.H;
      if (big_tiles >= 2 * sm_count_dev())
        return launch_dmma<128, 128>((const double *)L, (const double *)R, (double *)D, ga, st);
      return launch_dmma<64, 64>((const double *)L, (const double *)R, (double *)D, ga, st);
    }
    case R4: return launch_simt<float>(L, R, D, ga, st);
    case C4: return launch_simt<float2>(L, R, D, ga, st);
    default: return launch_zmma<64, 64>((const double2 *)L, (const double2 *)R, (double2 *)D, ga, st);
  }
}

}  // namespace tb

namespace tb {
// Offset tables (m -> L, D; n -> R, D; k -> L, R) for callers that only need
// the D scatter: bytes for given M, N, K, and a launch that builds them.
size_t contract_tables_bytes(int64_t M, int64_t N, int64_t K) {
  TableParams T;
  std::memset(&T, 0, sizeof(T));
  T.M = M; T.N = N; T.K = K;
  return table_bytes(T);
}

int contract_build_tables(const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                          int rrank, const int *rdims, void *tables, cudaStream_t st, int64_t &M,
                          int64_t &N, int64_t &K, const int64_t **mD, const int64_t **nD) {
  int rc = check_args(R8, cptrn, drank, ddims, lrank, ldims, rrank, rdims);
  if (rc) return rc;
  Analysis an;
  if ((rc = analyze(cptrn, drank, ddims, lrank, ldims, rrank, rdims, an)) != 0) return rc;
  if (an.hyper) return TALSH_NOT_IMPLEMENTED;
  TableParams T = an.T;
  int64_t *base = (int64_t *)tables;
  T.mL = base; T.mD = T.mL + T.M; T.nR = T.mD + T.M; T.nD = T.nR + T.N; T.kL = T.nD + T.N; T.kR = T.kL + T.K;
  const int64_t total = T.M + T.N + T.K;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 4096));
  build_tables_kernel<<<grid, 256, 0, st>>>(T);
  note_launch();
  if ((rc = check_launch("build_tables_kernel")) != 0) return rc;
  M = T.M; N = T.N; K = T.K;
  *mD = T.mD;
  *nD = T.nD;
  return TALSH_SUCCESS;
}
}  // namespace tb

extern "C" size_t tcTensorContractScratch(int data_kind, const int *cptrn, int drank,
                                          const int *ddims, int lrank, const int *ldims,
                                          int rrank, const int *rdims) {
  return tb::contract_scratch_bytes(data_kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims);
}


extern "C" int tcTensorContract(int data_kind, const int *cptrn, int drank, const int *ddims,
                                int lrank, const int *ldims, int rrank, const int *rdims, void *D,
                                const void *L, const void *R, double alpha_re, double alpha_im,
                                int conj_bits, int accumulative, void *scratch,
                                size_t scratch_bytes, void *stream) {
  return tb::contract_launch(data_kind, cptrn, drank, ddims, lrank, ldims, rrank, rdims, D, L, R,
                             alpha_re, alpha_im, conj_bits, accumulative, scratch, scratch_bytes,
                             stream);
}

// ---------------------------------------------------------------------------
// Batched contractions: many (small) contractions in one table launch and one
// persistent gather-GEMM launch per tile configuration.  Each task's compact
// descriptor (index groups, strides, GEMM arguments, operand pointers) is
// uploaded once; CTAs walk a flat list of tiles over all tasks of a
// configuration and find their task by binary search in its tile prefix sums.
// ---------------------------------------------------------------------------
namespace tb {
namespace {

constexpr int kBMaxG = 8;  // max dimensions per index group of a batched task

struct BatchDesc {
  int nm, nn, nk;
  int32_t mext[kBMaxG], next[kBMaxG], kext[kBMaxG];
  int64_t mstrL[kBMaxG], mstrD[kBMaxG], nstrR[kBMaxG], nstrD[kBMaxG], kstrL[kBMaxG], kstrR[kBMaxG];
  GemmArgs a;
  const void *L, *R;
  void *D;
};

// Tile configurations of the batch: 0 = DMMA 64x64, 1 = DMMA 32x32 (R8),
// 2 = SIMT 64x64 (R4, C4, C8: one list per kind).
enum : int { kCfgD64 = 0, kCfgD32 = 1, kCfgZ64 = 2, kCfgZ32 = 3, kCfgS4 = 4, kCfgS14 = 5, kNumCfg = 6 };
// Square tile edge of a configuration.
inline int cfg_tile(int c) { return (c == kCfgD32 || c == kCfgZ32) ? 32 : 64; }

__global__ void __launch_bounds__(256) batch_tables_kernel(const BatchDesc *descs) {
  const BatchDesc &d = descs[blockIdx.y];
  const int64_t M = d.a.M, N = d.a.N, K = d.a.K;
  const int64_t total = M + N + K;
  int64_t *mL = const_cast<int64_t *>(d.a.mL), *mD = const_cast<int64_t *>(d.a.mD);
  int64_t *nR = const_cast<int64_t *>(d.a.nR), *nD = const_cast<int64_t *>(d.a.nD);
  int64_t *kL = const_cast<int64_t *>(d.a.kL), *kR = const_cast<int64_t *>(d.a.kR);
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < total; i += (int64_t)gridDim.x * 256) {
    if (i < M) {
      int64_t r = i, x = 0, y = 0;
      for (int g = 0; g < d.nm; ++g) {
        const int64_t c = r % d.mext[g];
        r /= d.mext[g];
        x += c * d.mstrL[g];
        y += c * d.mstrD[g];
      }
      mL[i] = x;
      mD[i] = y;
    } else if (i < M + N) {
      int64_t r = i - M, x = 0, y = 0;
      for (int g = 0; g < d.nn; ++g) {
        const int64_t c = r % d.next[g];
        r /= d.next[g];
        x += c * d.nstrR[g];
        y += c * d.nstrD[g];
      }
      nR[i - M] = x;
      nD[i - M] = y;
    } else {
      int64_t r = i - M - N, x = 0, y = 0;
      for (int g = 0; g < d.nk; ++g) {
        const int64_t c = r % d.kext[g];
        r /= d.kext[g];
        x += c * d.kstrL[g];
        y += c * d.kstrR[g];
      }
      kL[i - M - N] = x;
      kR[i - M - N] = y;
    }
  }
}

// Task owning flat tile w: largest j with prefix[j] <= w.
__device__ __forceinline__ int find_task(const int64_t *prefix, int n, int64_t w) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= w) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Dynamic work distribution: CTAs take the next flat tile from a counter; the
// host orders the tasks by decreasing K (longest tiles first).
__device__ __forceinline__ int64_t next_item(unsigned long long *ctr) {
  __shared__ int64_t item;
  __syncthreads();
  if (threadIdx.x == 0) item = (int64_t)atomicAdd(ctr, 1ull);
  __syncthreads();
  return item;
}

// Resident CTAs per SM asked of the compiler for the persistent batch kernels.
template <int BM, int BN> struct BatchOcc { static constexpr int D = 1, Z = 1; };
template <> struct BatchOcc<64, 64> { static constexpr int D = 3, Z = 2; };
template <> struct BatchOcc<32, 32> { static constexpr int D = 6, Z = 5; };

template <int BM, int BN>
__global__ void __launch_bounds__(DmmaCfg<BM, BN>::THREADS, BatchOcc<BM, BN>::D)
    dmma_batch_kernel(const BatchDesc *descs, const int32_t *list, const int64_t *prefix, int n,
                      int64_t total, unsigned long long *ctr) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int64_t w = next_item(ctr); w < total; w = next_item(ctr)) {
    const int j = find_task(prefix, n, w);
    const BatchDesc &d = descs[list[j]];
    const GemmArgs a = d.a;
    const int local = (int)(w - prefix[j]);
    dmma_tile<BM, BN>((const double *)d.L, (const double *)d.R, (double *)d.D, a, local % a.tiles_m,
                      local / a.tiles_m, smem);
  }
}

template <int BM, int BN>
__global__ void __launch_bounds__(ZmmaCfg<BM, BN>::THREADS, BatchOcc<BM, BN>::Z)
    zmma_batch_kernel(const BatchDesc *descs, const int32_t *list, const int64_t *prefix, int n,
                      int64_t total, unsigned long long *ctr) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (int64_t w = next_item(ctr); w < total; w = next_item(ctr)) {
    const int j = find_task(prefix, n, w);
    const BatchDesc &d = descs[list[j]];
    const GemmArgs a = d.a;
    const int local = (int)(w - prefix[j]);
    zmma_tile<BM, BN>((const double2 *)d.L, (const double2 *)d.R, (double2 *)d.D, a, local % a.tiles_m,
                      local / a.tiles_m, smem);
  }
}

template <typename T>
__global__ void __launch_bounds__(kSThreads)
    simt_batch_kernel(const BatchDesc *descs, const int32_t *list, const int64_t *prefix, int n,
                      int64_t total, unsigned long long *ctr) {
  for (int64_t w = next_item(ctr); w < total; w = next_item(ctr)) {
    const int j = find_task(prefix, n, w);
    const BatchDesc &d = descs[list[j]];
    const GemmArgs a = d.a;
    const int local = (int)(w - prefix[j]);
    simt_tile<T>((const T *)d.L, (const T *)d.R, (T *)d.D, a, local % a.tiles_m, local / a.tiles_m);
  }
}

struct BatchPlan {
  std::vector<BatchDesc> descs;
  std::vector<int> cfg;          // per task: configuration, or -1 = single-task fallback
  std::vector<int64_t> tab_off;  // per task: offset of its tables (int64 elements)
  std::vector<size_t> fb_scratch;
  std::vector<size_t> fb_off;
  std::vector<int32_t> list[kNumCfg];
  std::vector<int64_t> prefix[kNumCfg];
  size_t off_desc = 0, off_list[kNumCfg] = {}, off_prefix[kNumCfg] = {}, off_tab = 0, off_fb = 0, off_ctr = 0,
         total = 0;
};

// Tile choices of the autotuner (tcTensorContractBatchTune) per task class:
// kind (R8, C8) x bucket of M x bucket of N, buckets < 16, < 48, < 128, >= 128.
// 0 = not tuned (the shape rule below applies), else the tile edge (32 or 64).
constexpr int kTuneBuckets = 4;
std::atomic<int> g_tune[2][kTuneBuckets][kTuneBuckets];

int tune_bucket(int64_t x) { return x < 16 ? 0 : x < 48 ? 1 : x < 128 ? 2 : 3; }

int batch_cfg_of(int kind, int64_t M, int64_t N) {
  if (kind == R8 || kind == C8) {
    const int t = g_tune[kind == C8][tune_bucket(M)][tune_bucket(N)].load(std::memory_order_relaxed);
    if (t == 32) return kind == R8 ? kCfgD32 : kCfgZ32;
    if (t == 64) return kind == R8 ? kCfgD64 : kCfgZ64;
  }
  switch (kind) {
    case R8: return (M >= 48 && N >= 48) ? kCfgD64 : kCfgD32;
    case C8: return (M >= 48 && N >= 48) ? kCfgZ64 : kCfgZ32;
    case R4: return kCfgS4;
    default: return kCfgS14;
  }
}

int batch_plan(int ntasks, const tcContractTask *tasks, BatchPlan &bp) {
  if (ntasks < 0 || ntasks > 65535 || (ntasks > 0 && tasks == nullptr)) return TALSH_INVALID_ARGS;
  bp.descs.assign(ntasks, BatchDesc());
  bp.cfg.assign(ntasks, -1);
  bp.tab_off.assign(ntasks, 0);
  bp.fb_scratch.assign(ntasks, 0);
  bp.fb_off.assign(ntasks, 0);
  int64_t tab = 0;
  for (int t = 0; t < ntasks; ++t) {
    const tcContractTask &x = tasks[t];
    if (x.drank > TC_BATCH_MAX_RANK || x.lrank > TC_BATCH_MAX_RANK || x.rrank > TC_BATCH_MAX_RANK)
      return TALSH_INVALID_ARGS;
    int rc = check_args(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims);
    if (rc) return rc;
    if (x.D == nullptr || x.L == nullptr || x.R == nullptr) return TALSH_INVALID_ARGS;
    if (!elements_aligned(x.data_kind, x.D, x.L, x.R)) return TALSH_INVALID_ARGS;
    Analysis an;
    bool batchable = x.lrank > 0 && x.rrank > 0;  // a full contraction (D of rank 0) is a 1 x 1 GEMM
    if (batchable) {
      if ((rc = analyze(x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims, an)) != 0) return rc;
      batchable = !an.hyper && an.T.nm <= kBMaxG && an.T.nn <= kBMaxG && an.T.nk <= kBMaxG &&
                  an.T.M <= 0x7fffffffLL && an.T.N <= 0x7fffffffLL && an.T.K <= 0x7fffffffLL;
    }
    if (!batchable) {  // scalar operands, hyper-indices: single-task path
      bp.fb_scratch[t] = contract_scratch_bytes(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims,
                                                x.rrank, x.rdims);
      continue;
    }
    const TableParams &T = an.T;
    BatchDesc &d = bp.descs[t];
    d.nm = T.nm; d.nn = T.nn; d.nk = T.nk;
    for (int g = 0; g < T.nm; ++g) { d.mext[g] = (int32_t)T.mext[g]; d.mstrL[g] = T.mstrL[g]; d.mstrD[g] = T.mstrD[g]; }
    for (int g = 0; g < T.nn; ++g) { d.next[g] = (int32_t)T.next[g]; d.nstrR[g] = T.nstrR[g]; d.nstrD[g] = T.nstrD[g]; }
    for (int g = 0; g < T.nk; ++g) { d.kext[g] = (int32_t)T.kext[g]; d.kstrL[g] = T.kstrL[g]; d.kstrR[g] = T.kstrR[g]; }
    const bool cplx = kind_is_complex(x.data_kind);
    int cl = 0, cr = 0;
    if (cplx) {
      int cb = x.conj_bits & 7;
      if (cb & 1) cb ^= 7;
      cl = (cb >> 1) & 1;
      cr = (cb >> 2) & 1;
    }
    GemmArgs &a = d.a;
    std::memset(&a, 0, sizeof(a));
    a.M = (int)T.M; a.N = (int)T.N; a.K = (int)T.K;
    a.alpha_re = x.alpha_re; a.alpha_im = cplx ? x.alpha_im : 0.0;
    a.beta = x.accumulative ? 1 : 0;
    a.a_along_m = an.a_along_m ? 1 : 0;
    a.b_along_n = an.b_along_n ? 1 : 0;
    a.conj_l = cl; a.conj_r = cr;
    d.L = x.L; d.R = x.R; d.D = x.D;
    const int c = batch_cfg_of(x.data_kind, T.M, T.N);
    const int bm = cfg_tile(c), bn = bm;
    a.tiles_m = (int)((T.M + bm - 1) / bm);
    const int64_t tiles = (int64_t)a.tiles_m * ((T.N + bn - 1) / bn);
    bp.cfg[t] = c;
    bp.tab_off[t] = tab;
    tab += 2 * (T.M + T.N + T.K);
    bp.list[c].push_back(t);
    (void)tiles;
  }
  // Longest tiles (largest K) first, then the tile prefix sums.
  for (int c = 0; c < kNumCfg; ++c) {
    auto &l = bp.list[c];
    std::stable_sort(l.begin(), l.end(), [&](int x, int y) { return bp.descs[x].a.K > bp.descs[y].a.K; });
    auto &pl = bp.prefix[c];
    if (l.empty()) continue;
    pl.push_back(0);
    for (int t : l) {
      const GemmArgs &a = bp.descs[t].a;
      const int bn = cfg_tile(c);
      pl.push_back(pl.back() + (int64_t)a.tiles_m * ((a.N + bn - 1) / bn));
    }
  }
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 255) & ~size_t(255); return o; };
  bp.off_desc = take(sizeof(BatchDesc) * (size_t)std::max(ntasks, 1));
  for (int c = 0; c < kNumCfg; ++c) {
    bp.off_list[c] = take(sizeof(int32_t) * bp.list[c].size());
    bp.off_prefix[c] = take(sizeof(int64_t) * bp.prefix[c].size());
  }
  bp.off_tab = take(sizeof(int64_t) * (size_t)tab);
  bp.off_ctr = take(sizeof(unsigned long long) * kNumCfg);
  for (int t = 0; t < ntasks; ++t)
    if (bp.cfg[t] < 0) bp.fb_off[t] = take(bp.fb_scratch[t]);
  bp.total = off;
  return TALSH_SUCCESS;
}

using BatchKernel = void (*)(const BatchDesc *, const int32_t *, const int64_t *, int, int64_t,
                             unsigned long long *);

// Persistent launch of one tensor-pipe batch kernel: as many CTAs as fit at once.
int launch_tc_batch(BatchKernel k, int threads, size_t smem, const char *name, const BatchPlan &bp, int c,
                    char *base, cudaStream_t st) {
  const int64_t total = bp.prefix[c].back();
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, threads, smem) != cudaSuccess || bps < 1) bps = 1;
  cudaGetLastError();
  const int64_t grid = std::min<int64_t>(total, (int64_t)sm_count_dev() * bps);
  k<<<(unsigned)grid, threads, smem, st>>>(
      (const BatchDesc *)(base + bp.off_desc), (const int32_t *)(base + bp.off_list[c]),
      (const int64_t *)(base + bp.off_prefix[c]), (int)bp.list[c].size(), total,
      (unsigned long long *)(base + bp.off_ctr) + c);
  note_launch();
  return check_launch(name);
}

template <int BM, int BN>
int launch_dmma_batch(const BatchPlan &bp, int c, char *base, cudaStream_t st) {
  using C = DmmaCfg<BM, BN>;
  static std::atomic<uint64_t> attr{0};
  once_per_device(attr, [] {
    cudaFuncSetAttribute(dmma_batch_kernel<BM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    cudaFuncSetAttribute(dmma_batch_kernel<BM, BN>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  });
  return launch_tc_batch(dmma_batch_kernel<BM, BN>, C::THREADS, C::SMEM, "dmma_batch_kernel", bp, c, base, st);
}

template <int BM, int BN>
int launch_zmma_batch(const BatchPlan &bp, int c, char *base, cudaStream_t st) {
  using Z = ZmmaCfg<BM, BN>;
  static std::atomic<uint64_t> attr{0};
  once_per_device(attr, [] {
    cudaFuncSetAttribute(zmma_batch_kernel<BM, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Z::SMEM);
    cudaFuncSetAttribute(zmma_batch_kernel<BM, BN>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  });
  return launch_tc_batch(zmma_batch_kernel<BM, BN>, Z::THREADS, Z::SMEM, "zmma_batch_kernel", bp, c, base, st);
}

template <typename T>
int launch_simt_batch(const BatchPlan &bp, int c, char *base, cudaStream_t st) {
  const int64_t total = bp.prefix[c].back();
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, simt_batch_kernel<T>, kSThreads, 0) != cudaSuccess ||
      bps < 1)
    bps = 1;
  cudaGetLastError();
  const int64_t grid = std::min<int64_t>(total, (int64_t)sm_count_dev() * bps);
  simt_batch_kernel<T><<<(unsigned)grid, kSThreads, 0, st>>>(
      (const BatchDesc *)(base + bp.off_desc), (const int32_t *)(base + bp.off_list[c]),
      (const int64_t *)(base + bp.off_prefix[c]), (int)bp.list[c].size(), total,
      (unsigned long long *)(base + bp.off_ctr) + c);
  note_launch();
  return check_launch("simt_batch_kernel");
}

}  // namespace
}  // namespace tb

namespace tb {
namespace {

// Uploads the descriptors, work lists and prefix sums (the scratch bytes below
// off_tab) as one copy, then launches the table build, one persistent kernel
// per configuration and the single-task fallbacks.  `stage`, when given, is a
// pinned host block of at least off_tab bytes that stays untouched until the
// copy has run; otherwise the block is packed in pageable memory.
int batch_run(int ntasks, const tcContractTask *tasks, BatchPlan &bp, void *scratch, size_t scratch_bytes,
              void *stage, cudaStream_t st) {
  if (scratch == nullptr || scratch_bytes < bp.total) return TALSH_INVALID_ARGS;
  char *base = (char *)scratch;
  int64_t *tabs = (int64_t *)(base + bp.off_tab);
  int64_t max_entries = 0;
  for (int t = 0; t < ntasks; ++t) {
    if (bp.cfg[t] < 0) continue;
    GemmArgs &a = bp.descs[t].a;
    int64_t *p = tabs + bp.tab_off[t];
    a.mL = p; a.mD = p + a.M; a.nR = a.mD + a.M; a.nD = a.nR + a.N; a.kL = a.nD + a.N; a.kR = a.kL + a.K;
    max_entries = std::max<int64_t>(max_entries, (int64_t)a.M + a.N + a.K);
  }
  std::vector<char> pageable;
  char *host = (char *)stage;
  if (host == nullptr) {
    pageable.assign(bp.off_tab, 0);
    host = pageable.data();
  }
  std::memcpy(host + bp.off_desc, bp.descs.data(), sizeof(BatchDesc) * ntasks);
  for (int c = 0; c < kNumCfg; ++c) {
    if (bp.list[c].empty()) continue;
    std::memcpy(host + bp.off_list[c], bp.list[c].data(), sizeof(int32_t) * bp.list[c].size());
    std::memcpy(host + bp.off_prefix[c], bp.prefix[c].data(), sizeof(int64_t) * bp.prefix[c].size());
  }
  cudaError_t e = cudaMemcpyAsync(base, host, bp.off_tab, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + bp.off_ctr, 0, sizeof(unsigned long long) * kNumCfg, st);
  if (e != cudaSuccess) {
    note_cuda_error("batch descriptor upload", (int)e);
    return TALSH_FAILURE;
  }
  int rc;
  if (max_entries > 0) {
    const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((max_entries + 255) / 256, 64));
    batch_tables_kernel<<<dim3(gx, ntasks), 256, 0, st>>>((const BatchDesc *)(base + bp.off_desc));
    note_launch();
    if ((rc = check_launch("batch_tables_kernel")) != 0) return rc;
  }
  if (!bp.list[kCfgD64].empty() && (rc = launch_dmma_batch<64, 64>(bp, kCfgD64, base, st)) != 0) return rc;
  if (!bp.list[kCfgD32].empty() && (rc = launch_dmma_batch<32, 32>(bp, kCfgD32, base, st)) != 0) return rc;
  if (!bp.list[kCfgZ64].empty() && (rc = launch_zmma_batch<64, 64>(bp, kCfgZ64, base, st)) != 0) return rc;
  if (!bp.list[kCfgZ32].empty() && (rc = launch_zmma_batch<32, 32>(bp, kCfgZ32, base, st)) != 0) return rc;
  if (!bp.list[kCfgS4].empty() && (rc = launch_simt_batch<float>(bp, kCfgS4, base, st)) != 0) return rc;
  if (!bp.list[kCfgS14].empty() && (rc = launch_simt_batch<float2>(bp, kCfgS14, base, st)) != 0) return rc;
  for (int t = 0; t < ntasks; ++t) {
    if (bp.cfg[t] >= 0) continue;
    const tcContractTask &x = tasks[t];
    rc = contract_launch(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims, x.D, x.L,
                         x.R, x.alpha_re, x.alpha_im, x.conj_bits, x.accumulative,
                         bp.fb_scratch[t] ? base + bp.fb_off[t] : nullptr, bp.fb_scratch[t], (void *)st);
    if (rc) return rc;
  }
  return TALSH_SUCCESS;
}

}  // namespace

// Upper bound of one task's share of a batch's scratch: its descriptor, work
// list and prefix entries, and its offset tables or single-task fallback
// scratch.  A batch needs the sum over its tasks plus batch_fixed_scratch().
size_t batch_task_scratch_bound(const tcContractTask &x) {
  const size_t fb = contract_scratch_bytes(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank,
                                           x.rdims);
  return sizeof(BatchDesc) + sizeof(int32_t) + sizeof(int64_t) + fb + 256;
}

size_t batch_fixed_scratch() { return (size_t)(2 * kNumCfg + 4) * 256 + sizeof(unsigned long long) * kNumCfg; }

// Plans a batch, asks `get` for device scratch and a pinned staging block of
// the sizes the plan needs (get returns nullptr to refuse: TRY_LATER), and
// launches it on `stream`.
int batch_launch_with(int ntasks, const tcContractTask *tasks, BatchScratchFn get, void *ctx, void *stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (ntasks == 0) return TALSH_SUCCESS;
  BatchPlan bp;
  int rc = batch_plan(ntasks, tasks, bp);
  if (rc) return rc;
  void *stage = nullptr;
  void *scratch = get(ctx, bp.total, bp.off_tab, &stage);
  if (scratch == nullptr) return TRY_LATER;
  return batch_run(ntasks, tasks, bp, scratch, bp.total, stage, st);
}

}  // namespace tb

extern "C" size_t tcTensorContractBatchScratch(int ntasks, const tcContractTask *tasks) {
  tb::BatchPlan bp;
  if (tb::batch_plan(ntasks, tasks, bp) != TALSH_SUCCESS) return 0;
  return bp.total;
}

extern "C" int tcTensorContractBatch(int ntasks, const tcContractTask *tasks, void *scratch,
                                     size_t scratch_bytes, void *stream) {
  if (ntasks == 0) return TALSH_SUCCESS;
  tb::BatchPlan bp;
  const int rc = tb::batch_plan(ntasks, tasks, bp);
  if (rc) return rc;
  return tb::batch_run(ntasks, tasks, bp, scratch, scratch_bytes, nullptr, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Graph-captured batches: the plan, the descriptor upload and the offset
// tables are done once at creation; the GEMM work is captured in one CUDA
// graph -- a reset of the work counters, then the persistent kernel of every
// tile configuration (and the single-task fallbacks) as concurrent branches,
// so one configuration's tail overlaps the others' work -- and replayed with
// one launch.  Each tile still runs the code of the single-task kernels, so a
// replay's results equal tcTensorContractBatch's bit for bit.
// ---------------------------------------------------------------------------
struct tcContractBatchGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int ntasks = 0;
  unsigned launches = 0;
};

extern "C" int tcContractBatchGraphCreate(int ntasks, const tcContractTask *tasks, void *scratch,
                                          size_t scratch_bytes, void *stream, tcContractBatchGraph **out) {
  using namespace tb;
  if (out == nullptr) return TALSH_INVALID_ARGS;
  *out = nullptr;
  if (ntasks < 1) return TALSH_INVALID_ARGS;
  BatchPlan bp;
  int rc = batch_plan(ntasks, tasks, bp);
  if (rc) return rc;
  if (scratch == nullptr || scratch_bytes < bp.total) return TALSH_INVALID_ARGS;
  cudaStream_t st = (cudaStream_t)stream;
  char *base = (char *)scratch;
  // Descriptors, lists and prefix sums, then the offset tables, once.
  int64_t *tabs = (int64_t *)(base + bp.off_tab);
  int64_t max_entries = 0;
  for (int t = 0; t < ntasks; ++t) {
    if (bp.cfg[t] < 0) continue;
    GemmArgs &a = bp.descs[t].a;
    int64_t *p = tabs + bp.tab_off[t];
    a.mL = p; a.mD = p + a.M; a.nR = a.mD + a.M; a.nD = a.nR + a.N; a.kL = a.nD + a.N; a.kR = a.kL + a.K;
    max_entries = std::max<int64_t>(max_entries, (int64_t)a.M + a.N + a.K);
  }
  std::vector<char> host(bp.off_tab, 0);
  std::memcpy(host.data() + bp.off_desc, bp.descs.data(), sizeof(BatchDesc) * ntasks);
  for (int c = 0; c < kNumCfg; ++c) {
    if (bp.list[c].empty()) continue;
    std::memcpy(host.data() + bp.off_list[c], bp.list[c].data(), sizeof(int32_t) * bp.list[c].size());
    std::memcpy(host.data() + bp.off_prefix[c], bp.prefix[c].data(), sizeof(int64_t) * bp.prefix[c].size());
  }
  cudaError_t e = cudaMemcpyAsync(base, host.data(), bp.off_tab, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    note_cuda_error("batch graph descriptor upload", (int)e);
    return TALSH_FAILURE;
  }
  if (max_entries > 0) {
    const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((max_entries + 255) / 256, 64));
    batch_tables_kernel<<<dim3(gx, ntasks), 256, 0, st>>>((const BatchDesc *)(base + bp.off_desc));
    note_launch();
    if ((rc = check_launch("batch_tables_kernel")) != 0) return rc;
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {  // the host block above goes out of scope
    note_cuda_error("batch graph setup", (int)e);
    return TALSH_FAILURE;
  }
  // Capture on a private stream: counters reset, then one branch per
  // configuration and one for the fallbacks, joined at the end.
  cudaStream_t cs = nullptr;
  std::vector<cudaStream_t> br;
  std::vector<cudaEvent_t> ev;
  cudaGraph_t graph = nullptr;
  unsigned launches = 0;
  auto cleanup = [&]() {
    for (auto x : ev) cudaEventDestroy(x);
    for (auto x : br) cudaStreamDestroy(x);
    if (cs) cudaStreamDestroy(cs);
    cudaGetLastError();
  };
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) { cleanup(); return TALSH_FAILURE; }
  std::vector<int> used;
  for (int c = 0; c < kNumCfg; ++c)
    if (!bp.list[c].empty()) used.push_back(c);
  bool fallbacks = false;
  for (int t = 0; t < ntasks; ++t) fallbacks = fallbacks || bp.cfg[t] < 0;
  const int nbr = (int)used.size() + (fallbacks ? 1 : 0);
  br.assign(nbr, nullptr);
  ev.assign(nbr + 1, nullptr);
  for (auto &x : br)
    if (cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking) != cudaSuccess) { cleanup(); return TALSH_FAILURE; }
  for (auto &x : ev)
    if (cudaEventCreateWithFlags(&x, cudaEventDisableTiming) != cudaSuccess) { cleanup(); return TALSH_FAILURE; }
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) { cleanup(); return TALSH_FAILURE; }
  e = cudaMemsetAsync(base + bp.off_ctr, 0, sizeof(unsigned long long) * kNumCfg, cs);
  cudaEventRecord(ev[nbr], cs);
  for (int b = 0; b < nbr; ++b) cudaStreamWaitEvent(br[b], ev[nbr], 0);
  const unsigned before = (unsigned)tcKernelLaunchCount();
  for (size_t b = 0; b < used.size() && rc == TALSH_SUCCESS && e == cudaSuccess; ++b) {
    const int c = used[b];
    cudaStream_t s2 = br[b];
    switch (c) {
      case kCfgD64: rc = launch_dmma_batch<64, 64>(bp, c, base, s2); break;
      case kCfgD32: rc = launch_dmma_batch<32, 32>(bp, c, base, s2); break;
      case kCfgZ64: rc = launch_zmma_batch<64, 64>(bp, c, base, s2); break;
      case kCfgZ32: rc = launch_zmma_batch<32, 32>(bp, c, base, s2); break;
      case kCfgS4: rc = launch_simt_batch<float>(bp, c, base, s2); break;
      default: rc = launch_simt_batch<float2>(bp, c, base, s2); break;
    }
  }
  for (int t = 0; t < ntasks && fallbacks && rc == TALSH_SUCCESS && e == cudaSuccess; ++t) {
    if (bp.cfg[t] >= 0) continue;
    const tcContractTask &x = tasks[t];
    rc = contract_launch(x.data_kind, x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims, x.D, x.L,
                         x.R, x.alpha_re, x.alpha_im, x.conj_bits, x.accumulative,
                         bp.fb_scratch[t] ? base + bp.fb_off[t] : nullptr, bp.fb_scratch[t], (void *)br[nbr - 1]);
  }
  launches = (unsigned)tcKernelLaunchCount() - before;
  for (int b = 0; b < nbr; ++b) {
    cudaEventRecord(ev[b], br[b]);
    cudaStreamWaitEvent(cs, ev[b], 0);
  }
  const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
  if (rc == TALSH_SUCCESS && (e != cudaSuccess || ce != cudaSuccess)) {
    note_cuda_error("batch graph capture", (int)(e != cudaSuccess ? e : ce));
    rc = TALSH_FAILURE;
  }
  cudaGraphExec_t exec = nullptr;
  if (rc == TALSH_SUCCESS && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
    note_error_text("batch graph instantiation failed");
    rc = TALSH_FAILURE;
  }
  cleanup();
  if (rc != TALSH_SUCCESS) {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  tcContractBatchGraph *g = new tcContractBatchGraph();
  g->graph = graph;
  g->exec = exec;
  g->ntasks = ntasks;
  g->launches = launches;
  *out = g;
  return TALSH_SUCCESS;
}

extern "C" int tcContractBatchGraphLaunch(tcContractBatchGraph *g, void *stream) {
  if (g == nullptr) return TALSH_INVALID_ARGS;
  const cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    tb::note_cuda_error("tcContractBatchGraphLaunch", (int)e);
    return TALSH_FAILURE;
  }
  tb::note_launch(g->launches);
  return TALSH_SUCCESS;
}

extern "C" int tcContractBatchGraphDestroy(tcContractBatchGraph *g) {
  if (g == nullptr) return TALSH_INVALID_ARGS;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return TALSH_SUCCESS;
}

// Autotuner: for every class present among the tasks, runs that class's tasks
// as one batch with each candidate tile (32x32, 64x64), `reps` times each,
// timed with events on `stream`, and keeps the faster tile for the class.
extern "C" int tcTensorContractBatchTune(int ntasks, const tcContractTask *tasks, void *scratch,
                                         size_t scratch_bytes, void *stream, int reps) {
  using namespace tb;
  if (ntasks < 0 || (ntasks > 0 && tasks == nullptr) || reps < 1) return TALSH_INVALID_ARGS;
  if (scratch_bytes < tcTensorContractBatchScratch(ntasks, tasks)) return TALSH_INVALID_ARGS;
  std::vector<int> cls[2][kTuneBuckets][kTuneBuckets];
  for (int t = 0; t < ntasks; ++t) {
    const tcContractTask &x = tasks[t];
    if (x.data_kind != R8 && x.data_kind != C8) continue;
    if (x.lrank == 0 || x.rrank == 0) continue;
    Analysis an;
    if (analyze(x.cptrn, x.drank, x.ddims, x.lrank, x.ldims, x.rrank, x.rdims, an) != 0 || an.hyper) continue;
    cls[x.data_kind == C8][tune_bucket(an.T.M)][tune_bucket(an.T.N)].push_back(t);
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return TALSH_FAILURE;
  }
  int rc = TALSH_SUCCESS;
  std::vector<tcContractTask> sub;
  for (int k = 0; k < 2 && rc == TALSH_SUCCESS; ++k)
    for (int mb = 0; mb < kTuneBuckets && rc == TALSH_SUCCESS; ++mb)
      for (int nb = 0; nb < kTuneBuckets && rc == TALSH_SUCCESS; ++nb) {
        const std::vector<int> &ids = cls[k][mb][nb];
        if (ids.empty()) continue;
        sub.clear();
        for (int t : ids) sub.push_back(tasks[t]);
        float best_ms = 0.0f;
        int best = 0;
        for (int edge : {32, 64}) {
          g_tune[k][mb][nb].store(edge);
          float ms = 0.0f;
          for (int r = 0; r <= reps && rc == TALSH_SUCCESS; ++r) {  // the first run warms up
            cudaEventRecord(e0, st);
            rc = tcTensorContractBatch((int)sub.size(), sub.data(), scratch, scratch_bytes, stream);
            cudaEventRecord(e1, st);
            if (rc == TALSH_SUCCESS && cudaEventSynchronize(e1) != cudaSuccess) rc = TALSH_FAILURE;
            float dt = 0.0f;
            if (rc == TALSH_SUCCESS && r > 0 && cudaEventElapsedTime(&dt, e0, e1) == cudaSuccess) ms += dt;
          }
          if (rc != TALSH_SUCCESS) break;
          if (best == 0 || ms < best_ms) { best_ms = ms; best = edge; }
        }
        g_tune[k][mb][nb].store(rc == TALSH_SUCCESS ? best : 0);
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  return rc;
}

// Tile edge the autotuner chose for a class (0: not tuned), or -1 for a bad class.
extern "C" int tcTensorContractBatchTuned(int data_kind, int m_bucket, int n_bucket) {
  using namespace tb;
  if ((data_kind != R8 && data_kind != C8) || m_bucket < 0 || m_bucket >= kTuneBuckets || n_bucket < 0 ||
      n_bucket >= kTuneBuckets)
    return -1;
  return g_tune[data_kind == C8][m_bucket][n_bucket].load();
}

// Forgets every tuned choice (the shape rule applies again).
extern "C" void tcTensorContractBatchTuneReset(void) {
  using namespace tb;
  for (auto &a : g_tune)
    for (auto &b : a)
      for (auto &c : b) c.store(0);
}
