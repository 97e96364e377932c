// Dense tensor permutation (transpose) and fused permute-add for sm_100a.
//
// Semantics follow the reference tensor_block_copy / tensor_block_add
// (tensor_algebra_cpu.F90:3151-3310, :3312-3673): out[O2N(idx)] = in[idx] over
// column-major bodies, and d = d + l*s with one rounding per operation.
//
// Design (written for B200, not a translation of the reference's
// gpu_tensor_block_copy_dlf__):
//  * Host planning fuses dimensions that stay adjacent, drops unit extents and
//    picks a tile = (input-minor group A) x (output-minor group B).  Both
//    groups are prefixes of their tensor's dimension order, so every tile is a
//    set of contiguous runs on the read side (length Li) and on the write side
//    (length Lo): reads and writes are coalesced for any permutation and any
//    extents, including odd ones.
//  * A persistent grid (SMs x resident CTAs) walks the tiles.  Each CTA stages
//    one tile in shared memory: all loads of a thread are issued before its
//    shared stores (memory-level parallelism), then the tile is written out
//    along the output runs.  Per-run offset tables are built once per CTA.
//  * 128-bit global accesses on each side whenever the host proves alignment
//    of every run start and run length; scalar accesses otherwise.
//  * The add variant reads D in the write phase and applies d + l*s with
//    explicit round-to-nearest intrinsics (no FMA contraction), which is
//    bit-exact with the reference CPU arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "common.h"

namespace tb {
namespace {

constexpr int kThreads = 256;
constexpr int kMinBlocks = 3;      // resident CTAs per SM the register budget is sized for
constexpr int kMaxFR = 40;         // max fused rank (every fused extent is >= 2)
constexpr int kTileBytes = 32768;  // byte budget of one tile buffer (kStages buffers per CTA)
constexpr int kMaxTabLo = 4096;    // output run length when B needs a table (more than 3 dims)
constexpr int kMaxRuns = 1024;     // run count bound (run tables live in shared memory)
constexpr int kStages = 3;              // tile buffers per CTA of permute_tiled_kernel: loads run 2 tiles ahead

// Tile buffers per CTA of permute_reg_kernel, by element size and operation:
// loads run S - 1 tiles ahead of the write phase.  Adds also prefetch the D
// vectors each thread will update into a private shared slot of the same stage
// (kAddPrefetch), so the write phase waits on no global load.
#ifndef TB_STAGES_COPY4
#define TB_STAGES_COPY4 3
#endif
#ifndef TB_STAGES_COPY8
#define TB_STAGES_COPY8 3
#endif
#ifndef TB_STAGES_ADD4
#define TB_STAGES_ADD4 3
#endif
#ifndef TB_STAGES_ADD8
#define TB_STAGES_ADD8 3
#endif
#ifndef TB_ADD_PREFETCH
#define TB_ADD_PREFETCH 1
#endif
#ifndef TB_MIN_BLOCKS8
#define TB_MIN_BLOCKS8 3  // resident CTAs per SM the K = 8 register budget is sized for
#endif
#ifndef TB_COPY_INPUT_MAJOR
#define TB_COPY_INPUT_MAJOR 0  // 1: copies walk their tiles in input order, as adds do
#endif
constexpr bool kAddPrefetch = TB_ADD_PREFETCH != 0;
__host__ __device__ constexpr int reg_stages(int esize, int op) {
  return op == 1 ? (esize <= 4 ? TB_STAGES_ADD4 : TB_STAGES_ADD8)
                 : (esize <= 4 ? TB_STAGES_COPY4 : TB_STAGES_COPY8);
}

// Mixed-radix decomposition of an index over up to 3 tile dimensions with
// precomputed magic divisors; groups of more dimensions use shared tables.
struct GroupMap {
  int n;              // dimensions (0..3), or -1: use the shared table
  int32_t ext[3];     // tile extents
  uint32_t mg[2], sh[2];
  int64_t gstr[3];    // global strides (input for read runs, output for write runs)
  int32_t sstr[3];    // shared-memory strides
  int mask;           // which coordinate is the partially covered split dimension (-1: none)
};

struct PermParams {
  int rank;
  int V, Li, Lo, Ri, Ro, Li_pad;
  uint32_t mg_li, sh_li, mg_lo, sh_lo;
  int a_last, b_last, a_pre, b_pre;
  int a_in_B, b_in_A;
  int y_step;         // 1: the VOUT elements y..y+VOUT-1 share all but the first B coordinate
  int swz;            // 1: shared indices are bank-swizzled (Li_pad == Li), 0: rows padded to Li_pad
  int nv;             // vectors (VOUT elements) per output run
  uint32_t mg_nv, sh_nv;
  int ytab;           // 1: output-run positions come from the shared table ySm
  GroupMap rmap, wmap, ymap;
  int nra, nwb, nb;
  int conj;
  int off_rin, off_rc, off_wout, off_wsm, off_wc, off_ysm, off_tab_end;
  int reg;            // 1: permute_reg_kernel (per-thread register tables)
  int ta_rem, tb_rem; // extents of the last (cut-short) tile along a_last / b_last
  int pre_bA, pre_aB; // tile volume of A below b_last (b_last in A) / of B before a_last (a_last in B)
  int buf_elems;      // elements per tile buffer (whole 128-byte rows)
  int bulk;           // 1: permute_bulk_kernel (input runs moved by bulk copies)
  int pitch_b;        // bulk form: bytes between the rows of a tile buffer (a multiple of 16)
  uint32_t mg_lip, sh_lip;  // magic divisor of Li_pad
  int64_t num_tiles;
  double s_re, s_im;
  const void *sdev;  // optional device scalar multiplying the scale (rank-0 operand)
  int sdev_kind, sdev_conj;
  int64_t ext[kMaxFR];
  int64_t istr[kMaxFR];
  int64_t ostr[kMaxFR];
  int64_t ntile[kMaxFR];
  uint32_t mg_ts[kMaxFR], sh_ts[kMaxFR];  // magic divisors of the tile-index stride of each dimension
  uint32_t mg_nt[kMaxFR], sh_nt[kMaxFR];  // and of its tile count
  int32_t tl[kMaxFR];
  int32_t smstr[kMaxFR];
  int8_t ra_dims[kMaxFR];
  int8_t wb_dims[kMaxFR];
  int8_t b_dims[kMaxFR];
};

struct TileSetup {
  int64_t in_base, out_base;
  int li_act, lo_act, ta_lim, tb_lim;
  int full;  // 1: no split dimension is cut short in this tile (no masking needed)
  int type;  // bit 0: a_last cut short, bit 1: b_last cut short
};

// Fast unsigned division for n < 2^31 (Granlund-Montgomery round-up method).
void make_magic(uint32_t d, uint32_t &mg, uint32_t &sh) {
  uint32_t s = 0;
  while ((1ull << s) < d) ++s;
  mg = (uint32_t)(((1ull << 32) * ((1ull << s) - d)) / d + 1ull);
  sh = s;
}
__device__ __forceinline__ uint32_t fast_div(uint32_t n, uint32_t mg, uint32_t sh) {
  return (__umulhi(n, mg) + n) >> sh;
}

// Bank swizzle of a shared-memory element index: the position inside each
// 128-byte row is XORed with a fold of the row number.  It is a bijection on
// every row, keeps unit-stride accesses conflict-free and spreads power-of-two
// strides (the output-run stride inside an input run) over all banks.
template <typename T>
__device__ __forceinline__ int swz(int idx) {
  constexpr int SB = sizeof(T) == 4 ? 5 : (sizeof(T) == 8 ? 4 : 3);  // log2(elements per row)
  const int row = idx >> SB;
  return idx ^ ((row ^ (row >> SB)) & ((1 << SB) - 1));
}

struct Coords {
  int64_t goff;
  int32_t soff;
  int32_t mask;
};

__device__ __forceinline__ Coords decompose(const GroupMap &g, uint32_t idx) {
  Coords c{0, 0, 0};
  if (g.n <= 0) return c;
  if (g.n == 1) {
    c.goff = (int64_t)idx * g.gstr[0];
    c.soff = (int32_t)idx * g.sstr[0];
    c.mask = (int32_t)idx;
    return c;
  }
  const uint32_t q0 = fast_div(idx, g.mg[0], g.sh[0]);
  const uint32_t c0 = idx - q0 * (uint32_t)g.ext[0];
  uint32_t c1 = q0, c2 = 0;
  if (g.n == 3) {
    c2 = fast_div(q0, g.mg[1], g.sh[1]);
    c1 = q0 - c2 * (uint32_t)g.ext[1];
  }
  c.goff = (int64_t)c0 * g.gstr[0] + (int64_t)c1 * g.gstr[1] + (int64_t)c2 * g.gstr[2];
  c.soff = (int32_t)(c0 * g.sstr[0] + c1 * g.sstr[1] + c2 * g.sstr[2]);
  c.mask = (int32_t)(g.mask == 0 ? c0 : (g.mask == 1 ? c1 : c2));
  return c;
}

// ---- element arithmetic (explicit rounding, never contracted into FMA) ----
template <typename T> struct Arith;
template <> struct Arith<float> {
  __device__ static float conj(float x) { return x; }
  __device__ static float mul(float l, double sr, double) { return __fmul_rn(l, (float)sr); }
  __device__ static float axpy(float d, float l, double sr, double) {
    return __fadd_rn(d, __fmul_rn(l, (float)sr));
  }
};
template <> struct Arith<double> {
  __device__ static double conj(double x) { return x; }
  __device__ static double mul(double l, double sr, double) { return __dmul_rn(l, sr); }
  __device__ static double axpy(double d, double l, double sr, double) {
    return __dadd_rn(d, __dmul_rn(l, sr));
  }
};
template <> struct Arith<float2> {
  __device__ static float2 conj(float2 x) { return make_float2(x.x, -x.y); }
  __device__ static float2 mul(float2 l, double sr, double si) {
    const float ar = (float)sr, ai = (float)si;
    return make_float2(__fsub_rn(__fmul_rn(l.x, ar), __fmul_rn(l.y, ai)),
                       __fadd_rn(__fmul_rn(l.x, ai), __fmul_rn(l.y, ar)));
  }
  __device__ static float2 axpy(float2 d, float2 l, double sr, double si) {
    const float ar = (float)sr, ai = (float)si;
    const float pr = __fsub_rn(__fmul_rn(l.x, ar), __fmul_rn(l.y, ai));
    const float pi = __fadd_rn(__fmul_rn(l.x, ai), __fmul_rn(l.y, ar));
    return make_float2(__fadd_rn(d.x, pr), __fadd_rn(d.y, pi));
  }
};
template <> struct Arith<double2> {
  __device__ static double2 conj(double2 x) { return make_double2(x.x, -x.y); }
  __device__ static double2 mul(double2 l, double sr, double si) {
    return make_double2(__dsub_rn(__dmul_rn(l.x, sr), __dmul_rn(l.y, si)),
                        __dadd_rn(__dmul_rn(l.x, si), __dmul_rn(l.y, sr)));
  }
  __device__ static double2 axpy(double2 d, double2 l, double sr, double si) {
    const double pr = __dsub_rn(__dmul_rn(l.x, sr), __dmul_rn(l.y, si));
    const double pi = __dadd_rn(__dmul_rn(l.x, si), __dmul_rn(l.y, sr));
    return make_double2(__dadd_rn(d.x, pr), __dadd_rn(d.y, pi));
  }
};

template <typename T, int N> struct alignas(sizeof(T) * N) Pack { T v[N]; };

template <typename T> struct CplxTraits { static constexpr bool value = false; };
template <> struct CplxTraits<float2> { static constexpr bool value = true; };
template <> struct CplxTraits<double2> { static constexpr bool value = true; };

// Operation applied in the write phase.
enum : int { kOpCopy = 0, kOpAdd = 1, kOpScaleCopy = 2 };

// Effective scale when a device-resident scalar multiplies alpha (scalar x
// tensor contractions): s = scalar * alpha as a complex(8) product, reduced to
// cmplx8_to_real8(s) for real kinds (reference tensor_block_contract ADD_TENSOR
// case, tensor_algebra_cpu.F90:4072-4084).
template <typename T>
__device__ __forceinline__ void effective_scale(const void *sdev, int sdev_kind, int sdev_conj,
                                                double &sr, double &si) {
  if (sdev == nullptr) return;
  double x = 0.0, y = 0.0;
  switch (sdev_kind) {
    case R4: x = *(const float *)sdev; break;
    case R8: x = *(const double *)sdev; break;
    case C4: x = ((const float2 *)sdev)->x; y = ((const float2 *)sdev)->y; break;
    default: x = ((const double2 *)sdev)->x; y = ((const double2 *)sdev)->y; break;
  }
  if (sdev_conj) y = -y;
  const double fr = __dsub_rn(__dmul_rn(x, sr), __dmul_rn(y, si));
  const double fi = __dadd_rn(__dmul_rn(x, si), __dmul_rn(y, sr));
  if (!CplxTraits<T>::value) {
    si = 0.0;
    sr = (fr != 0.0) ? (fr > 0.0 ? hypot(fr, fi) : -hypot(fr, fi)) : fi;
  } else {
    sr = fr;
    si = fi;
  }
}

template <typename T, int N>
__device__ __forceinline__ Pack<T, N> ld_pack(const T *p) {
  return *reinterpret_cast<const Pack<T, N> *>(p);
}
template <typename T, int N>
__device__ __forceinline__ void st_pack(T *p, const Pack<T, N> &v) {
  *reinterpret_cast<Pack<T, N> *>(p) = v;
}

// Asynchronous global -> shared copy of one element (LDGSTS); the element size
// is 4, 8 or 16 bytes and both addresses are element-aligned.
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void *smem_ptr, const void *gptr) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_ptr);
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gptr));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gptr), "n"(BYTES));
}
template <int BYTES>
__device__ __forceinline__ void cp_async_s(uint32_t s, const void *gptr) {
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gptr));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gptr), "n"(BYTES));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Per-dimension tiling data, copied to shared memory so that the lanes of a
// warp read different dimensions without serialising on the constant cache.
struct DimS {
  int64_t istr, ostr, ext;
  int32_t tl, nt;
  uint32_t mg_ts, sh_ts, mg_nt, sh_nt;
};

// Setup of tile t computed by one thread (coordinates by magic division of
// the tile index).  The lanes of a warp compute different tiles at once.
__device__ void setup_one(const PermParams &P, const DimS *D, int64_t t, TileSetup &S) {
  int64_t in_base = 0, out_base = 0;
  int ta = P.tl[P.a_last], tb = P.tl[P.b_last];
  for (int i = 0; i < P.rank; ++i) {
    const DimS d = D[i];
    if (d.nt <= 1) continue;
    const uint32_t qt = fast_div((uint32_t)t, d.mg_ts, d.sh_ts);
    const uint32_t c = qt - fast_div(qt, d.mg_nt, d.sh_nt) * (uint32_t)d.nt;
    const int64_t start = (int64_t)c * d.tl;
    in_base += start * d.istr;
    out_base += start * d.ostr;
    const int rem = (int)min((int64_t)d.tl, d.ext - start);
    if (i == P.a_last) ta = rem;
    if (i == P.b_last) tb = rem;
  }
  S.in_base = in_base;
  S.out_base = out_base;
  S.li_act = P.a_pre * ta;
  S.lo_act = P.b_pre * tb;
  S.ta_lim = P.a_in_B ? INT_MAX : ta;
  S.tb_lim = P.b_in_A ? INT_MAX : tb;
  S.full = (ta == P.tl[P.a_last] && tb == P.tl[P.b_last]) ? 1 : 0;
  S.type = (ta < P.tl[P.a_last] ? 1 : 0) | (tb < P.tl[P.b_last] ? 2 : 0);
}

// Setups of the CTA's iterations it0 .. it0 + 31 (tile blockIdx.x + it * gridDim.x),
// one per lane of warp 0, into a ring of kRing entries.
constexpr int kRing = 64;
__device__ __forceinline__ void fill_setups(const PermParams &P, const DimS *D, int it0, TileSetup *ring) {
  if (threadIdx.x < 32) {
    const int it = it0 + (int)threadIdx.x;
    const int64_t t = (int64_t)blockIdx.x + (int64_t)it * gridDim.x;
    if (t < P.num_tiles) setup_one(P, D, t, ring[it % kRing]);
  }
}

// Stores the valid ones of N output vectors (adds: all loads of D are issued
// before any store).
template <typename T, int VOUT, int OP, int N>
__device__ __forceinline__ void emit_masked(T *const *gp, Pack<T, VOUT> *v, const bool *ok, double sr,
                                            double si) {
  if constexpr (OP == kOpAdd) {
    Pack<T, VOUT> d[N];
#pragma unroll
    for (int u = 0; u < N; ++u)
      if (ok[u]) d[u] = ld_pack<T, VOUT>(gp[u]);
#pragma unroll
    for (int u = 0; u < N; ++u) {
      if (!ok[u]) continue;
#pragma unroll
      for (int j = 0; j < VOUT; ++j) d[u].v[j] = Arith<T>::axpy(d[u].v[j], v[u].v[j], sr, si);
      st_pack<T, VOUT>(gp[u], d[u]);
    }
  } else {
#pragma unroll
    for (int u = 0; u < N; ++u) {
      if (!ok[u]) continue;
      if constexpr (OP == kOpScaleCopy) {
#pragma unroll
        for (int j = 0; j < VOUT; ++j) v[u].v[j] = Arith<T>::mul(v[u].v[j], sr, si);
      }
      st_pack<T, VOUT>(gp[u], v[u]);
    }
  }
}

// Run tables of a plan (per-CTA, shared memory): input-run offsets and the
// coordinate of the output split dimension; output-run offsets, shared row
// offsets and the coordinate of the input split dimension; shared offset of
// every output-run position.
template <int NT>
__device__ void build_run_tables(const PermParams &P, int64_t *rIn, int32_t *rC, int64_t *wOut,
                                 int32_t *wSm, int32_t *wC, int32_t *ySm) {
  const int tid = threadIdx.x;
  for (int r = tid; r < P.Ri; r += NT) {
    int rem = r, cb = 0;
    int64_t off = 0;
    for (int k = 0; k < P.nra; ++k) {
      const int d = P.ra_dims[k];
      const int c = rem % P.tl[d];
      rem /= P.tl[d];
      off += (int64_t)c * P.istr[d];
      if (d == P.b_last) cb = c;
    }
    rIn[r] = off;
    rC[r] = P.b_in_A ? 0 : cb;
  }
  for (int r = tid; r < P.Ro; r += NT) {
    int rem = r, ca = 0, sm = 0;
    int64_t off = 0;
    for (int k = 0; k < P.nwb; ++k) {
      const int d = P.wb_dims[k];
      const int c = rem % P.tl[d];
      rem /= P.tl[d];
      off += (int64_t)c * P.ostr[d];
      sm += c * P.smstr[d];
      if (d == P.a_last) ca = c;
    }
    wOut[r] = off;
    wSm[r] = sm;
    wC[r] = P.a_in_B ? 0 : ca;
  }
  if (P.ytab) {
    for (int y = tid; y < P.Lo; y += NT) {
      int rem = y, sm = 0;
      for (int k = 0; k < P.nb; ++k) {
        const int d = P.b_dims[k];
        const int c = rem % P.tl[d];
        rem /= P.tl[d];
        sm += c * P.smstr[d];
      }
      ySm[y] = sm;
    }
  }
}

// Transpose / transpose-add with per-thread register tables.  Every tile of a
// plan has the same shape, so each thread's K read elements and K / VOUT write
// vectors have fixed offsets relative to the tile bases: they are computed once
// per CTA and held in registers (global offset, shared byte offset, and a
// 3-bit class: bit 0 the element lies beyond the last tile's extent along
// a_last, bit 1 likewise along b_last, bit 2 the slot is unused).  A tile
// moves each element with one asynchronous copy in and one shared load plus
// one (vector) store out; cut-short tiles mask by class.
template <typename T, int K, int VOUT, int OP, bool SWZ>
__global__ void __launch_bounds__(kThreads, K <= 4 ? 4 : TB_MIN_BLOCKS8)
    permute_reg_kernel(const T *__restrict__ src, T *dst, const PermParams P) {
  constexpr int KW = K / VOUT;  // write vectors per thread
  constexpr int S = reg_stages((int)sizeof(T), OP);
  constexpr bool DPF = OP == kOpAdd && kAddPrefetch;  // D vectors prefetched into shared slots
  using V = Pack<T, VOUT>;
  extern __shared__ __align__(16) unsigned char smem[];
  T *buf0 = reinterpret_cast<T *>(smem);
  __shared__ TileSetup setup[kRing];
  __shared__ DimS dimS[kMaxFR];
  const int tid = threadIdx.x;
  const int64_t G = gridDim.x;

  // Global offsets (elements, from the tile base), shared byte offsets (16-bit
  // pairs: the stage buffers are below 64 KB), classes (3 bits per slot).
  int32_t rg[K], wg[KW];
  uint32_t rs2[K / 2], ws2[K / 2];
  uint32_t rcls = 0, wcls = 0;
  auto half = [](const uint32_t *a, int i) -> uint32_t { return (i & 1) ? (a[i >> 1] >> 16) : (a[i >> 1] & 0xffffu); };
  {
    // Run tables live in shared memory only while the register tables are built.
    int64_t *rIn = reinterpret_cast<int64_t *>(smem + P.off_rin);
    int32_t *rC = reinterpret_cast<int32_t *>(smem + P.off_rc);
    int64_t *wOut = reinterpret_cast<int64_t *>(smem + P.off_wout);
    int32_t *wSm = reinterpret_cast<int32_t *>(smem + P.off_wsm);
    int32_t *wC = reinterpret_cast<int32_t *>(smem + P.off_wc);
    int32_t *ySm = reinterpret_cast<int32_t *>(smem + P.off_ysm);
    build_run_tables<kThreads>(P, rIn, rC, wOut, wSm, wC, ySm);
    if (tid < P.rank) {
      DimS d;
      d.istr = P.istr[tid];
      d.ostr = P.ostr[tid];
      d.ext = P.ext[tid];
      d.tl = P.tl[tid];
      d.nt = (int32_t)P.ntile[tid];
      d.mg_ts = P.mg_ts[tid];
      d.sh_ts = P.sh_ts[tid];
      d.mg_nt = P.mg_nt[tid];
      d.sh_nt = P.sh_nt[tid];
      dimS[tid] = d;
    }
    __syncthreads();
    auto sh = [](int p) -> uint32_t { return (uint32_t)(SWZ ? swz<T>(p) : p) * (uint32_t)sizeof(T); };
    auto cls_of = [&](int ca, int cb) -> uint32_t {
      return (ca >= P.ta_rem ? 1u : 0u) | (cb >= P.tb_rem ? 2u : 0u);
    };
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int e = tid + k * kThreads;
      rg[k] = 0;
      if ((k & 1) == 0) rs2[k >> 1] = 0;
      uint32_t c = 4u;
      if (e < P.V) {
        const int r = (int)fast_div((uint32_t)e, P.mg_li, P.sh_li);
        const int x = e - r * P.Li;
        rg[k] = (int32_t)(rIn[r] + x);
        rs2[k >> 1] |= sh(r * P.Li_pad + x) << (16 * (k & 1));
        const int ca = x / P.a_pre;
        const int cb = P.b_in_A ? (x / P.pre_bA) % P.tl[P.b_last] : rC[r];
        c = cls_of(ca, cb);
      }
      rcls |= c << (3 * k);
    }
    const int nv = P.nv, total = P.Ro * nv;
#pragma unroll
    for (int k = 0; k < KW; ++k) {
      const int f = tid + k * kThreads;
      wg[k] = 0;
#pragma unroll
      for (int j = 0; j < VOUT; ++j)
        if (((k * VOUT + j) & 1) == 0) ws2[(k * VOUT + j) >> 1] = 0;
      uint32_t c = 4u;
      if (f < total) {
        const int r = (int)fast_div((uint32_t)f, P.mg_nv, P.sh_nv);
        const int y = (f - r * nv) * VOUT;
        wg[k] = (int32_t)(wOut[r] + y);
#pragma unroll
        for (int j = 0; j < VOUT; ++j) {
          const int yj = y + j;
          const int p = wSm[r] + (P.ytab ? ySm[yj] : decompose(P.ymap, (uint32_t)yj).soff);
          ws2[(k * VOUT + j) >> 1] |= sh(p) << (16 * ((k * VOUT + j) & 1));
        }
        const int cb = y / P.b_pre;
        const int ca = P.a_in_B ? (y / P.pre_aB) % P.tl[P.a_last] : wC[r];
        c = cls_of(ca, cb);
      }
      wcls |= c << (3 * k);
    }
    __syncthreads();  // the run tables' space becomes tile buffers
  }
  fill_setups(P, dimS, 0, setup);
  fill_setups(P, dimS, 32, setup);
  __syncthreads();

  const bool cj = P.conj != 0;
  double sr = P.s_re, si = P.s_im;
  effective_scale<T>(P.sdev, P.sdev_kind, P.sdev_conj, sr, si);
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(buf0);
  const uint32_t stage_bytes = (uint32_t)P.buf_elems * (uint32_t)sizeof(T);
  // Prefetched D vectors: slot (stage, k) of thread tid, after the S tile buffers.
  constexpr uint32_t kSlotStage = (uint32_t)(KW * kThreads * sizeof(V));
  const uint32_t dbase = sbase + (uint32_t)S * stage_bytes + (uint32_t)tid * (uint32_t)sizeof(V);
  const unsigned char *dslots = smem + (size_t)S * stage_bytes + (size_t)tid * sizeof(V);

  auto issue_loads = [&](const TileSetup &St, int stage) {
    const T *g = src + St.in_base;
    const uint32_t sb = sbase + (uint32_t)stage * stage_bytes;
    const uint32_t m = (uint32_t)St.type | 4u;
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (((rcls >> (3 * k)) & m) == 0) cp_async_s<sizeof(T)>(sb + half(rs2, k), g + rg[k]);
    if constexpr (DPF) {
      const T *gd = dst + St.out_base;
      const uint32_t db = dbase + (uint32_t)stage * kSlotStage;
#pragma unroll
      for (int k = 0; k < KW; ++k)
        if (((wcls >> (3 * k)) & m) == 0)
          cp_async_s<sizeof(V)>(db + (uint32_t)(k * kThreads) * (uint32_t)sizeof(V), gd + wg[k]);
    }
  };

  int64_t t = blockIdx.x;
#pragma unroll
  for (int k = 0; k < S - 1; ++k) {
    if (t + k * G < P.num_tiles) issue_loads(setup[k], k);
    cp_async_commit();
  }
  for (int iter = 0; t < P.num_tiles; t += G, ++iter) {
    const int64_t tn = t + (S - 1) * G;
    if (tn < P.num_tiles)
      issue_loads(setup[(iter + S - 1) % kRing], (iter + S - 1) % S);
    cp_async_commit();
    if ((iter & 31) == 0 && iter > 0) fill_setups(P, dimS, iter + 32, setup);
    cp_async_wait<S - 1>();
    __syncthreads();
    const TileSetup St = setup[iter % kRing];
    const char *sbytes = reinterpret_cast<const char *>(smem) + (size_t)(iter % S) * stage_bytes;
    T *g = dst + St.out_base;
    const uint32_t m = (uint32_t)St.type | 4u;
    const unsigned char *ds = dslots + (size_t)(iter % S) * kSlotStage;
    // Batches of up to 4 vectors bound the live registers.
    constexpr int WB = KW < 4 ? KW : 4;
#pragma unroll
    for (int c0 = 0; c0 < KW; c0 += WB) {
      Pack<T, VOUT> v[WB];
      T *gp[WB];
      bool ok[WB];
#pragma unroll
      for (int u = 0; u < WB; ++u) {
        const int k = c0 + u;
        ok[u] = ((wcls >> (3 * k)) & m) == 0;
        gp[u] = g + wg[k];
        if (ok[u]) {
#pragma unroll
          for (int j = 0; j < VOUT; ++j) {
            const T x = *reinterpret_cast<const T *>(sbytes + half(ws2, k * VOUT + j));
            v[u].v[j] = cj ? Arith<T>::conj(x) : x;
          }
        }
      }
      if constexpr (DPF) {
#pragma unroll
        for (int u = 0; u < WB; ++u) {
          if (!ok[u]) continue;
          V d = *reinterpret_cast<const V *>(ds + (size_t)((c0 + u) * kThreads) * sizeof(V));
#pragma unroll
          for (int j = 0; j < VOUT; ++j) d.v[j] = Arith<T>::axpy(d.v[j], v[u].v[j], sr, si);
          st_pack<T, VOUT>(gp[u], d);
        }
      } else {
        emit_masked<T, VOUT, OP, WB>(gp, v, ok, sr, si);
      }
    }
    __syncthreads();
  }
}

// Bulk-read form of permute_reg_kernel.  Instead of one 4- or 8-byte
// asynchronous copy per element (which makes short runs fetch well beyond
// their bytes through the L1), every input run of a tile is moved by one bulk
// copy (cp.async.bulk, the TMA engine) of its 16-byte-aligned cover
// [floor16(start), ceil16(end)): the sectors read are the run's own.  Row r of
// a stage starts at r * pitch (a multiple of 16 bytes); the run's first element
// lands at byte (start mod 16) of its row.  That shift is the tile's
// (src + in_base * esize) mod 16 plus the run's (rIn * esize) mod 16, so each
// write slot keeps its row offset and the run's residue (4 bits) in registers
// and adds the tile's residue.  A stage is complete when its mbarrier has seen
// every thread arrive (with the byte count of the runs it copies) and every
// byte land; each wait is bounded, counting a CTA that gives up in
// g_permute_errors.  Writes, D prefetch and arithmetic are those of
// permute_reg_kernel, so results are bit-identical.
__device__ int g_permute_errors = 0;

__device__ __forceinline__ void mbar_init_s(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_s(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"((uint32_t)__cvta_generic_to_shared(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(uint32_t sdst, const void *gsrc, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(sdst),
      "l"(gsrc), "r"(bytes), "r"((uint32_t)__cvta_generic_to_shared(bar))
      : "memory");
}

constexpr int kBulkRunsPerThread = kMaxRuns / kThreads;  // runs a thread issues per tile (Ri <= kMaxRuns)
constexpr uint32_t kBulkSpin = 1u << 20;                 // bounded waits (about a second at most)

template <typename T, int K, int VOUT, int OP>
__global__ void __launch_bounds__(kThreads, K <= 4 ? 4 : 3)
    permute_bulk_kernel(const T *__restrict__ src, T *dst, const PermParams P) {
  constexpr int KW = K / VOUT;
  constexpr int S = reg_stages((int)sizeof(T), OP);
  constexpr bool DPF = OP == kOpAdd && kAddPrefetch;
  constexpr uint32_t ES = (uint32_t)sizeof(T);
  using V = Pack<T, VOUT>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ TileSetup setup[kRing];
  __shared__ DimS dimS[kMaxFR];
  __shared__ __align__(8) uint64_t full[S];
  const int tid = threadIdx.x;
  const int64_t G = gridDim.x;

  int32_t wg[KW];
  uint32_t ws2[K / 2];  // row offset + element offset (bytes, 16-bit pairs)
  uint32_t wnib = 0;    // per write element: (rIn * esize) mod 16 of its run (4 bits)
  uint32_t wcls = 0;
  int32_t my_rin[kBulkRunsPerThread], my_rc[kBulkRunsPerThread];
  auto half = [](const uint32_t *a, int i) -> uint32_t { return (i & 1) ? (a[i >> 1] >> 16) : (a[i >> 1] & 0xffffu); };
  {
    int64_t *rIn = reinterpret_cast<int64_t *>(smem + P.off_rin);
    int32_t *rC = reinterpret_cast<int32_t *>(smem + P.off_rc);
    int64_t *wOut = reinterpret_cast<int64_t *>(smem + P.off_wout);
    int32_t *wSm = reinterpret_cast<int32_t *>(smem + P.off_wsm);
    int32_t *wC = reinterpret_cast<int32_t *>(smem + P.off_wc);
    int32_t *ySm = reinterpret_cast<int32_t *>(smem + P.off_ysm);
    build_run_tables<kThreads>(P, rIn, rC, wOut, wSm, wC, ySm);
    if (tid < P.rank) {
      DimS d;
      d.istr = P.istr[tid];
      d.ostr = P.ostr[tid];
      d.ext = P.ext[tid];
      d.tl = P.tl[tid];
      d.nt = (int32_t)P.ntile[tid];
      d.mg_ts = P.mg_ts[tid];
      d.sh_ts = P.sh_ts[tid];
      d.mg_nt = P.mg_nt[tid];
      d.sh_nt = P.sh_nt[tid];
      dimS[tid] = d;
    }
    if (tid < S) mbar_init_s(&full[tid], kThreads);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kBulkRunsPerThread; ++j) {
      const int r = tid + j * kThreads;
      my_rin[j] = r < P.Ri ? (int32_t)rIn[r] : 0;
      my_rc[j] = r < P.Ri ? rC[r] : 0;
    }
    auto cls_of = [&](int ca, int cb) -> uint32_t {
      return (ca >= P.ta_rem ? 1u : 0u) | (cb >= P.tb_rem ? 2u : 0u);
    };
    const int nv = P.nv, total = P.Ro * nv;
#pragma unroll
    for (int k = 0; k < KW; ++k) {
      const int f = tid + k * kThreads;
      wg[k] = 0;
#pragma unroll
      for (int j = 0; j < VOUT; ++j)
        if (((k * VOUT + j) & 1) == 0) ws2[(k * VOUT + j) >> 1] = 0;
      uint32_t c = 4u;
      if (f < total) {
        const int r = (int)fast_div((uint32_t)f, P.mg_nv, P.sh_nv);
        const int y = (f - r * nv) * VOUT;
        wg[k] = (int32_t)(wOut[r] + y);
#pragma unroll
        for (int j = 0; j < VOUT; ++j) {
          const int yj = y + j;
          const int p = wSm[r] + (P.ytab ? ySm[yj] : decompose(P.ymap, (uint32_t)yj).soff);  // r_in * Li_pad + x
          const int rr = (int)fast_div((uint32_t)p, P.mg_lip, P.sh_lip), x = p - rr * P.Li_pad;
          const uint32_t off = (uint32_t)rr * (uint32_t)P.pitch_b + (uint32_t)x * ES;
          ws2[(k * VOUT + j) >> 1] |= off << (16 * ((k * VOUT + j) & 1));
          wnib |= (uint32_t)((rIn[rr] * (int64_t)ES) & 15) << (4 * (k * VOUT + j));
        }
        const int cb = y / P.b_pre;
        const int ca = P.a_in_B ? (y / P.pre_aB) % P.tl[P.a_last] : wC[r];
        c = cls_of(ca, cb);
      }
      wcls |= c << (3 * k);
    }
    __syncthreads();  // the run tables' space becomes tile buffers
    // The stage buffers were just written through the generic proxy; the bulk
    // copies write them through the async proxy.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  fill_setups(P, dimS, 0, setup);
  fill_setups(P, dimS, 32, setup);
  __syncthreads();

  const bool cj = P.conj != 0;
  double sr = P.s_re, si = P.s_im;
  effective_scale<T>(P.sdev, P.sdev_kind, P.sdev_conj, sr, si);
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  const uint32_t stage_bytes = (uint32_t)P.buf_elems * ES;
  constexpr uint32_t kSlotStage = (uint32_t)(KW * kThreads * sizeof(V));
  const uint32_t dbase = sbase + (uint32_t)S * stage_bytes + (uint32_t)tid * (uint32_t)sizeof(V);
  const unsigned char *dslots = smem + (size_t)S * stage_bytes + (size_t)tid * sizeof(V);
  const uintptr_t src_addr = reinterpret_cast<uintptr_t>(src);
  bool failed = false;

  auto issue_loads = [&](const TileSetup &St, int stage) {
    const uintptr_t gbase = src_addr + (uintptr_t)St.in_base * ES;
    const uint32_t sb = sbase + (uint32_t)stage * stage_bytes;
    const uint32_t len = (uint32_t)St.li_act * ES;
    uint32_t bytes = 0;
#pragma unroll
    for (int j = 0; j < kBulkRunsPerThread; ++j) {
      const int r = tid + j * kThreads;
      if (r < P.Ri && (P.b_in_A || my_rc[j] < St.tb_lim)) {
        const uintptr_t a0 = gbase + (uintptr_t)(int64_t)my_rin[j] * ES;
        bytes += (uint32_t)(((a0 + len + 15) & ~(uintptr_t)15) - (a0 & ~(uintptr_t)15));
      }
    }
    mbar_arrive_tx(&full[stage], bytes);
#pragma unroll
    for (int j = 0; j < kBulkRunsPerThread; ++j) {
      const int r = tid + j * kThreads;
      if (r < P.Ri && (P.b_in_A || my_rc[j] < St.tb_lim)) {
        const uintptr_t a0 = gbase + (uintptr_t)(int64_t)my_rin[j] * ES;
        const uintptr_t lo = a0 & ~(uintptr_t)15;
        const uint32_t n = (uint32_t)(((a0 + len + 15) & ~(uintptr_t)15) - lo);
        bulk_g2s(sb + (uint32_t)r * (uint32_t)P.pitch_b, reinterpret_cast<const void *>(lo), n, &full[stage]);
      }
    }
    if constexpr (DPF) {
      const T *gd = dst + St.out_base;
      const uint32_t db = dbase + (uint32_t)stage * kSlotStage;
      const uint32_t m = (uint32_t)St.type | 4u;
#pragma unroll
      for (int k = 0; k < KW; ++k)
        if (((wcls >> (3 * k)) & m) == 0)
          cp_async_s<sizeof(V)>(db + (uint32_t)(k * kThreads) * (uint32_t)sizeof(V), gd + wg[k]);
    }
  };

  int64_t t = blockIdx.x;
#pragma unroll
  for (int k = 0; k < S - 1; ++k) {
    if (t + k * G < P.num_tiles) issue_loads(setup[k], k);
    cp_async_commit();
  }
  for (int iter = 0; t < P.num_tiles; t += G, ++iter) {
    const int64_t tn = t + (S - 1) * G;
    if (tn < P.num_tiles) issue_loads(setup[(iter + S - 1) % kRing], (iter + S - 1) % S);
    cp_async_commit();
    if ((iter & 31) == 0 && iter > 0) fill_setups(P, dimS, iter + 32, setup);
    cp_async_wait<S - 1>();
    if (!failed) {  // after one wait has run out the CTA stops waiting and only finishes its loop
      const uint32_t parity = (uint32_t)((iter / S) & 1);
      uint32_t n = 0;
      while (!mbar_try_s(&full[iter % S], parity))
        if (++n == kBulkSpin) { failed = true; break; }
    }
    __syncthreads();
    const TileSetup St = setup[iter % kRing];
    const char *sbytes = reinterpret_cast<const char *>(smem) + (size_t)(iter % S) * stage_bytes;
    const uint32_t tnib = (uint32_t)((src_addr + (uintptr_t)St.in_base * ES) & 15);
    T *g = dst + St.out_base;
    const uint32_t m = (uint32_t)St.type | 4u;
    const unsigned char *ds = dslots + (size_t)(iter % S) * kSlotStage;
    constexpr int WB = KW < 4 ? KW : 4;
#pragma unroll
    for (int c0 = 0; c0 < KW; c0 += WB) {
      Pack<T, VOUT> v[WB];
      T *gp[WB];
      bool ok[WB];
#pragma unroll
      for (int u = 0; u < WB; ++u) {
        const int k = c0 + u;
        ok[u] = ((wcls >> (3 * k)) & m) == 0;
        gp[u] = g + wg[k];
        if (ok[u]) {
#pragma unroll
          for (int j = 0; j < VOUT; ++j) {
            const int e = k * VOUT + j;
            const uint32_t shift = (tnib + ((wnib >> (4 * e)) & 15u)) & 15u;
            const T x = *reinterpret_cast<const T *>(sbytes + half(ws2, e) + shift);
            v[u].v[j] = cj ? Arith<T>::conj(x) : x;
          }
        }
      }
      if constexpr (DPF) {
#pragma unroll
        for (int u = 0; u < WB; ++u) {
          if (!ok[u]) continue;
          V d = *reinterpret_cast<const V *>(ds + (size_t)((c0 + u) * kThreads) * sizeof(V));
#pragma unroll
          for (int j = 0; j < VOUT; ++j) d.v[j] = Arith<T>::axpy(d.v[j], v[u].v[j], sr, si);
          st_pack<T, VOUT>(gp[u], d);
        }
      } else {
        emit_masked<T, VOUT, OP, WB>(gp, v, ok, sr, si);
      }
    }
    __syncthreads();
  }
  if (failed) atomicAdd(&g_permute_errors, 1);
}

// Transpose / transpose-add for plans whose tiles span more than 32-bit
// offsets (tensors of more than 2^31 elements): positions come from the
// shared run tables (64-bit offsets) for every element.
template <typename T, int VOUT, int OP, bool SWZ>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    permute_tiled_kernel(const T *__restrict__ src, T *dst, const PermParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  T *buf0 = reinterpret_cast<T *>(smem);
  int64_t *rIn = reinterpret_cast<int64_t *>(smem + P.off_rin);
  int32_t *rC = reinterpret_cast<int32_t *>(smem + P.off_rc);
  int64_t *wOut = reinterpret_cast<int64_t *>(smem + P.off_wout);
  int32_t *wSm = reinterpret_cast<int32_t *>(smem + P.off_wsm);
  int32_t *wC = reinterpret_cast<int32_t *>(smem + P.off_wc);
  int32_t *ySm = reinterpret_cast<int32_t *>(smem + P.off_ysm);
  __shared__ TileSetup setup[kRing];
  __shared__ DimS dimS[kMaxFR];
  const int tid = threadIdx.x;
  const int64_t G = gridDim.x;
  build_run_tables<kThreads>(P, rIn, rC, wOut, wSm, wC, ySm);
  if (tid < P.rank) {
    DimS d;
    d.istr = P.istr[tid];
    d.ostr = P.ostr[tid];
    d.ext = P.ext[tid];
    d.tl = P.tl[tid];
    d.nt = (int32_t)P.ntile[tid];
    d.mg_ts = P.mg_ts[tid];
    d.sh_ts = P.sh_ts[tid];
    d.mg_nt = P.mg_nt[tid];
    d.sh_nt = P.sh_nt[tid];
    dimS[tid] = d;
  }
  __syncthreads();
  fill_setups(P, dimS, 0, setup);
  fill_setups(P, dimS, 32, setup);
  __syncthreads();

  const bool cj = P.conj != 0;
  double sr = P.s_re, si = P.s_im;
  effective_scale<T>(P.sdev, P.sdev_kind, P.sdev_conj, sr, si);
  auto sh = [](int p) -> int { return SWZ ? swz<T>(p) : p; };
  const int pitch = P.Li_pad;
  const int nv = P.nv, total = P.Ro * nv;
  const int ystr = P.ymap.sstr[0];
  auto ypos = [&](int ws, int y) -> int {
    return ws + (P.ytab ? ySm[y] : decompose(P.ymap, (uint32_t)y).soff);
  };
  auto tile_buf = [&](int k) -> T * { return buf0 + (size_t)(k % kStages) * P.buf_elems; };
  auto issue_loads = [&](const TileSetup &S, T *buf) {
    const T *g = src + S.in_base;
#pragma unroll 2
    for (int e = tid; e < P.V; e += kThreads) {
      const int r = (int)fast_div((uint32_t)e, P.mg_li, P.sh_li);
      const int x = e - r * P.Li;
      if (!S.full && (x >= S.li_act || rC[r] >= S.tb_lim)) continue;
      cp_async_elem<sizeof(T)>(buf + sh(r * pitch + x), g + (rIn[r] + x));
    }
  };

  int64_t t = blockIdx.x;
#pragma unroll
  for (int k = 0; k < kStages - 1; ++k) {
    if (t + k * G < P.num_tiles) issue_loads(setup[k], tile_buf(k));
    cp_async_commit();
  }
  for (int iter = 0; t < P.num_tiles; t += G, ++iter) {
    const int64_t tn = t + (kStages - 1) * G;
    if (tn < P.num_tiles) issue_loads(setup[(iter + kStages - 1) % kRing], tile_buf(iter + kStages - 1));
    cp_async_commit();
    if ((iter & 31) == 0 && iter > 0) fill_setups(P, dimS, iter + 32, setup);
    cp_async_wait<kStages - 1>();
    __syncthreads();
    const TileSetup S = setup[iter % kRing];
    const T *buf = tile_buf(iter);
    T *g = dst + S.out_base;
    constexpr int U = 4;  // vectors per batch: U shared gathers (and loads of D) in flight
    for (int f0 = tid; f0 < total; f0 += U * kThreads) {
      Pack<T, VOUT> v[U];
      T *gp[U];
      bool ok[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int f = f0 + u * kThreads;
        const int r = (int)fast_div((uint32_t)f, P.mg_nv, P.sh_nv);
        const int y = (f - r * nv) * VOUT;
        ok[u] = f < total && (S.full || (y < S.lo_act && wC[r] < S.ta_lim));
        gp[u] = g;
        if (!ok[u]) continue;
        const int ws = wSm[r];
        if (P.y_step) {
          const int base = ypos(ws, y);
#pragma unroll
          for (int j = 0; j < VOUT; ++j) v[u].v[j] = buf[sh(base + j * ystr)];
        } else {
#pragma unroll
          for (int j = 0; j < VOUT; ++j) v[u].v[j] = buf[sh(ypos(ws, y + j))];
        }
        if (cj) {
#pragma unroll
          for (int j = 0; j < VOUT; ++j) v[u].v[j] = Arith<T>::conj(v[u].v[j]);
        }
        gp[u] = g + (wOut[r] + y);
      }
      emit_masked<T, VOUT, OP, U>(gp, v, ok, sr, si);
    }
    __syncthreads();
  }
}

// Identity permutation after fusion: straight streaming copy / add.
template <typename T, int VEC, int OP>
__global__ void __launch_bounds__(kThreads) linear_kernel(const T *__restrict__ src, T *dst,
                                                          int64_t nvec, int64_t tail_start,
                                                          int64_t vol, int conj, double sr,
                                                          double si, const void *sdev,
                                                          int sdev_kind, int sdev_conj) {
  const bool cj = conj != 0;
  effective_scale<T>(sdev, sdev_kind, sdev_conj, sr, si);
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < nvec; i += stride) {
    Pack<T, VEC> v = ld_pack<T, VEC>(src + i * VEC);
    if (cj) {
#pragma unroll
      for (int j = 0; j < VEC; ++j) v.v[j] = Arith<T>::conj(v.v[j]);
    }
    if constexpr (OP == kOpAdd) {
      Pack<T, VEC> d = ld_pack<T, VEC>(dst + i * VEC);
#pragma unroll
      for (int j = 0; j < VEC; ++j) d.v[j] = Arith<T>::axpy(d.v[j], v.v[j], sr, si);
      st_pack<T, VEC>(dst + i * VEC, d);
    } else if constexpr (OP == kOpScaleCopy) {
#pragma unroll
      for (int j = 0; j < VEC; ++j) v.v[j] = Arith<T>::mul(v.v[j], sr, si);
      st_pack<T, VEC>(dst + i * VEC, v);
    } else {
      st_pack<T, VEC>(dst + i * VEC, v);
    }
  }
  for (int64_t i = tail_start + (int64_t)blockIdx.x * kThreads + threadIdx.x; i < vol; i += stride) {
    T v = src[i];
    if (cj) v = Arith<T>::conj(v);
    if constexpr (OP == kOpAdd) dst[i] = Arith<T>::axpy(dst[i], v, sr, si);
    else if constexpr (OP == kOpScaleCopy) dst[i] = Arith<T>::mul(v, sr, si);
    else dst[i] = v;
  }
}

// ------------------------------------------------------------------------
// Host planning
// ------------------------------------------------------------------------

struct Fused {
  int n = 0;
  int64_t ext[kMaxFR];
  int perm[kMaxFR];  // O2N, 0-based
  int64_t vol = 1;
};

// Drops unit extents and fuses input dimensions that stay adjacent and in order
// in the output: consecutive kept input dimensions i-1, i form one group when
// their output positions are consecutive too.
int fuse_dims(int rank, const int *dims, const int *o2n, Fused &F) {
  int keep_pos[kMaxRank];
  int64_t keep_ext[kMaxRank];
  int nk = 0;
  F.vol = 1;
  for (int i = 0; i < rank; ++i) {
    F.vol *= dims[i];
    if (dims[i] > 1) { keep_ext[nk] = dims[i]; keep_pos[nk] = o2n[i] - 1; ++nk; }
  }
  int order[kMaxRank], newpos[kMaxRank];
  for (int i = 0; i < nk; ++i) order[i] = i;
  std::sort(order, order + nk, [&](int a, int b) { return keep_pos[a] < keep_pos[b]; });
  for (int k = 0; k < nk; ++k) newpos[order[k]] = k;
  int n = 0;
  int64_t gext[kMaxRank];
  int gfirst[kMaxRank];
  for (int i = 0; i < nk; ++i) {
    if (i > 0 && newpos[i] == newpos[i - 1] + 1) {
      gext[n - 1] *= keep_ext[i];
    } else {
      gext[n] = keep_ext[i];
      gfirst[n] = newpos[i];
      ++n;
    }
  }
  if (n > kMaxFR) return TALSH_LIMIT_EXCEEDED;
  int ord[kMaxRank];
  for (int g = 0; g < n; ++g) ord[g] = g;
  std::sort(ord, ord + n, [&](int a, int b) { return gfirst[a] < gfirst[b]; });
  F.n = n;
  for (int g = 0; g < n; ++g) F.ext[g] = gext[g];
  for (int k = 0; k < n; ++k) F.perm[ord[k]] = k;
  return TALSH_SUCCESS;
}

// Elements per thread of permute_reg_kernel (its tile is at most 256 x this):
// 8, or 4 for 16-byte elements; TALSH_B200_REG_K=4 selects 4 for every kind.
int reg_k(int esize) {
  static int forced = -1;
  if (forced < 0) {
    const char *e = std::getenv("TALSH_B200_REG_K");
    forced = (e && std::atoi(e) == 4) ? 4 : 0;
  }
  if (esize >= 16) return 4;
  return forced ? forced : 8;
}

// Where the bulk-read form of the register-table kernel runs: by default for
// elements of 8 bytes or more, copies and scalar-output adds (measured on the
// transpose/add sweep: 4-byte elements lose to bank conflicts in the 16-byte
// aligned rows, vector-output adds lose a little); TALSH_B200_PERMUTE_BULK=1
// selects it for every plan it can take, 0 for none.
int permute_bulk_mode() {
  static const int v = [] {
    const char *e = std::getenv("TALSH_B200_PERMUTE_BULK");
    return e ? (std::atoi(e) != 0 ? 1 : 0) : 2;
  }();
  return v;
}
bool permute_bulk_wanted(int esize, int op, int vout) {
  const int mode = permute_bulk_mode();
  if (mode != 2) return mode == 1;
  return esize >= 8 && (op != kOpAdd || vout == 1);
}

// Tile buffer budget in bytes: kTileBytes, or TALSH_B200_TILE_BYTES (4096..49152) for tuning.
int tile_bytes() {
  static int v = 0;
  if (v == 0) {
    v = kTileBytes;
    if (const char *e = std::getenv("TALSH_B200_TILE_BYTES")) {
      const int t = std::atoi(e);
      if (t >= 4096 && t <= 49152) v = t;
    }
  }
  return v;
}

struct Plan {
  bool linear = false;
  int64_t vol = 0;
  PermParams P;
  int vin = 1, vout = 1;
  size_t smem = 0;
};

// Next tile extent for a split dimension: about twice the current one, but
// chosen so that the dimension divides into equal tiles (little masked work).
int64_t balanced_grow(int64_t ext, int64_t cur) {
  // An exact divisor up to 3x leaves no cut-short tile along this dimension.
  for (int64_t t = cur + 1; t <= std::min(ext, cur * 3); ++t)
    if (ext % t == 0) return t;
  for (int64_t target = cur * 2; target < ext; target += cur) {
    const int64_t pieces = (ext + target - 1) / target;
    const int64_t t = (ext + pieces - 1) / pieces;
    if (t > cur) return t;
  }
  return ext;
}

// Plan choices the transpose autotuner (tcTensorPermuteTune) can override;
// the defaults are the heuristics of build_plan.
struct PlanCfg {
  int bulk = -1;   // -1: permute_bulk_wanted decides; 0: never; 1: wherever the plan allows it
  int small = 0;   // 1: tiles of at most 4 elements per thread (more resident CTAs per SM)
  int flip = 0;    // 1: walk the tiles in the other tensor's dimension order
  int grow = -1;   // tile growth: -1 the shorter run first, 0 input runs first, 1 output runs first
  int longrun = 0; // initial runs of at least 2^longrun times the usual elements
  int keep = 0;    // 1: small tensors keep the full tile budget
};

// out_major: tile index order follows the output's dimensions (copies), else
// the input's (adds, whose output sectors are read before they are written).
int build_plan(int esize, const Fused &F, Plan &plan, int op = kOpCopy, const PlanCfg &cfg = PlanCfg()) {
  const bool out_major = (op != kOpAdd && !TB_COPY_INPUT_MAJOR) != (cfg.flip != 0);
  plan.vol = F.vol;
  if (F.n <= 1) { plan.linear = true; return TALSH_SUCCESS; }
  PermParams &P = plan.P;
  std::memset(&P, 0, sizeof(P));
  const int n = F.n;
  P.rank = n;
  int q[kMaxFR];  // N2O
  for (int i = 0; i < n; ++i) { P.ext[i] = F.ext[i]; q[F.perm[i]] = i; }
  int64_t s = 1;
  for (int i = 0; i < n; ++i) { P.istr[i] = s; s *= P.ext[i]; }
  s = 1;
  for (int k = 0; k < n; ++k) { P.ostr[q[k]] = s; s *= P.ext[q[k]]; }

  // Tile budget: at most reg_k(esize) elements per thread of the register-table
  // kernel.  Small tensors get smaller tiles so that every SM still holds a few.
  int elems_max = std::min(tile_bytes() / esize, kThreads * (cfg.small ? 4 : reg_k(esize)));
  {
    const int64_t slots = 148LL * kMinBlocks * 2;
    while (!cfg.keep && elems_max / 2 >= 1024 && F.vol / elems_max < slots) elems_max /= 2;  // floor 1024: every plan fits
  }
  const int run_min = (esize >= 16 ? 16 : 32) << cfg.longrun;
  // Initial groups: shortest prefixes reaching run_min elements.
  int na = 0, nb = 0;
  int64_t tA = 1, tB = 1;
  {
    int64_t pre = 1;
    for (int i = 0; i < n; ++i) {
      if (pre * P.ext[i] >= run_min || i == n - 1) {
        na = i + 1;
        tA = std::min<int64_t>(P.ext[i], (run_min + pre - 1) / pre);
        tA = (P.ext[i] + (P.ext[i] + tA - 1) / tA - 1) / ((P.ext[i] + tA - 1) / tA);  // equal pieces
        break;
      }
      pre *= P.ext[i];
    }
    pre = 1;
    for (int k = 0; k < n; ++k) {
      if (pre * P.ext[q[k]] >= run_min || k == n - 1) {
        nb = k + 1;
        const int64_t e = P.ext[q[k]];
        tB = std::min<int64_t>(e, (run_min + pre - 1) / pre);
        tB = (e + (e + tB - 1) / tB - 1) / ((e + tB - 1) / tB);  // equal pieces
        break;
      }
      pre *= P.ext[q[k]];
    }
  }
  struct Geo { int64_t tl[kMaxFR]; int64_t V, Li, Lo; };
  auto geometry = [&](int na_, int64_t tA_, int nb_, int64_t tB_, Geo &G) {
    for (int i = 0; i < n; ++i) G.tl[i] = 1;
    for (int i = 0; i < na_ - 1; ++i) G.tl[i] = P.ext[i];
    for (int k = 0; k < nb_ - 1; ++k) G.tl[q[k]] = P.ext[q[k]];
    const int al = na_ - 1, bl = q[nb_ - 1];
    G.tl[al] = std::max(G.tl[al], tA_);
    G.tl[bl] = std::max(G.tl[bl], tB_);
    G.V = 1;
    for (int i = 0; i < n; ++i) G.V *= G.tl[i];
    G.Li = 1;
    for (int i = 0; i < na_; ++i) G.Li *= G.tl[i];
    G.Lo = 1;
    for (int k = 0; k < nb_; ++k) G.Lo *= G.tl[q[k]];
  };
  // Groups of more than three tile dimensions fall back to shared tables,
  // which bound their length; everything else only has the tile budget.
  auto group_dims = [&](const Geo &G, int na_, int nb_, int &nra, int &nwb) {
    bool inA[kMaxFR] = {false}, inB[kMaxFR] = {false};
    for (int i = 0; i < na_; ++i) inA[i] = true;
    for (int k = 0; k < nb_; ++k) inB[q[k]] = true;
    nra = nwb = 0;
    for (int i = 0; i < n; ++i) {
      if (G.tl[i] <= 1) continue;
      if (!inA[i]) ++nra;
      if (!inB[i]) ++nwb;
    }
  };
  int cur_na = na, cur_nb = nb;
  auto acceptable = [&](const Geo &G) {
    if (G.V > elems_max) return false;
    int nra, nwb;
    group_dims(G, cur_na, cur_nb, nra, nwb);
    (void)nra; (void)nwb;
    if (cur_nb > 3 && G.Lo > kMaxTabLo) return false;  // B positions need the table
    if (G.V / G.Li > kMaxRuns || G.V / G.Lo > kMaxRuns) return false;
    return true;
  };
  Geo G;
  geometry(na, tA, nb, tB, G);
  if (!acceptable(G)) {
    // Groups alone overflow the tile budget: shrink the split extents.
    while (!acceptable(G) && (tA > 1 || tB > 1)) {
      if (tA >= tB && tA > 1) tA = (tA + 1) / 2; else if (tB > 1) tB = (tB + 1) / 2;
      geometry(na, tA, nb, tB, G);
    }
    if (!acceptable(G)) return TALSH_NOT_IMPLEMENTED;
  }
  // Grow the tile toward the budget, favouring the shorter run.
  for (int iter = 0; iter < 256; ++iter) {
    if (G.V * 2 > elems_max) break;
    bool done = false;
    for (int pass = 0; pass < 2 && !done; ++pass) {
      const bool firstA = cfg.grow < 0 ? (G.Li <= G.Lo) : (cfg.grow == 0);
      const bool growA = (pass == 0) ? firstA : !firstA;
      int na2 = na, nb2 = nb;
      int64_t tA2 = tA, tB2 = tB;
      if (growA) {
        const int al = na - 1;
        if (G.tl[al] < P.ext[al]) {
          tA2 = balanced_grow(P.ext[al], G.tl[al]);
        } else if (na < n) {
          na2 = na + 1;
          tA2 = std::min<int64_t>(P.ext[na2 - 1], std::max<int64_t>(2, G.tl[na2 - 1]));
        } else {
          continue;
        }
      } else {
        const int bl = q[nb - 1];
        if (G.tl[bl] < P.ext[bl]) {
          tB2 = balanced_grow(P.ext[bl], G.tl[bl]);
        } else if (nb < n) {
          nb2 = nb + 1;
          tB2 = std::min<int64_t>(P.ext[q[nb2 - 1]], std::max<int64_t>(2, G.tl[q[nb2 - 1]]));
        } else {
          continue;
        }
      }
      Geo G2;
      geometry(na2, tA2, nb2, tB2, G2);
      cur_na = na2; cur_nb = nb2;
      const bool ok = acceptable(G2);
      cur_na = na; cur_nb = nb;
      if (ok) {
        na = na2; nb = nb2; tA = tA2; tB = tB2; G = G2;
        cur_na = na; cur_nb = nb;
        done = true;
      }
    }
    if (!done) break;
  }
  // Fill parameters.
  for (int i = 0; i < n; ++i) {
    P.tl[i] = (int32_t)G.tl[i];
    P.ntile[i] = (P.ext[i] + G.tl[i] - 1) / G.tl[i];
  }
  // Tile index order.  Output-major for copies: the tiles in flight at any time
  // write neighbouring stretches of the output, so the sectors that straddle
  // two tiles are completed in L2 before they are written back (a misaligned
  // output run otherwise costs a read-modify-write).  Input-major for adds,
  // which read the output sectors anyway.
  P.num_tiles = 1;
  for (int k = 0; k < n; ++k) {
    const int i = out_major ? q[k] : k;
    make_magic((uint32_t)P.num_tiles, P.mg_ts[i], P.sh_ts[i]);  // tile-index stride of dimension i
    make_magic((uint32_t)P.ntile[i], P.mg_nt[i], P.sh_nt[i]);
    P.num_tiles *= P.ntile[i];
  }
  if (P.num_tiles >= INT_MAX) return TALSH_LIMIT_EXCEEDED;  // tile indices use 32-bit magic division
  P.V = (int)G.V;
  P.Li = (int)G.Li;
  P.Lo = (int)G.Lo;
  P.Ri = (int)(G.V / G.Li);
  P.Ro = (int)(G.V / G.Lo);
  P.a_last = na - 1;
  P.b_last = q[nb - 1];
  P.a_pre = (int)(G.Li / G.tl[P.a_last]);
  P.b_pre = (int)(G.Lo / G.tl[P.b_last]);
  bool inA[kMaxFR] = {false}, inB[kMaxFR] = {false};
  for (int i = 0; i < na; ++i) inA[i] = true;
  for (int k = 0; k < nb; ++k) inB[q[k]] = true;
  P.a_in_B = inB[P.a_last] ? 1 : 0;
  P.b_in_A = inA[P.b_last] ? 1 : 0;
  // Shared layout: x over A (input order) contiguous, input runs over U\A with
  // row pitch Li_pad.  The write phase walks the output's fastest dimension
  // q[0] with shared stride smstr[q[0]].  When q[0] lies inside A (and is not
  // its first dimension) that stride is a product of A extents, often a power
  // of two: the indices are then bank-swizzled.  Otherwise the stride is a
  // multiple of the row pitch, which is made odd.
  P.swz = (inA[q[0]] && q[0] != 0) ? 1 : 0;
  P.Li_pad = P.swz ? P.Li : (P.Li % 2 == 0 ? P.Li + 1 : P.Li);
  {
    int32_t st = 1;
    for (int i = 0; i < na; ++i) { P.smstr[i] = st; st *= P.tl[i]; }
    st = P.Li_pad;
    P.nra = 0;
    for (int i = 0; i < n; ++i) {
      if (inA[i] || P.tl[i] == 1) continue;
      P.smstr[i] = st;
      st *= P.tl[i];
      P.ra_dims[P.nra++] = (int8_t)i;
    }
    P.nwb = 0;
    for (int i = 0; i < n; ++i)
      if (!inB[i] && P.tl[i] > 1) P.wb_dims[P.nwb++] = (int8_t)i;
    P.nb = nb;
    for (int k = 0; k < nb; ++k) P.b_dims[k] = (int8_t)q[k];
  }
  make_magic((uint32_t)P.Li, P.mg_li, P.sh_li);
  make_magic((uint32_t)P.Lo, P.mg_lo, P.sh_lo);
  // Group maps: read runs over U\A (input strides), write runs over U\B
  // (output strides), output-run positions over B (shared strides only).
  auto fill_map = [&](GroupMap &g, const int8_t *dims, int nd, bool output_side, int mask_dim) {
    std::memset(&g, 0, sizeof(g));
    g.mask = -1;
    if (nd > 3) { g.n = -1; return; }
    g.n = nd;
    for (int k = 0; k < nd; ++k) {
      const int d = dims[k];
      g.ext[k] = P.tl[d];
      g.gstr[k] = output_side ? P.ostr[d] : P.istr[d];
      g.sstr[k] = P.smstr[d];
      if (d == mask_dim) g.mask = k;
    }
    for (int k = 0; k < 2 && k < nd; ++k) make_magic((uint32_t)g.ext[k], g.mg[k], g.sh[k]);
  };
  fill_map(P.rmap, P.ra_dims, P.nra, false, P.b_in_A ? -1 : P.b_last);
  fill_map(P.wmap, P.wb_dims, P.nwb, true, P.a_in_B ? -1 : P.a_last);
  fill_map(P.ymap, P.b_dims, P.nb, false, -1);
  // Output vector width: every output run start, run length and partial run
  // length must be a multiple of the vector (16 bytes, or 8 bytes for 4-byte
  // elements when 16 do not divide them).  Reads are element-granular
  // asynchronous copies and need no alignment beyond the element.
  const int vec = 16 / esize;
  plan.vin = 1;
  plan.vout = 1;
  for (int v = vec; v > 1 && plan.vout == 1 && (v == vec || esize == 4); v /= 2) {
    bool ok = (P.Lo % v) == 0;
    const int64_t partial = P.ext[P.b_last] % P.tl[P.b_last];
    if (partial && ((int64_t)P.b_pre * partial) % v) ok = false;
    for (int i = 0; i < n && ok; ++i) {
      if (!inB[i] && P.tl[i] > 1 && P.ostr[i] % v) ok = false;       // run offsets
      if (P.ntile[i] > 1 && (P.tl[i] * P.ostr[i]) % v) ok = false;   // tile bases
    }
    if (ok) plan.vout = v;
  }
  // Shared memory: the stage buffers and the run tables.  Each buffer is
  // rounded up to whole 128-byte rows: the swizzle permutes within rows.  The
  // register-table kernel reads the run tables only before its first tile, so
  // they overlay the buffers when they fit there; its adds also hold the
  // prefetched D vectors of every stage (K per thread).
  const size_t buf_elems = (((size_t)P.Ri * P.Li_pad * esize + 127) / 128) * 128 / esize;
  P.buf_elems = (int)buf_elems;
  P.ytab = (P.Lo <= kMaxTabLo || P.ymap.n < 0) ? 1 : 0;
  const size_t run_tabs = (size_t)P.Ri * 12 + (size_t)P.Ro * 16 + (P.ytab ? (size_t)P.Lo * 4 : 0) + 16;
  int64_t span_in = 0, span_out = 0;
  for (int i = 0; i < n; ++i) {
    span_in += (int64_t)(P.tl[i] - 1) * P.istr[i];
    span_out += (int64_t)(P.tl[i] - 1) * P.ostr[i];
  }
  // TALSH_B200_PERMUTE_GENERIC=1 sends every plan to the generic kernel (for tests).
  static const bool force_generic = [] {
    const char *e = std::getenv("TALSH_B200_PERMUTE_GENERIC");
    return e && std::atoi(e) == 1;
  }();
  P.reg = (!force_generic && span_in < INT_MAX && span_out < INT_MAX && P.V <= kThreads * reg_k(esize)) ? 1 : 0;
  const int stages = P.reg ? reg_stages(esize, op) : kStages;
  // Bulk-read form: rows of pitch_b bytes (16-byte aligned, an odd number of
  // 16-byte units), each holding a run's 16-byte-aligned cover.
  P.bulk = 0;
  if (P.reg && (cfg.bulk < 0 ? permute_bulk_wanted(esize, op, plan.vout) : cfg.bulk == 1)) {
    int pitch = (int)(((int64_t)P.Li * esize + 15 + 15) / 16 * 16);
    if ((pitch / 16) % 2 == 0) pitch += 16;
    const int64_t stage_b = ((int64_t)P.Ri * pitch + 127) / 128 * 128;
    if (stage_b + 16 < 65536) {
      P.bulk = 1;
      P.pitch_b = pitch;
      P.buf_elems = (int)(stage_b / esize);
      make_magic((uint32_t)P.Li_pad, P.mg_lip, P.sh_lip);
    }
  }
  const size_t stage_elems = (size_t)P.buf_elems;
  size_t bufs = (size_t)stages * stage_elems * esize;
  if (P.reg && op == kOpAdd && kAddPrefetch) {
    const int kreg = (P.V <= kThreads * 4) ? 4 : 8;  // the K permute_reg_kernel is launched with
    bufs += (size_t)stages * kreg * kThreads * esize;
  }
  size_t off = (P.reg && run_tabs <= bufs) ? 0 : ((bufs + 15) & ~size_t(15));
  P.off_rin = (int)off; off += (size_t)P.Ri * 8;
  P.off_wout = (int)off; off += (size_t)P.Ro * 8;
  P.off_rc = (int)off; off += (size_t)P.Ri * 4;
  P.off_wsm = (int)off; off += (size_t)P.Ro * 4;
  P.off_wc = (int)off; off += (size_t)P.Ro * 4;
  P.off_ysm = (int)off; if (P.ytab) off += (size_t)P.Lo * 4;
  P.off_tab_end = (int)off;
  off = std::max(off, bufs);
  {
    P.ta_rem = (int)(P.ext[P.a_last] - (P.ntile[P.a_last] - 1) * P.tl[P.a_last]);
    P.tb_rem = (int)(P.ext[P.b_last] - (P.ntile[P.b_last] - 1) * P.tl[P.b_last]);
    P.pre_bA = 1;
    for (int i = 0; i < P.b_last && P.b_in_A; ++i) P.pre_bA *= P.tl[i];
    P.pre_aB = 1;
    for (int k = 0; k < nb && P.a_in_B && q[k] != P.a_last; ++k) P.pre_aB *= P.tl[q[k]];
  }
  plan.smem = off;
  return TALSH_SUCCESS;
}

// Resident CTAs per SM for a kernel with `smem` dynamic bytes.  The kernel's
// dynamic shared-memory limit is raised once to the device maximum, so plans of
// any size can share the same kernel function.
int blocks_per_sm(const void *fn, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void *, size_t, int>, int> cache;  // (function, dynamic smem, device)
  static std::unordered_map<const void *, uint64_t> raised;  // per function: devices already set up
  std::lock_guard<std::mutex> lk(mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); dev = 0; }
  const uint64_t dev_bit = (dev >= 0 && dev < 64) ? (uint64_t(1) << dev) : 0;
  uint64_t &raised_on = raised[fn];
  if (dev_bit == 0 || (raised_on & dev_bit) == 0) {
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) optin = 0;
    cudaFuncAttributes fa;
    const int static_bytes = (cudaFuncGetAttributes(&fa, fn) == cudaSuccess) ? (int)fa.sharedSizeBytes : 1024;
    if (optin - static_bytes > 48 * 1024)
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - static_bytes);
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaGetLastError();
    raised_on |= dev_bit;
  }
  const auto key = std::make_tuple(fn, smem, dev);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kThreads, smem) != cudaSuccess || nb < 1) {
    cudaGetLastError();
    nb = 1;
  }
  cache[key] = nb;
  return nb;
}

struct ScaleArgs {
  double sr = 0.0, si = 0.0;
  const void *sdev = nullptr;
  int sdev_kind = 0, sdev_conj = 0;
};

template <typename T, int OP>
int launch_typed(const Plan &plan, const void *src, void *dst, int conj, const ScaleArgs &sc,
                 cudaStream_t st) {
  const int sms = current_sm_count();
  if (plan.linear) {
    constexpr int VEC = 16 / sizeof(T) > 0 ? 16 / sizeof(T) : 1;
    const bool aligned = ((uintptr_t)src % 16 == 0) && ((uintptr_t)dst % 16 == 0);
    const int64_t nvec = aligned ? plan.vol / VEC : 0;
    const int64_t tail = nvec * VEC;
    const void *fn = (const void *)linear_kernel<T, VEC, OP>;
    const int bps = blocks_per_sm(fn, 0);
    const int64_t want = (std::max<int64_t>(nvec, plan.vol - tail) + kThreads - 1) / kThreads;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * bps));
    linear_kernel<T, VEC, OP><<<grid, kThreads, 0, st>>>((const T *)src, (T *)dst, nvec, tail,
                                                         plan.vol, conj, sc.sr, sc.si, sc.sdev,
                                                         sc.sdev_kind, sc.sdev_conj);
    note_launch();
    return check_launch("linear_kernel");
  }
  PermParams P = plan.P;
  P.conj = conj;
  P.s_re = sc.sr;
  P.s_im = sc.si;
  P.sdev = sc.sdev;
  P.sdev_kind = sc.sdev_kind;
  P.sdev_conj = sc.sdev_conj;
  constexpr int VEC = 16 / sizeof(T);
  // 4-byte elements may also run with 8-byte vectors (VOUT 2), on the
  // register-table and bulk kernels
  int vout = plan.vout;
  if (vout != VEC && (VEC != 4 || !P.reg)) vout = 1;
  if (vout > 1 && ((uintptr_t)dst % ((uintptr_t)vout * sizeof(T))) != 0) vout = 1;
  P.y_step = (P.ymap.n >= 1 && P.ymap.ext[0] % vout == 0) ? 1 : 0;
  P.nv = P.Lo / vout;
  make_magic((uint32_t)P.nv, P.mg_nv, P.sh_nv);
  auto run = [&](auto kern) {
    const void *fn = (const void *)kern;
    const int bps = blocks_per_sm(fn, plan.smem);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(P.num_tiles, (int64_t)sms * bps));
    kern<<<grid, kThreads, plan.smem, st>>>((const T *)src, (T *)dst, P);
  };
  if (P.reg && P.bulk) {
    auto run_b = [&](auto kc) {
      constexpr int K = decltype(kc)::value;
      if (vout == VEC) run(permute_bulk_kernel<T, K, VEC, OP>);
      else if constexpr (VEC == 4) {
        if (vout == 2) run(permute_bulk_kernel<T, K, 2, OP>);
        else run(permute_bulk_kernel<T, K, 1, OP>);
      } else run(permute_bulk_kernel<T, K, 1, OP>);
    };
    if (P.V <= kThreads * 4) run_b(std::integral_constant<int, 4>{});
    else run_b(std::integral_constant<int, 8>{});
    note_launch();
    return check_launch("permute_bulk_kernel");
  }
  if (P.reg) {
    auto run_k = [&](auto kc) {
      constexpr int K = decltype(kc)::value;
      auto pick = [&](auto swz) {
        constexpr bool SW = decltype(swz)::value;
        if (vout == VEC) run(permute_reg_kernel<T, K, VEC, OP, SW>);
        else if constexpr (VEC == 4) {
          if (vout == 2) run(permute_reg_kernel<T, K, 2, OP, SW>);
          else run(permute_reg_kernel<T, K, 1, OP, SW>);
        } else run(permute_reg_kernel<T, K, 1, OP, SW>);
      };
      if (P.swz) pick(std::true_type{});
      else pick(std::false_type{});
    };
    if (P.V <= kThreads * 4) run_k(std::integral_constant<int, 4>{});
    else run_k(std::integral_constant<int, 8>{});
    note_launch();
    return check_launch("permute_reg_kernel");
  }
  if (P.swz) {
    if (vout > 1) run(permute_tiled_kernel<T, VEC, OP, true>);
    else run(permute_tiled_kernel<T, 1, OP, true>);
  } else {
    if (vout > 1) run(permute_tiled_kernel<T, VEC, OP, false>);
    else run(permute_tiled_kernel<T, 1, OP, false>);
  }
  note_launch();
  return check_launch("permute_tiled_kernel");
}

int validate(int kind, int rank, const int *dims, const int *o2n) {
  if (kind_size(kind) == 0) return TALSH_INVALID_ARGS;
  if (rank < 0 || rank > kMaxRank) return TALSH_INVALID_ARGS;
  if (rank > 0 && (dims == nullptr || o2n == nullptr)) return TALSH_INVALID_ARGS;
  bool seen[kMaxRank + 1] = {false};
  for (int i = 0; i < rank; ++i) {
    if (dims[i] <= 0) return TALSH_INVALID_ARGS;
    if (o2n[i] < 1 || o2n[i] > rank || seen[o2n[i]]) return TALSH_INVALID_ARGS;
    seen[o2n[i]] = true;
  }
  return TALSH_SUCCESS;
}

// ---------------------------------------------------------------------------
// Transpose autotuner.  Cases fall in classes by element kind, operation, the
// fused rank and permutation, the volume bucket (floor log2), the buckets of
// the input- and output-minor extents and whether those extents fill whole
// 16-byte units; tcTensorPermuteTune times the candidate plan choices of one
// case (CUDA events) and records the fastest for its class, which every later
// call of that class then uses.  Candidates: every combination of the read
// path (heuristics, bulk reads on, off), the tile size (heuristics, at most 4
// elements per thread), the tile walk order, the tile's growth order
// (heuristics, input runs first, output runs first), the initial run length
// (the planner's minimum, twice or four times that) and, for small tensors,
// the tile budget (shrunk so that every SM gets tiles, or kept).  Results do not depend on the choice (the same
// element arithmetic runs in every kernel), only the speed does.
// ---------------------------------------------------------------------------
// choice = bulk + 3 small + 6 flip + 12 grow + 36 longrun: bulk 0 the
// heuristics, 1 bulk reads on, 2 off; small 1: tiles of at most 4 elements per
// thread; flip 1: the other tile order; grow 0 the heuristics (the shorter run
// grows first), 1 input runs first, 2 output runs first; longrun 1 / 2:
// initial runs of at least 2 / 4 times the usual 32 elements (16 for 16-byte
// elements); keep 1 (code + 108): small tensors keep the full tile budget.
constexpr int kTuneConfigs = 216;
PlanCfg tune_cfg(int code) {
  PlanCfg c;
  if (code <= 0 || code >= kTuneConfigs) return c;
  const int b = code % 3;
  c.bulk = b == 0 ? -1 : (b == 1 ? 1 : 0);
  c.small = (code / 3) % 2;
  c.flip = (code / 6) % 2;
  c.grow = (code / 12) % 3 - 1;
  c.longrun = (code / 36) % 3;
  c.keep = code / 108;
  return c;
}

int ilog2_64(int64_t x) {
  int b = 0;
  while (x > 1) { x >>= 1; ++b; }
  return b;
}

// Class key of a fused case (0: not tunable -- straight copies and fused ranks
// above 6).
uint64_t tune_key(int kind, int op, const Fused &F) {
  if (F.n < 2 || F.n > 6) return 0;
  const int esize = kind_size(kind);
  int q0 = 0;
  for (int i = 0; i < F.n; ++i)
    if (F.perm[i] == 0) q0 = i;
  uint64_t k = (uint64_t)(kind & 3);
  k = (k << 1) | (uint64_t)(op == kOpAdd);
  k = (k << 3) | (uint64_t)F.n;
  for (int i = 0; i < F.n; ++i) k = (k << 3) | (uint64_t)F.perm[i];
  k = (k << 6) | (uint64_t)std::min(63, ilog2_64(F.vol));
  k = (k << 5) | (uint64_t)std::min(31, ilog2_64(F.ext[0]));
  k = (k << 5) | (uint64_t)std::min(31, ilog2_64(F.ext[q0]));
  k = (k << 1) | (uint64_t)((F.ext[0] * esize) % 16 == 0);
  k = (k << 1) | (uint64_t)((F.ext[q0] * esize) % 16 == 0);
  return k | (uint64_t(1) << 63);
}

std::mutex g_tune_mu;
std::unordered_map<uint64_t, int> g_tune_table;
std::atomic<int> g_tune_entries{0};

int tuned_choice(uint64_t key) {
  if (key == 0 || g_tune_entries.load(std::memory_order_relaxed) == 0) return -1;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune_table.find(key);
  return it == g_tune_table.end() ? -1 : it->second;
}

template <int OP>
int permute_entry(int kind, int rank, const int *dims, const int *o2n, const void *src, void *dst,
                  int conj, const ScaleArgs &sc, void *stream) {
  int rc = validate(kind, rank, dims, o2n);
  if (rc) return rc;
  if (src == nullptr || dst == nullptr) return TALSH_INVALID_ARGS;
  if (!elem_aligned(kind, src) || !elem_aligned(kind, dst)) return TALSH_INVALID_ARGS;
  if (!kind_is_complex(kind)) conj = 0;
  Fused F;
  if (rank == 0) { F.n = 0; F.vol = 1; }
  else if ((rc = fuse_dims(rank, dims, o2n, F)) != 0) return rc;
  const int choice = tuned_choice(tune_key(kind, OP, F));
  Plan plan;
  if ((rc = build_plan(kind_size(kind), F, plan, OP, tune_cfg(choice))) != 0) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  switch (kind) {
    case R4: return launch_typed<float, OP>(plan, src, dst, conj, sc, st);
    case R8: return launch_typed<double, OP>(plan, src, dst, conj, sc, st);
    case C4: return launch_typed<float2, OP>(plan, src, dst, conj, sc, st);
    case C8: return launch_typed<double2, OP>(plan, src, dst, conj, sc, st);
  }
  return TALSH_INVALID_ARGS;
}

}  // namespace
}  // namespace tb

extern "C" int tcTensorPermute(int data_kind, int rank, const int *dims_in, const int *o2n,
                               const void *src, void *dst, int conj, void *stream) {
  tb::ScaleArgs sc;
  return tb::permute_entry<tb::kOpCopy>(data_kind, rank, dims_in, o2n, src, dst, conj, sc, stream);
}

extern "C" int tcTensorPermuteAdd(int data_kind, int rank, const int *dims_in, const int *o2n,
                                  const void *src, void *dst, double alpha_re, double alpha_im,
                                  int conj, void *stream) {
  tb::ScaleArgs sc;
  sc.sr = alpha_re;
  sc.si = alpha_im;
  if (!tb::kind_is_complex(data_kind)) { sc.sr = tb::cmplx8_to_real8(alpha_re, alpha_im); sc.si = 0.0; }
  return tb::permute_entry<tb::kOpAdd>(data_kind, rank, dims_in, o2n, src, dst, conj, sc, stream);
}

namespace tb {
namespace {
template <int OP>
int launch_kind(int kind, const Plan &plan, const void *src, void *dst, const ScaleArgs &sc, cudaStream_t st) {
  switch (kind) {
    case R4: return launch_typed<float, OP>(plan, src, dst, 0, sc, st);
    case R8: return launch_typed<double, OP>(plan, src, dst, 0, sc, st);
    case C4: return launch_typed<float2, OP>(plan, src, dst, 0, sc, st);
    case C8: return launch_typed<double2, OP>(plan, src, dst, 0, sc, st);
  }
  return TALSH_INVALID_ARGS;
}
}  // namespace
}  // namespace tb

extern "C" int tcTensorPermuteTune(int data_kind, int rank, const int *dims_in, const int *o2n, int accumulate,
                                   const void *src, void *dst, void *stream, int reps, int *choice) {
  using namespace tb;
  int rc = validate(data_kind, rank, dims_in, o2n);
  if (rc) return rc;
  if (src == nullptr || dst == nullptr || reps < 1 || choice == nullptr) return TALSH_INVALID_ARGS;
  if (!elem_aligned(data_kind, src) || !elem_aligned(data_kind, dst)) return TALSH_INVALID_ARGS;
  *choice = 0;
  Fused F;
  if (rank == 0) return TALSH_SUCCESS;
  if ((rc = fuse_dims(rank, dims_in, o2n, F)) != 0) return rc;
  const int op = accumulate ? kOpAdd : kOpCopy;
  const uint64_t key = tune_key(data_kind, op, F);
  if (key == 0) return TALSH_SUCCESS;  // one plan only
  const int esize = kind_size(data_kind);
  Plan plans[kTuneConfigs];
  bool live[kTuneConfigs] = {false};
  for (int c = 0; c < kTuneConfigs; ++c) {
    if (build_plan(esize, F, plans[c], op, tune_cfg(c)) != 0) continue;
    live[c] = true;
    for (int d = 0; d < c && live[c]; ++d)  // a choice that changes nothing is not timed twice
      if (live[d] && plans[d].linear == plans[c].linear && plans[d].smem == plans[c].smem &&
          std::memcmp(&plans[d].P, &plans[c].P, sizeof(PermParams)) == 0)
        live[c] = false;
  }
  if (!live[0]) return TALSH_FAILURE;
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return TALSH_FAILURE;
  }
  ScaleArgs sc;
  sc.sr = 1.0;
  int best = 0;
  float best_ms = 0.0f;
  for (int c = 0; c < kTuneConfigs && rc == TALSH_SUCCESS; ++c) {
    if (!live[c]) continue;
    float ms = 0.0f;
    for (int r = 0; r <= reps && rc == TALSH_SUCCESS; ++r) {  // the first run warms up
      cudaEventRecord(e0, st);
      rc = (op == kOpAdd) ? launch_kind<kOpAdd>(data_kind, plans[c], src, dst, sc, st)
                          : launch_kind<kOpCopy>(data_kind, plans[c], src, dst, sc, st);
      cudaEventRecord(e1, st);
      if (rc == TALSH_SUCCESS && cudaEventSynchronize(e1) != cudaSuccess) rc = TALSH_FAILURE;
      float dt = 0.0f;
      if (rc == TALSH_SUCCESS && r > 0 && cudaEventElapsedTime(&dt, e0, e1) == cudaSuccess) ms += dt;
    }
    if (rc == TALSH_SUCCESS && (c == 0 || ms < best_ms)) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGetLastError();
  if (rc != TALSH_SUCCESS) return rc;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_table[key] = best;
    g_tune_entries.store((int)g_tune_table.size());
  }
  *choice = best;
  return TALSH_SUCCESS;
}

extern "C" int tcTensorPermuteTuned(int data_kind, int rank, const int *dims_in, const int *o2n, int accumulate,
                                    int *choice) {
  using namespace tb;
  int rc = validate(data_kind, rank, dims_in, o2n);
  if (rc) return rc;
  if (choice == nullptr) return TALSH_INVALID_ARGS;
  *choice = -1;
  if (rank == 0) return TALSH_SUCCESS;
  Fused F;
  if ((rc = fuse_dims(rank, dims_in, o2n, F)) != 0) return rc;
  *choice = tuned_choice(tune_key(data_kind, accumulate ? kOpAdd : kOpCopy, F));
  return TALSH_SUCCESS;
}

extern "C" int tcTensorPermuteTuneSet(int data_kind, int rank, const int *dims_in, const int *o2n, int accumulate,
                                      int choice) {
  using namespace tb;
  int rc = validate(data_kind, rank, dims_in, o2n);
  if (rc) return rc;
  if (choice < -1 || choice >= kTuneConfigs) return TALSH_INVALID_ARGS;
  if (rank == 0) return TALSH_SUCCESS;
  Fused F;
  if ((rc = fuse_dims(rank, dims_in, o2n, F)) != 0) return rc;
  const uint64_t key = tune_key(data_kind, accumulate ? kOpAdd : kOpCopy, F);
  if (key == 0) return TALSH_SUCCESS;
  if (choice >= 0) {  // the plan of the choice must exist for this case
    Plan plan;
    if (build_plan(kind_size(data_kind), F, plan, accumulate ? kOpAdd : kOpCopy, tune_cfg(choice)) != 0)
      return TALSH_INVALID_ARGS;
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (choice < 0) g_tune_table.erase(key);
  else g_tune_table[key] = choice;
  g_tune_entries.store((int)g_tune_table.size());
  return TALSH_SUCCESS;
}

extern "C" void tcTensorPermuteTuneReset(void) {
  using namespace tb;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_table.clear();
  g_tune_entries.store(0);
}

namespace tb {
// dst = permute(src) on a given stream, for the library's own staging steps.
int permute_launch_o2n(int kind, int rank, const int *dims, const int *o2n, const void *src, void *dst,
                       cudaStream_t st) {
  ScaleArgs sc;
  return permute_entry<kOpCopy>(kind, rank, dims, o2n, src, dst, 0, sc, (void *)st);
}

// dst (+)= permute(src) * (scalar_dev * alpha): the scalar-times-tensor case of a
// contraction, with the scale combined on the device (no host round trip).
int permute_scaled_by_device_scalar(int kind, int rank, const int *dims, const int *o2n,
                                    const void *src, void *dst, double alpha_re, double alpha_im,
                                    const void *scalar_dev, int scalar_conj, int tensor_conj,
                                    int accumulate, void *stream) {
  ScaleArgs sc;
  sc.sr = alpha_re;
  sc.si = alpha_im;
  sc.sdev = scalar_dev;
  sc.sdev_kind = kind;
  sc.sdev_conj = scalar_conj;
  if (accumulate)
    return permute_entry<kOpAdd>(kind, rank, dims, o2n, src, dst, tensor_conj, sc, stream);
  return permute_entry<kOpScaleCopy>(kind, rank, dims, o2n, src, dst, tensor_conj, sc, stream);
}
}  // namespace tb

// Host-side view of the plan, for tests and diagnostics.
extern "C" int tcPermutePlanInfo(int data_kind, int rank, const int *dims_in, const int *o2n,
                                 int *info /* [12] */) {
  int rc = tb::validate(data_kind, rank, dims_in, o2n);
  if (rc) return rc;
  tb::Fused F;
  if (rank == 0) { F.n = 0; F.vol = 1; }
  else if ((rc = tb::fuse_dims(rank, dims_in, o2n, F)) != 0) return rc;
  tb::Plan plan;
  if ((rc = tb::build_plan(tb::kind_size(data_kind), F, plan)) != 0) return rc;
  std::memset(info, 0, 12 * sizeof(int));
  info[0] = F.n;
  info[1] = plan.linear ? 1 : 0;
  if (!plan.linear) {
    info[2] = plan.P.V; info[3] = plan.P.Li; info[4] = plan.P.Lo;
    info[5] = plan.P.Ri; info[6] = plan.P.Ro; info[7] = plan.vin; info[8] = plan.vout;
    info[9] = (int)plan.smem;
    info[10] = (int)std::min<int64_t>(plan.P.num_tiles, INT_MAX);
    info[11] = plan.P.reg;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Batched transposes (tcPermuteBatch*).  Small tasks (up to kPBSmall output
// elements) run in ONE persistent launch over device-side task descriptors:
// every task is cut into chunks of kPBChunk output elements, the chunks of all
// small tasks are numbered through a prefix sum (largest tasks first), and
// each CTA takes chunk numbers from one atomic counter, finds the task by
// binary search and writes the chunk's output elements in order (coalesced),
// gathering each element from its input position (output coordinates by magic
// division, the input offset as a dot product with the input strides).  The
// arithmetic of an add is Arith<T>::axpy, as in the tiled kernels, so a
// task's result does not depend on the path that ran it.  Larger tasks keep
// their tiled plan (a tcTensorPermute(Add) launch).  Everything is recorded
// once into a CUDA graph -- counter reset, the persistent launch and the
// large tasks as concurrent branches -- and replayed with one launch.  No
// reference counterpart: the reference issues one gpu_tensor_block_copy / _add
// per call.
// ---------------------------------------------------------------------------
namespace tb {
namespace {

constexpr int64_t kPBSmall = 1 << 18;  // output elements: at most this many run in the persistent launch
constexpr int64_t kPBChunk = 4096;     // output elements per work item
constexpr int kPBMaxRank = TC_BATCH_MAX_RANK;
constexpr int kPBThreads = 256;

struct PBTask {
  const void *src;
  void *dst;
  int64_t first_chunk;     // prefix: first work item of this task
  int64_t vol;             // elements
  int rank;                // output dimensions after dropping unit extents
  int kind, add, conj;
  double sr, si;
  int32_t oext[kPBMaxRank];  // output extents, fastest first
  uint32_t mg[kPBMaxRank], sh[kPBMaxRank];
  int64_t istr[kPBMaxRank];  // input stride of each output dimension
};

template <typename T>
__device__ __forceinline__ void pb_chunk(const PBTask &d, int64_t e0, int64_t e1) {
  const T *src = (const T *)d.src;
  T *dst = (T *)d.dst;
  const bool cj = d.conj != 0;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += kPBThreads) {
    uint32_t rem = (uint32_t)e;  // vol < 2^31 for small tasks
    int64_t in = 0;
#pragma unroll 1
    for (int i = 0; i + 1 < d.rank; ++i) {
      const uint32_t q = fast_div(rem, d.mg[i], d.sh[i]);
      in += (int64_t)(rem - q * (uint32_t)d.oext[i]) * d.istr[i];
      rem = q;
    }
    if (d.rank > 0) in += (int64_t)rem * d.istr[d.rank - 1];
    T x = src[in];
    if (cj) x = Arith<T>::conj(x);
    if (d.add) dst[e] = Arith<T>::axpy(dst[e], x, d.sr, d.si);
    else dst[e] = x;
  }
}

__global__ void __launch_bounds__(kPBThreads) permute_batch_kernel(const PBTask *tasks, int ntasks,
                                                                   int64_t nchunks, unsigned long long *ctr) {
  __shared__ int64_t item_sh;
  __shared__ int task_sh;
  __shared__ __align__(16) PBTask d;  // the current task's descriptor
  for (;;) {
    if (threadIdx.x == 0) {
      const int64_t item = (int64_t)atomicAdd(ctr, 1ull);
      int lo = 0, hi = ntasks - 1;  // last task whose first chunk <= item
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].first_chunk <= item) lo = mid; else hi = mid - 1;
      }
      item_sh = item;
      task_sh = lo;
    }
    __syncthreads();
    const int64_t item = item_sh;
    if (item >= nchunks) return;
    {
      const uint32_t *from = reinterpret_cast<const uint32_t *>(tasks + task_sh);
      uint32_t *to = reinterpret_cast<uint32_t *>(&d);
      for (int w = threadIdx.x; w < (int)(sizeof(PBTask) / 4); w += kPBThreads) to[w] = from[w];
    }
    __syncthreads();
    const int64_t e0 = (item - d.first_chunk) * kPBChunk;
    const int64_t e1 = min(d.vol, e0 + kPBChunk);
    switch (d.kind) {
      case R4: pb_chunk<float>(d, e0, e1); break;
      case R8: pb_chunk<double>(d, e0, e1); break;
      case C4: pb_chunk<float2>(d, e0, e1); break;
      default: pb_chunk<double2>(d, e0, e1); break;
    }
    __syncthreads();  // d and item_sh are rewritten for the next item
  }
}

}  // namespace
}  // namespace tb

struct tcPermuteBatch {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *dev = nullptr;  // descriptors + work counter of the persistent launch
  int ntasks = 0;
  unsigned launches = 0;
};

extern "C" int tcPermuteBatchCreate(int ntasks, const tcPermuteTask *tasks, int branches, tcPermuteBatch **out) {
  using namespace tb;
  if (out == nullptr) return TALSH_INVALID_ARGS;
  *out = nullptr;
  if (ntasks < 1 || tasks == nullptr || branches < 1 || branches > 32) return TALSH_INVALID_ARGS;
  // Validate every task and split small (persistent launch) from large (tiled plan).
  std::vector<PBTask> small;
  std::vector<int> large;
  for (int t = 0; t < ntasks; ++t) {
    const tcPermuteTask &x = tasks[t];
    if (x.rank < 0 || x.rank > TC_BATCH_MAX_RANK) return TALSH_INVALID_ARGS;
    int rc = validate(x.data_kind, x.rank, x.dims, x.o2n);
    if (rc) return rc;
    if (x.src == nullptr || x.dst == nullptr) return TALSH_INVALID_ARGS;
    if (!elem_aligned(x.data_kind, x.src) || !elem_aligned(x.data_kind, x.dst)) return TALSH_INVALID_ARGS;
    int64_t vol = 1;
    for (int i = 0; i < x.rank; ++i) vol *= x.dims[i];
    if (vol > kPBSmall) { large.push_back(t); continue; }
    PBTask d;
    std::memset(&d, 0, sizeof(d));
    d.src = x.src; d.dst = x.dst; d.vol = vol; d.kind = x.data_kind; d.add = x.add ? 1 : 0;
    d.conj = kind_is_complex(x.data_kind) ? (x.conj ? 1 : 0) : 0;
    d.sr = x.alpha_re; d.si = x.alpha_im;
    if (x.add && !kind_is_complex(x.data_kind)) { d.sr = cmplx8_to_real8(x.alpha_re, x.alpha_im); d.si = 0.0; }
    // output order (fastest first) of the non-unit input dimensions
    int n2o[TC_BATCH_MAX_RANK];
    for (int i = 0; i < x.rank; ++i) n2o[x.o2n[i] - 1] = i;
    int64_t istr[TC_BATCH_MAX_RANK];
    int64_t s_ = 1;
    for (int i = 0; i < x.rank; ++i) { istr[i] = s_; s_ *= x.dims[i]; }
    int r = 0;
    for (int k = 0; k < x.rank; ++k) {
      const int i = n2o[k];
      if (x.dims[i] == 1) continue;
      d.oext[r] = x.dims[i];
      d.istr[r] = istr[i];
      make_magic((uint32_t)x.dims[i], d.mg[r], d.sh[r]);
      ++r;
    }
    d.rank = r;
    small.push_back(d);
  }
  std::stable_sort(small.begin(), small.end(), [](const PBTask &a, const PBTask &b) { return a.vol > b.vol; });
  int64_t nchunks = 0;
  for (PBTask &d : small) { d.first_chunk = nchunks; nchunks += (d.vol + kPBChunk - 1) / kPBChunk; }
  tcPermuteBatch *b = new tcPermuteBatch();
  b->ntasks = ntasks;
  int rc = TALSH_SUCCESS;
  const size_t desc_bytes = (sizeof(PBTask) * small.size() + 255) & ~size_t(255);
  if (!small.empty()) {
    if (cudaMalloc(&b->dev, desc_bytes + 256) != cudaSuccess ||
        cudaMemcpy(b->dev, small.data(), sizeof(PBTask) * small.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      note_cuda_error("tcPermuteBatchCreate descriptors", (int)cudaGetLastError());
      rc = TALSH_FAILURE;
    }
  }
  unsigned long long *ctr = b->dev ? (unsigned long long *)((char *)b->dev + desc_bytes) : nullptr;
  // Capture: counter reset and the persistent launch on stream 0; large tasks
  // round-robin over the other branches; all joined into stream 0.
  const int nbr = std::max(1, std::min(branches, 1 + (int)large.size()));
  std::vector<cudaStream_t> st(nbr, nullptr);
  std::vector<cudaEvent_t> ev(nbr + 1, nullptr);
  for (int i = 0; i < nbr && rc == TALSH_SUCCESS; ++i)
    if (cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking) != cudaSuccess) rc = TALSH_FAILURE;
  for (int i = 0; i <= nbr && rc == TALSH_SUCCESS; ++i)
    if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) rc = TALSH_FAILURE;
  int pb_grid = 1;
  if (rc == TALSH_SUCCESS && !small.empty()) {
    int bps = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, permute_batch_kernel, kPBThreads, 0) != cudaSuccess ||
        bps < 1)
      bps = 4;
    pb_grid = (int)std::max<int64_t>(1, std::min<int64_t>(nchunks, (int64_t)current_sm_count() * bps));
  }
  cudaGraph_t graph = nullptr;
  const unsigned before = (unsigned)tcKernelLaunchCount();
  if (rc == TALSH_SUCCESS) {
    if (cudaStreamBeginCapture(st[0], cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = TALSH_FAILURE;
    if (rc == TALSH_SUCCESS) {
      cudaEventRecord(ev[nbr], st[0]);
      for (int i = 1; i < nbr; ++i) cudaStreamWaitEvent(st[i], ev[nbr], 0);
      if (!small.empty()) {
        cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), st[0]);
        permute_batch_kernel<<<pb_grid, kPBThreads, 0, st[0]>>>((const PBTask *)b->dev, (int)small.size(), nchunks,
                                                                ctr);
        note_launch();
        rc = check_launch("permute_batch_kernel");
      }
      for (size_t j = 0; j < large.size() && rc == TALSH_SUCCESS; ++j) {
        const tcPermuteTask &x = tasks[large[j]];
        cudaStream_t s2 = st[nbr > 1 ? 1 + (int)(j % (size_t)(nbr - 1)) : 0];
        rc = x.add ? tcTensorPermuteAdd(x.data_kind, x.rank, x.dims, x.o2n, x.src, x.dst, x.alpha_re, x.alpha_im,
                                        x.conj, s2)
                   : tcTensorPermute(x.data_kind, x.rank, x.dims, x.o2n, x.src, x.dst, x.conj, s2);
      }
      for (int i = 1; i < nbr; ++i) {
        cudaEventRecord(ev[i], st[i]);
        cudaStreamWaitEvent(st[0], ev[i], 0);
      }
      const cudaError_t e = cudaStreamEndCapture(st[0], &graph);
      if (e != cudaSuccess && rc == TALSH_SUCCESS) {
        note_cuda_error("tcPermuteBatchCreate capture", (int)e);
        rc = TALSH_FAILURE;
      }
    }
  }
  b->launches = (unsigned)tcKernelLaunchCount() - before;
  if (rc == TALSH_SUCCESS && cudaGraphInstantiate(&b->exec, graph, 0) != cudaSuccess) rc = TALSH_FAILURE;
  b->graph = graph;
  cudaGetLastError();
  for (auto e : ev) if (e) cudaEventDestroy(e);
  for (auto s2 : st) if (s2) cudaStreamDestroy(s2);
  if (rc != TALSH_SUCCESS) {
    tcPermuteBatchDestroy(b);
    return rc;
  }
  *out = b;
  return TALSH_SUCCESS;
}

extern "C" int tcPermuteBatchLaunch(tcPermuteBatch *b, void *stream) {
  if (b == nullptr) return TALSH_INVALID_ARGS;
  const cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    tb::note_cuda_error("tcPermuteBatchLaunch", (int)e);
    return TALSH_FAILURE;
  }
  tb::note_launch(b->launches);
  return TALSH_SUCCESS;
}

extern "C" int tcPermuteBatchDestroy(tcPermuteBatch *b) {
  if (b == nullptr) return TALSH_INVALID_ARGS;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->dev) cudaFree(b->dev);
  delete b;
  return TALSH_SUCCESS;
}
