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
#include <climits>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.h"

namespace tb {
namespace {

constexpr int kThreads = 256;
constexpr int kMinBlocks = 3;      // resident CTAs per SM the register budget is sized for
constexpr int kMaxFR = 40;         // max fused rank (every fused extent is >= 2)
constexpr int kTileBytes = 32768;  // bytes of one tile buffer (two buffers per CTA)
constexpr int kMaxTabLo = 4096;    // output run length when B needs a table (more than 3 dims)
constexpr int kMaxRuns = 1024;     // run count bound (run tables live in shared memory)
constexpr int kChunk = 256;        // elements (vectors on the write side) per warp chunk

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
  int nch_r, nch_w;   // warp chunks per input run (kChunk elements) / output run (kChunk*VOUT)
  uint32_t mg_cr, sh_cr, mg_cw, sh_cw;
  int ytab;           // 1: output-run positions come from the shared table ySm
  GroupMap rmap, wmap, ymap;
  int nra, nwb, nb;
  int conj;
  int off_rin, off_rc, off_wout, off_wsm, off_wc, off_ysm, off_tab_end;
  int buf_elems;      // elements per tile buffer (whole 128-byte rows)
  int64_t num_tiles;
  double s_re, s_im;
  const void *sdev;  // optional device scalar multiplying the scale (rank-0 operand)
  int sdev_kind, sdev_conj;
  int64_t ext[kMaxFR];
  int64_t istr[kMaxFR];
  int64_t ostr[kMaxFR];
  int64_t ntile[kMaxFR];
  int32_t tl[kMaxFR];
  int32_t smstr[kMaxFR];
  int8_t ra_dims[kMaxFR];
  int8_t wb_dims[kMaxFR];
  int8_t b_dims[kMaxFR];
};

struct TileSetup {
  int64_t in_base, out_base;
  int li_act, lo_act, ta_lim, tb_lim;
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
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Tile coordinates of one CTA, advanced by gridDim.x tiles at a time with
// mixed-radix carries (no divisions per tile).  Held by thread 0 in shared memory.
struct TileCursor {
  int32_t c[kMaxFR];
  int32_t step[kMaxFR];
};

__device__ void cursor_init(const PermParams &P, TileCursor &cur, int64_t first, int64_t step) {
  for (int i = 0; i < P.rank; ++i) {
    const int64_t nt = P.ntile[i];
    cur.c[i] = (int32_t)(first % nt);
    first /= nt;
    cur.step[i] = (int32_t)(step % nt);
    step /= nt;
  }
}

__device__ void cursor_advance(const PermParams &P, TileCursor &cur) {
  int carry = 0;
  for (int i = 0; i < P.rank; ++i) {
    const int32_t nt = (int32_t)P.ntile[i];
    int32_t v = cur.c[i] + cur.step[i] + carry;
    carry = 0;
    if (v >= nt) { v -= nt; carry = 1; }
    cur.c[i] = v;
  }
}

__device__ void make_setup(const PermParams &P, const TileCursor &cur, TileSetup &S) {
  int64_t in_base = 0, out_base = 0;
  int ta = P.tl[P.a_last], tb = P.tl[P.b_last];
  for (int i = 0; i < P.rank; ++i) {
    if (P.ntile[i] == 1) continue;
    const int64_t start = (int64_t)cur.c[i] * P.tl[i];
    in_base += start * P.istr[i];
    out_base += start * P.ostr[i];
    const int rem = (int)min((int64_t)P.tl[i], P.ext[i] - start);
    if (i == P.a_last) ta = rem;
    if (i == P.b_last) tb = rem;
  }
  S.in_base = in_base;
  S.out_base = out_base;
  S.li_act = P.a_pre * ta;
  S.lo_act = P.b_pre * tb;
  S.ta_lim = P.a_in_B ? INT_MAX : ta;
  S.tb_lim = P.b_in_A ? INT_MAX : tb;
}

template <typename T, int VOUT, int OP>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    permute_tiled_kernel(const T *__restrict__ src, T *dst, const PermParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  T *buf0 = reinterpret_cast<T *>(smem);
  T *buf1 = buf0 + P.buf_elems;
  int64_t *rIn = reinterpret_cast<int64_t *>(smem + P.off_rin);
  int32_t *rC = reinterpret_cast<int32_t *>(smem + P.off_rc);
  int64_t *wOut = reinterpret_cast<int64_t *>(smem + P.off_wout);
  int32_t *wSm = reinterpret_cast<int32_t *>(smem + P.off_wsm);
  int32_t *wC = reinterpret_cast<int32_t *>(smem + P.off_wc);
  int32_t *ySm = reinterpret_cast<int32_t *>(smem + P.off_ysm);
  __shared__ TileSetup setup[3];
  __shared__ TileCursor cursor;

  const int tid = threadIdx.x;
  const int64_t G = gridDim.x;
  // Per-CTA shared tables, valid for every tile of this plan: run offsets of
  // the input runs (global offset + coordinate of the output split dimension)
  // and of the output runs (global offset, shared offset, coordinate of the
  // input split dimension), and the shared offset of every output-run position.
  for (int r = tid; r < P.Ri; r += kThreads) {
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
  for (int r = tid; r < P.Ro; r += kThreads) {
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
    for (int y = tid; y < P.Lo; y += kThreads) {
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
  if (tid == 0 && blockIdx.x < P.num_tiles) {
    cursor_init(P, cursor, blockIdx.x, G);
    make_setup(P, cursor, setup[0]);
    cursor_advance(P, cursor);
    if (blockIdx.x + G < P.num_tiles) {
      make_setup(P, cursor, setup[1]);
      cursor_advance(P, cursor);
    }
  }
  __syncthreads();

  const bool cj = P.conj != 0;
  double sr = P.s_re, si = P.s_im;
  effective_scale<T>(P.sdev, P.sdev_kind, P.sdev_conj, sr, si);
  const int lane = tid & 31, warp = tid >> 5;
  constexpr int kWarps = kThreads / 32;

  // Read phase: warps take chunks of input runs (chunk = up to 256 elements);
  // one table lookup per chunk, then every lane streams elements 32 apart.
  auto issue_loads = [&](const TileSetup &S, T *buf) {
    const int nch = P.nch_r, total = P.Ri * nch;
    for (int it = warp; it < total; it += kWarps) {
      const int r = (int)fast_div((uint32_t)it, P.mg_cr, P.sh_cr);
      const int x0 = (it - r * nch) * kChunk;
      if (rC[r] >= S.tb_lim) continue;
      const int xe = min(x0 + kChunk, S.li_act);
      const T *g = src + (S.in_base + rIn[r]);
      const int sb = r * P.Li;
#pragma unroll 4
      for (int x = x0 + lane; x < xe; x += 32) cp_async_elem<sizeof(T)>(buf + swz<T>(sb + x), g + x);
    }
  };

  int64_t t = blockIdx.x;
  if (t < P.num_tiles) issue_loads(setup[0], buf0);
  cp_async_commit();
  for (int iter = 0; t < P.num_tiles; t += G, ++iter) {
    const int64_t tn = t + G;
    if (tn < P.num_tiles) issue_loads(setup[(iter + 1) % 3], (iter & 1) ? buf0 : buf1);
    cp_async_commit();
    if (tid == 0 && tn + G < P.num_tiles) {
      make_setup(P, cursor, setup[(iter + 2) % 3]);
      cursor_advance(P, cursor);
    }
    cp_async_wait_1();
    __syncthreads();
    // Write phase: warps take chunks of output runs; lanes move VOUT elements
    // per step with one (vector) store.
    const TileSetup S = setup[iter % 3];
    const T *buf = (iter & 1) ? buf1 : buf0;
    const int nch = P.nch_w, total = P.Ro * nch;
    for (int it = warp; it < total; it += kWarps) {
      const int r = (int)fast_div((uint32_t)it, P.mg_cw, P.sh_cw);
      const int y0 = (it - r * nch) * (kChunk * VOUT);
      if (wC[r] >= S.ta_lim) continue;
      const int ye = min(y0 + kChunk * VOUT, S.lo_act);
      T *g = dst + (S.out_base + wOut[r]);
      const int ws = wSm[r];
      constexpr int U = (OP == kOpAdd) ? 4 : 2;  // steps per batch (adds keep U loads of D in flight)
      for (int yb = y0 + lane * VOUT; yb < ye; yb += 32 * VOUT * U) {
        Pack<T, VOUT> v[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int y = yb + u * 32 * VOUT;
          ok[u] = y < ye;
          if (!ok[u]) continue;
          if (P.ytab) {
            if (P.y_step) {
              const int base = ws + ySm[y];
#pragma unroll
              for (int j = 0; j < VOUT; ++j) v[u].v[j] = buf[swz<T>(base + j * P.ymap.sstr[0])];
            } else {
#pragma unroll
              for (int j = 0; j < VOUT; ++j) v[u].v[j] = buf[swz<T>(ws + ySm[y + j])];
            }
          } else {
            if (P.y_step) {
              const int base = ws + decompose(P.ymap, (uint32_t)y).soff;
#pragma unroll
              for (int j = 0; j < VOUT; ++j) v[u].v[j] = buf[swz<T>(base + j * P.ymap.sstr[0])];
            } else {
#pragma unroll
              for (int j = 0; j < VOUT; ++j) v[u].v[j] = buf[swz<T>(ws + decompose(P.ymap, (uint32_t)(y + j)).soff)];
            }
          }
          if (cj) {
#pragma unroll
            for (int j = 0; j < VOUT; ++j) v[u].v[j] = Arith<T>::conj(v[u].v[j]);
          }
        }
        if constexpr (OP == kOpAdd) {
          Pack<T, VOUT> d[U];
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (ok[u]) d[u] = ld_pack<T, VOUT>(g + yb + u * 32 * VOUT);
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
#pragma unroll
            for (int j = 0; j < VOUT; ++j) d[u].v[j] = Arith<T>::axpy(d[u].v[j], v[u].v[j], sr, si);
            st_pack<T, VOUT>(g + yb + u * 32 * VOUT, d[u]);
          }
        } else {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (!ok[u]) continue;
            if constexpr (OP == kOpScaleCopy) {
#pragma unroll
              for (int j = 0; j < VOUT; ++j) v[u].v[j] = Arith<T>::mul(v[u].v[j], sr, si);
            }
            st_pack<T, VOUT>(g + yb + u * 32 * VOUT, v[u]);
          }
        }
      }
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
  for (int64_t target = cur * 2; target < ext; target += cur) {
    const int64_t pieces = (ext + target - 1) / target;
    const int64_t t = (ext + pieces - 1) / pieces;
    if (t > cur) return t;
  }
  return ext;
}

int build_plan(int esize, const Fused &F, Plan &plan) {
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

  // Small tensors get smaller tiles so that every SM still holds a few of them.
  int elems_max = tile_bytes() / esize;
  {
    const int64_t slots = 148LL * kMinBlocks * 2;
    while (elems_max > 1024 && F.vol / elems_max < slots) elems_max /= 2;
  }
  const int run_min = esize >= 16 ? 16 : 32;
  // Initial groups: shortest prefixes reaching run_min elements.
  int na = 0, nb = 0;
  int64_t tA = 1, tB = 1;
  {
    int64_t pre = 1;
    for (int i = 0; i < n; ++i) {
      if (pre * P.ext[i] >= run_min || i == n - 1) {
        na = i + 1;
        tA = std::min<int64_t>(P.ext[i], (run_min + pre - 1) / pre);
        break;
      }
      pre *= P.ext[i];
    }
    pre = 1;
    for (int k = 0; k < n; ++k) {
      if (pre * P.ext[q[k]] >= run_min || k == n - 1) {
        nb = k + 1;
        tB = std::min<int64_t>(P.ext[q[k]], (run_min + pre - 1) / pre);
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
      const bool growA = (pass == 0) ? (G.Li <= G.Lo) : !(G.Li <= G.Lo);
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
  P.num_tiles = 1;
  for (int i = 0; i < n; ++i) P.num_tiles *= P.ntile[i];
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
  // shared layout: x over A (input order) contiguous, runs over U\A with pitch Li_pad
  P.Li_pad = P.Li;  // no padding: shared indices are bank-swizzled instead
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
  P.nch_r = (P.Li + kChunk - 1) / kChunk;
  make_magic((uint32_t)P.nch_r, P.mg_cr, P.sh_cr);
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
  // length must be a multiple of 16 bytes.  Reads are element-granular
  // asynchronous copies and need no alignment beyond the element.
  const int vec = 16 / esize;
  plan.vin = 1;
  plan.vout = 1;
  if (vec > 1) {
    bool ok = (P.Lo % vec) == 0;
    const int64_t partial = P.ext[P.b_last] % P.tl[P.b_last];
    if (partial && ((int64_t)P.b_pre * partial) % vec) ok = false;
    for (int i = 0; i < n && ok; ++i) {
      if (!inB[i] && P.tl[i] > 1 && P.ostr[i] % vec) ok = false;       // run offsets
      if (P.ntile[i] > 1 && (P.tl[i] * P.ostr[i]) % vec) ok = false;   // tile bases
    }
    if (ok) plan.vout = vec;
  }
  // Shared memory: two tile buffers, then the tables that are in use.
  // each buffer is rounded up to whole 128-byte rows: the swizzle permutes within rows
  const size_t buf_elems = (((size_t)P.Ri * P.Li_pad * esize + 127) / 128) * 128 / esize;
  P.buf_elems = (int)buf_elems;
  size_t off = 2 * buf_elems * esize;
  off = (off + 15) & ~size_t(15);
  P.ytab = (P.Lo <= kMaxTabLo || P.ymap.n < 0) ? 1 : 0;
  P.off_rin = (int)off; off += (size_t)P.Ri * 8;
  P.off_wout = (int)off; off += (size_t)P.Ro * 8;
  P.off_rc = (int)off; off += (size_t)P.Ri * 4;
  P.off_wsm = (int)off; off += (size_t)P.Ro * 4;
  P.off_wc = (int)off; off += (size_t)P.Ro * 4;
  P.off_ysm = (int)off; if (P.ytab) off += (size_t)P.Lo * 4;
  P.off_tab_end = (int)off;
  plan.smem = off;
  return TALSH_SUCCESS;
}

int sm_count(int dev) {
  static int cache[64] = {0};
  if (dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cache[dev] = v;
  }
  return cache[dev];
}

// Resident CTAs per SM for a kernel with `smem` dynamic bytes.  The kernel's
// dynamic shared-memory limit is raised once to the device maximum, so plans of
// any size can share the same kernel function.
int blocks_per_sm(const void *fn, size_t smem) {
  static std::mutex mu;
  static std::unordered_map<uint64_t, int> cache;
  static std::unordered_map<const void *, bool> raised;
  std::lock_guard<std::mutex> lk(mu);
  if (!raised[fn]) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) optin = 0;
    cudaFuncAttributes fa;
    const int static_bytes = (cudaFuncGetAttributes(&fa, fn) == cudaSuccess) ? (int)fa.sharedSizeBytes : 1024;
    if (optin - static_bytes > 48 * 1024)
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - static_bytes);
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaGetLastError();
    raised[fn] = true;
  }
  const uint64_t key = (uint64_t)(uintptr_t)fn ^ ((uint64_t)smem << 44);
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
  int dev = 0;
  cudaGetDevice(&dev);
  const int sms = sm_count(dev);
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
  const bool dst_al = ((uintptr_t)dst % 16) == 0;
  const int vout = (plan.vout > 1 && dst_al) ? VEC : 1;
  P.y_step = (P.ymap.n >= 1 && P.ymap.ext[0] % vout == 0) ? 1 : 0;
  P.nch_w = (P.Lo + kChunk * vout - 1) / (kChunk * vout);
  make_magic((uint32_t)P.nch_w, P.mg_cw, P.sh_cw);
  auto run = [&](auto kern) {
    const void *fn = (const void *)kern;
    const int bps = blocks_per_sm(fn, plan.smem);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(P.num_tiles, (int64_t)sms * bps));
    kern<<<grid, kThreads, plan.smem, st>>>((const T *)src, (T *)dst, P);
  };
  if constexpr (VEC > 1) {
    if (vout > 1) run(permute_tiled_kernel<T, VEC, OP>);
    else run(permute_tiled_kernel<T, 1, OP>);
  } else {
    run(permute_tiled_kernel<T, 1, OP>);
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

template <int OP>
int permute_entry(int kind, int rank, const int *dims, const int *o2n, const void *src, void *dst,
                  int conj, const ScaleArgs &sc, void *stream) {
  int rc = validate(kind, rank, dims, o2n);
  if (rc) return rc;
  if (src == nullptr || dst == nullptr) return TALSH_INVALID_ARGS;
  if (!kind_is_complex(kind)) conj = 0;
  Fused F;
  if (rank == 0) { F.n = 0; F.vol = 1; }
  else if ((rc = fuse_dims(rank, dims, o2n, F)) != 0) return rc;
  Plan plan;
  if ((rc = build_plan(kind_size(kind), F, plan)) != 0) return rc;
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
  }
  return 0;
}
