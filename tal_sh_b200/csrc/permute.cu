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
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.h"

namespace tb {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxFR = 40;       // max fused rank (every fused extent is >= 2)
constexpr int kTileBytes = 32768;  // shared tile budget (bytes of elements)
constexpr int kMaxLo = 2048;     // output run length bound (ySm table)
constexpr int kMaxRuns = 1024;   // run count bound (rIn / wOut tables)

struct PermParams {
  int rank;
  int V, Li, Lo, Ri, Ro, Li_pad;
  uint32_t mg_li, sh_li, mg_lo, sh_lo;
  int a_last, b_last, a_pre, b_pre;
  int a_in_B, b_in_A;
  int nra, nwb, nb;
  int conj;
  int off_rin, off_rc, off_wout, off_wsm, off_wc, off_ysm;
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

__device__ void compute_setup(const PermParams &P, int64_t tile, TileSetup &S) {
  int64_t in_base = 0, out_base = 0;
  int ta = P.tl[P.a_last], tb = P.tl[P.b_last];
  for (int i = 0; i < P.rank; ++i) {
    const int64_t nt = P.ntile[i];
    if (nt == 1) continue;
    const int64_t c = tile % nt;
    tile /= nt;
    const int64_t start = c * P.tl[i];
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

template <typename T, int VIN, int VOUT, int OP>
__global__ void __launch_bounds__(kThreads) permute_tiled_kernel(const T *__restrict__ src,
                                                                 T *dst, const PermParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  T *tile = reinterpret_cast<T *>(smem);
  int64_t *rIn = reinterpret_cast<int64_t *>(smem + P.off_rin);
  int32_t *rC = reinterpret_cast<int32_t *>(smem + P.off_rc);
  int64_t *wOut = reinterpret_cast<int64_t *>(smem + P.off_wout);
  int32_t *wSm = reinterpret_cast<int32_t *>(smem + P.off_wsm);
  int32_t *wC = reinterpret_cast<int32_t *>(smem + P.off_wc);
  int32_t *ySm = reinterpret_cast<int32_t *>(smem + P.off_ysm);
  __shared__ TileSetup setup[2];

  const int tid = threadIdx.x;
  // Run tables for the full tile shape (shared by all tiles of this CTA).
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
    rC[r] = cb;
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
    wC[r] = ca;
  }
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
  if (tid == 0 && blockIdx.x < P.num_tiles) compute_setup(P, blockIdx.x, setup[0]);
  __syncthreads();

  constexpr int kTileElems = kTileBytes / (int)sizeof(T);
  constexpr int KR = (kTileElems + kThreads * VIN - 1) / (kThreads * VIN);
  constexpr int KW = (kTileElems + kThreads * VOUT - 1) / (kThreads * VOUT);
  const bool cj = P.conj != 0;
  double sr = P.s_re, si = P.s_im;
  effective_scale<T>(P.sdev, P.sdev_kind, P.sdev_conj, sr, si);

  int it = 0;
  for (int64_t t = blockIdx.x; t < P.num_tiles; t += gridDim.x, ++it) {
    const TileSetup S = setup[it & 1];
    // ---- read phase: global (input runs) -> shared ----
    {
      Pack<T, VIN> v[KR];
      int sidx[KR];
#pragma unroll
      for (int k = 0; k < KR; ++k) {
        const int e = (tid + k * kThreads) * VIN;
        sidx[k] = -1;
        if (e < P.V) {
          const int r = (int)fast_div((uint32_t)e, P.mg_li, P.sh_li);
          const int x = e - r * P.Li;
          if (x < S.li_act && rC[r] < S.tb_lim) {
            v[k] = ld_pack<T, VIN>(src + (S.in_base + rIn[r] + x));
            sidx[k] = x + r * P.Li_pad;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < KR; ++k) {
        if (sidx[k] >= 0) {
#pragma unroll
          for (int j = 0; j < VIN; ++j) tile[sidx[k] + j] = v[k].v[j];
        }
      }
    }
    __syncthreads();
    // ---- write phase: shared -> global (output runs) ----
    {
      Pack<T, VOUT> v[KW];
      int64_t goff[KW];
#pragma unroll
      for (int k = 0; k < KW; ++k) {
        const int e = (tid + k * kThreads) * VOUT;
        goff[k] = -1;
        if (e < P.V) {
          const int r = (int)fast_div((uint32_t)e, P.mg_lo, P.sh_lo);
          const int y = e - r * P.Lo;
          if (y < S.lo_act && wC[r] < S.ta_lim) {
            const int base = wSm[r];
#pragma unroll
            for (int j = 0; j < VOUT; ++j) {
              T x = tile[base + ySm[y + j]];
              if (cj) x = Arith<T>::conj(x);
              v[k].v[j] = x;
            }
            goff[k] = S.out_base + wOut[r] + y;
          }
        }
      }
      if constexpr (OP == kOpAdd) {
        Pack<T, VOUT> d[KW];
#pragma unroll
        for (int k = 0; k < KW; ++k)
          if (goff[k] >= 0) d[k] = ld_pack<T, VOUT>(dst + goff[k]);
#pragma unroll
        for (int k = 0; k < KW; ++k) {
          if (goff[k] >= 0) {
#pragma unroll
            for (int j = 0; j < VOUT; ++j) d[k].v[j] = Arith<T>::axpy(d[k].v[j], v[k].v[j], sr, si);
            st_pack<T, VOUT>(dst + goff[k], d[k]);
          }
        }
      } else if constexpr (OP == kOpScaleCopy) {
#pragma unroll
        for (int k = 0; k < KW; ++k) {
          if (goff[k] >= 0) {
#pragma unroll
            for (int j = 0; j < VOUT; ++j) v[k].v[j] = Arith<T>::mul(v[k].v[j], sr, si);
            st_pack<T, VOUT>(dst + goff[k], v[k]);
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < KW; ++k)
          if (goff[k] >= 0) st_pack<T, VOUT>(dst + goff[k], v[k]);
      }
    }
    if (tid == 0 && t + gridDim.x < P.num_tiles) compute_setup(P, t + gridDim.x, setup[(it + 1) & 1]);
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

struct Plan {
  bool linear = false;
  int64_t vol = 0;
  PermParams P;
  int vin = 1, vout = 1;
  size_t smem = 0;
};

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

  const int elems_max = kTileBytes / esize;
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
  auto acceptable = [&](const Geo &G) {
    return G.V <= elems_max && G.Lo <= kMaxLo && G.V / G.Li <= kMaxRuns && G.V / G.Lo <= kMaxRuns;
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
          tA2 = std::min<int64_t>(P.ext[al], G.tl[al] * 2);
        } else if (na < n) {
          na2 = na + 1;
          tA2 = std::min<int64_t>(P.ext[na2 - 1], std::max<int64_t>(2, G.tl[na2 - 1]));
        } else {
          continue;
        }
      } else {
        const int bl = q[nb - 1];
        if (G.tl[bl] < P.ext[bl]) {
          tB2 = std::min<int64_t>(P.ext[bl], G.tl[bl] * 2);
        } else if (nb < n) {
          nb2 = nb + 1;
          tB2 = std::min<int64_t>(P.ext[q[nb2 - 1]], std::max<int64_t>(2, G.tl[q[nb2 - 1]]));
        } else {
          continue;
        }
      }
      Geo G2;
      geometry(na2, tA2, nb2, tB2, G2);
      if (acceptable(G2)) {
        na = na2; nb = nb2; tA = tA2; tB = tB2; G = G2;
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
  P.Li_pad = (P.Li % 2 == 0) ? P.Li + 1 : P.Li;
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
  // Vector widths: every run start, run length and partial run length must be
  // a multiple of the vector (16 bytes) on that side.
  const int vec = 16 / esize;
  plan.vin = plan.vout = 1;
  if (vec > 1) {
    auto side_ok = [&](bool in_side) {
      const int L = in_side ? P.Li : P.Lo;
      if (L % vec) return false;
      const int last = in_side ? P.a_last : P.b_last;
      const int pre = in_side ? P.a_pre : P.b_pre;
      const int64_t partial = P.ext[last] % P.tl[last];
      if (partial && ((int64_t)pre * partial) % vec) return false;
      for (int i = 0; i < n; ++i) {
        const int64_t st = in_side ? P.istr[i] : P.ostr[i];
        const bool in_group = in_side ? inA[i] : inB[i];
        if (!in_group && P.tl[i] > 1 && st % vec) return false;      // run offsets
        if (P.ntile[i] > 1 && (P.tl[i] * st) % vec) return false;    // tile bases
      }
      return true;
    };
    if (side_ok(true)) plan.vin = vec;
    if (side_ok(false)) plan.vout = vec;
  }
  // Shared memory carve-up.
  size_t off = (size_t)P.Ri * P.Li_pad * esize;
  off = (off + 15) & ~size_t(15);
  P.off_rin = (int)off; off += (size_t)P.Ri * 8;
  P.off_wout = (int)off; off += (size_t)P.Ro * 8;
  P.off_rc = (int)off; off += (size_t)P.Ri * 4;
  P.off_wsm = (int)off; off += (size_t)P.Ro * 4;
  P.off_wc = (int)off; off += (size_t)P.Ro * 4;
  P.off_ysm = (int)off; off += (size_t)P.Lo * 4;
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

int blocks_per_sm(const void *fn, size_t smem) {
  static std::mutex mu;
  static std::unordered_map<uint64_t, int> cache;
  const uint64_t key = (uint64_t)(uintptr_t)fn ^ ((uint64_t)smem << 48);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int nb = 0;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kThreads, smem) != cudaSuccess || nb < 1)
    nb = 1;
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
  const bool src_al = ((uintptr_t)src % 16) == 0, dst_al = ((uintptr_t)dst % 16) == 0;
  const int vin = (plan.vin > 1 && src_al) ? VEC : 1;
  const int vout = (plan.vout > 1 && dst_al) ? VEC : 1;
  auto run = [&](auto kern) {
    const void *fn = (const void *)kern;
    const int bps = blocks_per_sm(fn, plan.smem);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(P.num_tiles, (int64_t)sms * bps));
    kern<<<grid, kThreads, plan.smem, st>>>((const T *)src, (T *)dst, P);
  };
  if constexpr (VEC > 1) {
    if (vin > 1 && vout > 1) run(permute_tiled_kernel<T, VEC, VEC, OP>);
    else if (vin > 1) run(permute_tiled_kernel<T, VEC, 1, OP>);
    else if (vout > 1) run(permute_tiled_kernel<T, 1, VEC, OP>);
    else run(permute_tiled_kernel<T, 1, 1, OP>);
  } else {
    run(permute_tiled_kernel<T, 1, 1, OP>);
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
