// A complex(8) contraction written as one real(8) contraction (host code; the
// split-precision form runs complex contractions this way).
//
// With the conjugation flags applied (the D flag flips the L and R flags, as in
// the reference's get_contraction_permutations, tensor_algebra_cpu.F90:5757-5956),
// let X = R or conj(R).  Then
//   Re(L X) = sum_k Lr Yr + Li Yi,   Im(L X) = sum_k Lr Zr + Li Zi,
// with Y = conj(X), Z = i conj(X) when L is not conjugated, and Y = X, Z = -i X
// when it is (conj(L) X has real part Lr Xr + Li Xi, imaginary part Lr Xi - Li Xr).
// A complex tensor's body read as real numbers is a real tensor with one more,
// leading index c of extent 2 (its interleaved (re, im) pairs).  Stacking Y and Z
// along a trailing index e of extent 2 into one complex tensor Rx(r..., e) gives
//   D'(e, d...) = sum_{c, k} L'(c, l...) Rx'(c, r..., e),
// a real contraction over the bodies of D and L as they are stored and the body
// of Rx.  alpha is folded into Rx by taking alpha X for X: Y and Z then carry
// conj(alpha) when L is not conjugated, alpha when it is.  The product is
// M x 2N x 2K: 8 M N K flops, the complex count.
#pragma once

#include "talsh.h"

namespace tb {

struct ComplexSplitForm {
  int cptrn[2 * MAX_TENSOR_RANK];
  int drank = 0, lrank = 0, rrank = 0;
  int ddims[MAX_TENSOR_RANK];
  int ldims[MAX_TENSOR_RANK];
  int rdims[MAX_TENSOR_RANK];
  int y_conj = 0;      // Y = conj(R) when 1, R when 0
  double z_im = 1.0;   // Z = Y * (0 + z_im i), z_im = +1 or -1
  int alpha_conj = 1;  // Y and Z carry conj(alpha) when 1, alpha when 0
};

// The real form of a complex contraction (pattern and extents as for
// tcTensorContract, already validated).  Returns TALSH_LIMIT_EXCEEDED when a
// rewritten rank would exceed MAX_TENSOR_RANK.
inline int complex_split_form(const int *cptrn, int drank, const int *ddims, int lrank, const int *ldims,
                              int rrank, const int *rdims, int conj_bits, ComplexSplitForm &f) {
  if (drank + 1 > MAX_TENSOR_RANK || lrank + 1 > MAX_TENSOR_RANK || rrank + 2 > MAX_TENSOR_RANK)
    return TALSH_LIMIT_EXCEEDED;
  int cl = (conj_bits >> 1) & 1, cr = (conj_bits >> 2) & 1;
  if (conj_bits & 1) { cl ^= 1; cr ^= 1; }
  f.y_conj = cl ? cr : cr ^ 1;
  f.z_im = cl ? -1.0 : 1.0;
  f.alpha_conj = cl ^ 1;
  f.drank = drank + 1;
  f.lrank = lrank + 1;
  f.rrank = rrank + 2;
  const auto shift = [](int v) { return v > 0 ? v + 1 : v - 1; };
  // L': c (partner: position 1 of Rx'), then L's indices.
  f.cptrn[0] = -1;
  f.ldims[0] = 2;
  for (int i = 0; i < lrank; ++i) {
    f.cptrn[1 + i] = shift(cptrn[i]);
    f.ldims[1 + i] = ldims[i];
  }
  // Rx': c (partner: position 1 of L'), R's indices, e (position 1 of D').
  int *rp = f.cptrn + f.lrank;
  rp[0] = -1;
  f.rdims[0] = 2;
  for (int j = 0; j < rrank; ++j) {
    rp[1 + j] = shift(cptrn[lrank + j]);
    f.rdims[1 + j] = rdims[j];
  }
  rp[1 + rrank] = 1;
  f.rdims[1 + rrank] = 2;
  f.ddims[0] = 2;
  for (int i = 0; i < drank; ++i) f.ddims[1 + i] = ddims[i];
  return TALSH_SUCCESS;
}

}  // namespace tb
