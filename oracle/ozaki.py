"""Model of the split-precision (Ozaki int8-slice) contraction -- TEST
INFRASTRUCTURE ONLY.

A numpy restatement of the arithmetic the split-precision form performs, used
to check its stated error bound on the CPU; the GPU form itself is checked
against the FP64 oracle (tests/test_split_gpu.py).  Steps:
  1. every row of A (M x K) and of Bt (N x K) is scaled by 2^-e, e the exponent
     of the row's largest magnitude, so all entries lie in (-1, 1);
  2. each scaled entry is cut into S signed 7-bit digits by truncation:
     x = sum_s d_s 2^(-7 s) + r, d_s in [-127, 127], |r| < 2^(-7 S);
  3. for every anti-diagonal g = s + t <= S + 1 the digit products are summed
     exactly in integers, P_g = sum_{s+t=g} D^A_s (D^B_t)^T;
  4. C = 2^(e_m + f_n) * sum_g 2^(-7 g) P_g in float64.
Only tests/ import this module.
"""
import numpy as np


def slice_rows(X, S):
    """Row exponents and the S digit planes (int64) of the rows of X."""
    X = np.asarray(X, dtype=np.float64)
    mx = np.abs(X).max(axis=1)
    e = np.where(mx > 0, np.frexp(mx)[1], 0)  # mx = f 2^e with f in [0.5, 1)
    v = np.ldexp(X, -e[:, None])
    digits = []
    for _ in range(S):
        y = v * 128.0
        t = np.trunc(y)
        digits.append(t.astype(np.int64))
        v = y - t
    return e, digits


def split_gemm(A, Bt, S):
    """C = A Bt^T through S slices per operand and the diagonals g <= S + 1."""
    ea, da = slice_rows(A, S)
    eb, db = slice_rows(Bt, S)
    C = np.zeros((A.shape[0], Bt.shape[0]), dtype=np.float64)
    for g in range(2, S + 2):
        P = np.zeros_like(C, dtype=np.int64)
        for s in range(1, g):
            t = g - s
            if s <= S and t <= S:
                P += da[s - 1] @ db[t - 1].T
        C += np.ldexp(P.astype(np.float64), -7 * g)
    return np.ldexp(C, ea[:, None] + eb[None, :])
