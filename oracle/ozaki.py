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
The floating-point slice forms (bf16, tf32 and e4m3 slices, fp32 sums per
diagonal) are modelled by split_gemm_float.  Only tests/ import this module.
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


# ---------------------------------------------------------------------------
# Floating-point slice forms (bf16, tf32, e4m3 slices; fp32 sums per diagonal)
# ---------------------------------------------------------------------------
FORM_BITS = {"bf16": 8, "tf32": 11, "fp8": 4}
FORM_KSTEP = {"bf16": 16, "tf32": 8, "fp8": 32}  # elements per 32-byte tensor-core K step


def _round_bits(x, p, min_exp=None):
    """Round to p significant bits (ties to even); below 2^min_exp the spacing is
    that of the smallest normal binade (subnormals), as e4m3's is below 2^-6."""
    x = np.asarray(x, dtype=np.float64)
    m, e = np.frexp(x)  # x = m 2^e, |m| in [0.5, 1)
    if min_exp is not None:
        e = np.maximum(e, min_exp + 1)
    q = np.ldexp(np.round(np.ldexp(x, -(e - p))), e - p)
    return np.where(x == 0, 0.0, q)


def round_slice(x, form):
    if form == "bf16":
        return _round_bits(x, 8)
    if form == "tf32":
        return _round_bits(x, 11)
    return _round_bits(x, 4, min_exp=-6)  # e4m3: 3 stored bits, min normal 2^-6


def slice_rows_float(X, S, form):
    """Row exponents and the S floating slices y_s (float64 values) of the rows of X:
    v = X 2^-e, y_s = round(v_s 2^(b s)), v_{s+1} = v_s - y_s 2^(-b s)."""
    X = np.asarray(X, dtype=np.float64)
    b = FORM_BITS[form]
    mx = np.abs(X).max(axis=1)
    e = np.where(mx > 0, np.frexp(mx)[1], 0)
    v = np.ldexp(X, -e[:, None])
    ys = []
    for s in range(S):
        y = round_slice(np.ldexp(v, b * s), form)
        ys.append(y)
        v = v - np.ldexp(y, -b * s)
    return e, ys


def split_gemm_float(A, Bt, S, form):
    """C = A Bt^T through S floating slices per operand, pairs s + t <= S - 1,
    one fp32 accumulator per diagonal, FP64 recombination."""
    b = FORM_BITS[form]
    ea, ya = slice_rows_float(A, S, form)
    eb, yb = slice_rows_float(Bt, S, form)
    C = np.zeros((A.shape[0], Bt.shape[0]), dtype=np.float64)
    kstep = FORM_KSTEP[form]
    K = A.shape[1]
    for g in range(0, S):
        acc = np.zeros_like(C, dtype=np.float32)
        for k0 in range(0, K, kstep):
            part = np.zeros_like(C)
            for s in range(0, g + 1):
                part += ya[s][:, k0:k0 + kstep] @ yb[g - s][:, k0:k0 + kstep].T
            acc = (acc.astype(np.float64) + part).astype(np.float32)
        C += np.ldexp(acc.astype(np.float64), -b * g)
    return np.ldexp(C, ea[:, None] + eb[None, :])
