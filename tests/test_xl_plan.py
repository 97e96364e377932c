"""The out-of-core decomposition of talshTensorContractXL, planned on the host
(tcContractXLPlan), against the oracle's restatement of the reference's
halving rule (talshTensorOpDecompose2, talshc.cpp:3150-3294): the same pieces,
in the same order, covering every element of D, L and R."""
import itertools

import numpy as np
import pytest

import tal_sh_b200 as T
from oracle.decompose import xl_plan

CASES = [  # pattern, extents, kind, budget
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=24, b=20, c=18, i=9, j=8, k=7), T.R8, 1 << 20),
    ("D(a,b)+=L(k,a,c)*R(c,k,b)", dict(a=70, b=60, c=40, k=30), T.C8, 1 << 19),
    ("D(i,j,k)+=L(k,a,i,b)*R(b,k,a,j)", dict(i=30, j=20, k=16, a=12, b=10), T.C8, 1 << 20),  # hyper k
    ("D()+=L(a,b,c)*R(c,b,a)", dict(a=60, b=50, c=40), T.R8, 1 << 18),                       # full
    ("D(a,b,c)+=L(c,a)*R(b,c)", dict(a=33, b=17, c=65), T.R4, 1 << 14),                        # hyper, no k
    ("D(a,b,c,d)+=L(a,b)*R(c,d)", dict(a=31, b=7, c=19, d=40), T.R8, 1 << 16),                 # outer product
]


def _dims(pattern, ext):
    import re
    return [[ext[x] for x in g.split(",") if x] for g in re.findall(r"\(([^)]*)\)", pattern)]


@pytest.mark.parametrize("pattern,ext,kind,budget", CASES)
def test_xl_plan_matches_the_reference_rule(built, pattern, ext, kind, budget):
    L = T.lib()
    e, dig, dr, lr, rr, _ = T.parse_pattern(pattern)
    dd, ld, rd = _dims(pattern, ext)
    es = {T.R4: 4, T.R8: 8, T.C4: 8, T.C8: 16}[kind]
    want = xl_plan(dig, dd, ld, rd, es, budget)
    assert want is not None and len(want) > 1  # every case decomposes
    w = dr + lr + rr
    n = len(want)
    offs, exts = T.ivec([0] * (n * w)), T.ivec([0] * (n * w))
    got = L.tcContractXLPlan(kind, T.ivec(dig), dr, T.ivec(dd), lr, T.ivec(ld), rr, T.ivec(rd), budget, n, offs,
                             exts)
    assert got == n, (got, n)
    for p, (o, d) in enumerate(want):
        assert list(offs[p * w:(p + 1) * w]) == o[0] + o[1] + o[2]
        assert list(exts[p * w:(p + 1) * w]) == d[0] + d[1] + d[2]
        need = es * sum(int(np.prod(x)) if x else 1 for x in d)
        assert need * 4 <= budget or all(v == 1 for x in d for v in x)
    # the D pieces tile D (each element once per contracted-index piece it belongs to)
    # and the L / R pieces together cover L and R
    for a, full in enumerate((dd, ld, rd)):
        cover = np.zeros(full if full else [1], dtype=np.int64)
        for o, d in want:
            idx = tuple(slice(o[a][i], o[a][i] + d[a][i]) for i in range(len(full))) if full else (0,)
            cover[idx] += 1
        assert cover.min() >= 1


def test_xl_plan_limits(built):
    L = T.lib()
    e, dig, dr, lr, rr, _ = T.parse_pattern("D(a,b)+=L(a,k)*R(k,b)")
    args = (T.R8, T.ivec(dig), dr, T.ivec([512, 512]), lr, T.ivec([512, 512]), rr, T.ivec([512, 512]))
    assert L.tcContractXLPlan(*args, 1 << 40, 4, None, None) == 1            # fits: one piece
    assert L.tcContractXLPlan(*args, 1 << 10, 4, None, None) == T.TALSH_LIMIT_EXCEEDED
    assert L.tcContractXLPlan(T.R8, T.ivec(dig), dr, T.ivec([512, 0]), lr, T.ivec([512, 512]), rr,
                              T.ivec([512, 512]), 1 << 20, 4, None, None) == T.TALSH_INVALID_ARGS
