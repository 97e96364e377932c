"""Tensor contraction on the GPU through talshTensorContract against the oracle
(reference tensor_block_contract): relative Frobenius error <= 1e-12 for R8/C8,
<= 2e-5 for R4/C4 (single-precision accumulation), plus the reference tests'
known answers."""
import json
import os

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, gpu_contract, rand, rel_err

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = {T.R8: 1e-12, T.C8: 1e-12, T.R4: 2e-5, T.C4: 2e-5}


def run_case(pattern, dd, ld, rd, kind, alpha=(1.0, 0.0), accumulative=True, seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    L, R, D0 = rand(ld, kind, rng, scale), rand(rd, kind, rng, scale), rand(dd, kind, rng)
    D = D0.copy(order="F")
    assert gpu_contract(pattern, D, L, R, *alpha, accumulative=accumulative) == 0, pattern
    e, dig, _, _, _, cj = O.str2dig(pattern)
    ref = D0.copy(order="F")
    assert O.tensor_contract(ref, L, R, dig, alpha[0], alpha[1], cj, accumulative) == 0
    err = rel_err(D, ref)
    assert err <= TOL[kind], (pattern, kind, err)
    return err


CASES = [
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", (9, 10, 7, 6), (9, 5, 11, 7), (11, 10, 5, 6)),
    ("D(a,b,c,d)+=L(d,c,i,j)*R(b,a,i,j)", (6, 5, 4, 3), (3, 4, 7, 5), (5, 6, 7, 5)),
    ("D(a,b,i,j)+=L(c,b,d,a)*R(j,d,i,c)", (8, 8, 4, 4), (8, 8, 8, 8), (4, 8, 4, 8)),
    ("D(a,b)+=L(a,c)*R(c,b)", (130, 70), (130, 257), (257, 70)),
    ("D(a,b)+=L(c,a)*R(b,c)", (33, 65), (129, 33), (65, 129)),
    ("D(a,b)+=L(a)*R(b)", (37, 41), (37,), (41,)),
    ("D()+=L(a,b,c)*R(c,a,b)", (), (13, 17, 19), (19, 13, 17)),
    ("D(b,a)+=L(a,b)*R()", (21, 13), (13, 21), ()),
    ("D(a,b)+=L()*R(b,a)", (21, 13), (), (13, 21)),
    ("D()+=L()*R()", (), (), ()),
    ("D(a,b,c)+=L(a,d,e)*R(e,b,c,d)", (7, 6, 5), (7, 4, 3), (3, 6, 5, 4)),
]


@pytest.mark.parametrize("kind", [T.R8, T.C8, T.R4, T.C4])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_contract_parity(talsh, case, kind):
    pat, dd, ld, rd = case
    run_case(pat, dd, ld, rd, kind, alpha=(-1.25, 0.0))
    run_case(pat, dd, ld, rd, kind, alpha=(0.5, 0.0), accumulative=False, seed=1)
    if kind in (T.C4, T.C8):
        run_case(pat, dd, ld, rd, kind, alpha=(0.25, -0.75), seed=2)


@pytest.mark.parametrize("kind", [T.C8, T.C4])
@pytest.mark.parametrize("pat", ["D(a,b,i,j)+=L+(a,k,c,i)*R(c,b,k,j)", "D(a,b,i,j)+=L(a,k,c,i)*R+(c,b,k,j)",
                                 "D+(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", "D(a,b,i,j)+=L+(a,k,c,i)*R+(c,b,k,j)",
                                 "D()+=L+(a,b)*R(b,a)", "D(b,a)+=L+(a,b)*R()", "D(b,a)+=L()*R+(a,b)"])
def test_conjugated_contractions(talsh, kind, pat):
    shapes = {"D(a,b,i,j)": ((6, 7, 5, 4), (6, 3, 8, 5), (8, 7, 3, 4)), "D()": ((), (9, 11), (11, 9)),
              "D(b,a)+=L+(a,b)*R()": ((5, 4), (4, 5), ()), "D(b,a)+=L()*R+": ((5, 4), (), (4, 5))}
    key = next(k for k in shapes if pat.replace("+(", "(").startswith(k.replace("+(", "(")) or pat.startswith(k))
    dd, ld, rd = shapes[key]
    run_case(pat, dd, ld, rd, kind, alpha=(0.5, 0.5), seed=3)


def test_c1_full_size(talsh):
    """C1: D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j), extents 32, L and R uniform[-1,1] from seed 0, D = 0."""
    L = O.uniform((32,) * 4, O.R8, 0)
    R = O.uniform((32,) * 4, O.R8, 1)
    D = fort(np.zeros((32,) * 4))
    assert gpu_contract("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", D, L, R) == 0
    ref = fort(np.zeros((32,) * 4))
    e, dig, _, _, _, _ = O.str2dig("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)")
    assert O.tensor_contract(ref, L, R, dig) == 0
    assert rel_err(D, ref) <= 1e-12


def test_large_tiles_r8(talsh):
    """Shapes that select the 128x128 DMMA tile (>= 2 tiles per SM)."""
    run_case("D(a,b)+=L(k,a)*R(k,b)", (2304, 2176), (96, 2304), (96, 2176), T.R8, alpha=(0.75, 0.0), seed=5)
    run_case("D(a,b,c)+=L(a,k,b)*R(k,c)", (48, 50, 2100), (48, 33, 50), (33, 2100), T.R8, seed=6)


def test_reference_benchmark_patterns(talsh):
    """The 48 patterns of the reference's tensor_contractions.txt, extents scaled
    down (every extent e -> 2 + e % 5 + small offset) to keep the oracle fast."""
    cases = json.load(open(os.path.join(GOLD, "tensor_contractions.json")))
    for n, c in enumerate(cases):
        e, dig, dr, lr, rr, cj = O.str2dig(c["pattern"])
        assert e == 0
        label_ext = {}
        ext = []
        for pos in range(dr):
            ext.append(3 + (c["D"][pos] + pos) % 4)
        dd = ext
        ld = [dd[v - 1] if v > 0 else None for v in dig[:lr]]
        rd = [dd[v - 1] if v > 0 else None for v in dig[lr:]]
        for i, v in enumerate(dig[:lr]):
            if v < 0:
                ld[i] = rd[-v - 1] = 2 + (c["L"][i] + i) % 6
        run_case(c["pattern"], tuple(dd), tuple(ld), tuple(rd), T.R8, alpha=(1.0, 0.0), seed=n)


def test_known_answer_talsh_c(talsh):
    """test.cpp:38-165 with the reference sizes V=40, O=20: constant inputs, alpha=2;
    every element of D equals 2*V*V*1e-5 and the 1-norm is gflops*1e-5*1e9."""
    V, Od = 40, 20
    pat = json.load(open(os.path.join(GOLD, "patterns.json")))["talsh_c_pattern"]
    D = fort(np.zeros((V, V, Od, Od)))
    L = fort(np.full((V, V, V, V), 0.001))
    R = fort(np.full((Od, V, Od, V), 0.01))
    assert gpu_contract(pat, D, L, R, 2.0) == 0
    gflops = np.sqrt(float(D.size) * L.size * R.size) * 2.0 / 1e9
    assert np.allclose(D, 2.0 * V * V * 1e-5, rtol=1e-13)
    assert abs(O.norm1(D) - gflops * 0.01 * 0.001 * 1e9) <= 1e-9 * gflops * 1e4


def test_known_answer_nwchem(talsh):
    """test.cpp:895-1013: alpha=-2 then +1 on the GPU, then the explicit loop: residual 0."""
    rng = np.random.default_rng(7)
    Vd, Od = 5, 2
    pat = json.load(open(os.path.join(GOLD, "patterns.json")))["nwchem_pattern"]
    D = fort(np.zeros((Od, Vd)))
    L = fort(1e6 / (rng.integers(0, 2 ** 31, (Vd, Od)) + 1.0))
    R = fort(1e5 / (rng.integers(0, 2 ** 31, (Od, Od, Vd, Vd)) + 1.0))
    assert gpu_contract(pat, D, L, R, -2.0) == 0
    assert gpu_contract(pat, D, L, R, 1.0) == 0
    D += np.einsum("cd,dabc->ab", L, R)
    assert np.abs(D).sum() <= 1e-12 * np.abs(np.einsum("cd,dabc->ab", L, R)).sum()


HYPER_CASES = [  # indices in D, L and R: one GEMM per hyper combination
    ("D(a,b,c)+=L(c,a)*R(b,c)", dict(a=3, b=4, c=5)),                       # no contracted index
    ("D(i,j,k)+=L(k,a,i,b)*R(b,k,a,j)", dict(i=12, j=10, k=7, a=6, b=5)),   # the reference's hyper test shape
    ("D(x,h,g)+=L(x,h,k,g)*R(g,k,h)", dict(h=4, g=3, x=33, k=17)),          # two hyper indices, R without free index
    ("D(h)+=L(k,h)*R(h,k)", dict(h=9, k=40)),                                # D only hyper: a dot per h
    ("D(a,h,b)+=L(a,k,h)*R(h,k,b)", dict(a=70, b=66, h=1, k=20)),            # extent-1 hyper index
]


@pytest.mark.parametrize("kind", [T.R8, T.C8, T.R4, T.C4])
@pytest.mark.parametrize("pattern,ext", HYPER_CASES)
def test_hyper_contractions_match_oracle(talsh, pattern, ext, kind):
    """Hyper-contractions (reference nhu path, tensor_algebra_cpu.F90:5829-5839,
    tensor_block_pcontract_batch_dlf :11256) against the oracle."""
    import re
    rng = np.random.default_rng(8)
    groups = [[x for x in g.split(",") if x] for g in re.findall(r"\(([^)]*)\)", pattern)]
    dd, ld, rd = ([ext[x] for x in g] for g in groups)
    D, L, R = rand(dd, kind, rng), rand(ld, kind, rng), rand(rd, kind, rng)
    ref = D.copy(order="F")
    e, dig, *_ = T.parse_pattern(pattern)
    alpha = (0.5, -0.25) if kind in (T.C4, T.C8) else (0.5, 0.0)
    assert O.tensor_contract(ref, L, R, dig, alpha[0], alpha[1], 0, True) == 0
    got = D.copy(order="F")
    assert gpu_contract(pattern, got, L, R, alpha[0], alpha[1]) == 0
    tol = 1e-12 if kind in (T.R8, T.C8) else 2e-5
    assert np.linalg.norm(got - ref) <= tol * np.linalg.norm(ref - D), (pattern, kind)


def test_hyper_indices_anywhere_in_d(talsh):
    """Hyper indices ahead of simple ones in D.  The reference's CPU matricization
    assumes they trail D (get_contraction_permutations, tensor_algebra_cpu.F90:5878,
    puts them at D's end unpermuted) and the oracle follows it, so this placement is
    checked against an FP64 einsum instead."""
    rng = np.random.default_rng(12)
    for pattern, spec, dims in (("D(h,g,x)+=L(x,h,k,g)*R(g,k,h)", "xhkg,gkh->hgx", ((4, 3, 33), (33, 4, 17, 3), (3, 17, 4))),
                                ("D(b,h,a)+=L(a,k,h)*R(h,b,k)", "akh,hbk->bha", ((21, 5, 19), (19, 23, 5), (5, 21, 23)))):
        for kind in (T.R8, T.C8):
            D, L, R = (rand(d, kind, rng) for d in dims)
            got = D.copy(order="F")
            assert gpu_contract(pattern, got, L, R, 0.5, 0.0) == 0
            want = D + 0.5 * np.einsum(spec, L, R)
            assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want - D), (pattern, kind)


def test_hyper_contraction_reference_known_answer(talsh):
    """test.cpp:377-430 (test_talsh_hyper): C4 D(i,j,k)+=L(k,a,i,b)*R(b,k,a,j) with
    constant L = (0.001,-0.0001), R = (0.002,-0.0002), alpha 0.5; the 1-norm of D is
    |l r| * 48*24 * vol(D) * 0.5."""
    l, r = np.complex64(0.001 - 0.0001j), np.complex64(0.002 - 0.0002j)
    D = fort(np.zeros((48, 24, 32), dtype=np.complex64))
    L = fort(np.full((32, 48, 48, 24), l, dtype=np.complex64))
    R = fort(np.full((24, 32, 48, 24), r, dtype=np.complex64))
    assert gpu_contract("D(i,j,k)+=L(k,a,i,b)*R(b,k,a,j)", D, L, R, 0.5, 0.0) == 0
    want = abs(48.0 * 24.0) * abs(complex(l) * complex(r)) * (48.0 * 24.0 * 32.0) * 0.5
    assert abs(np.abs(D).sum() - want) <= 1e-5 * want
