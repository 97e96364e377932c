"""The oracle (CPU restatement of the reference) pinned against the reference's
stated digital patterns and matricizations, the known answers of its own tests,
and numpy's independent transpose / einsum."""
import itertools
import json
import os
import re

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _lib(built):
    O.lib()


def gold(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def einsum_ref(pattern, D0, L, R, alpha, conj_bits):
    toks = re.findall(r"\(([^)]*)\)", pattern)
    sD, sL, sR = [[x.rstrip("+") for x in t.replace("|", ",").split(",") if x] for t in toks]
    labels = sorted(set(sD + sL + sR))
    m = {x: "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ"[i] for i, x in enumerate(labels)}
    cplx = np.iscomplexobj(L)
    cl = ((conj_bits >> 1) ^ conj_bits) & 1 if cplx else 0
    cr = ((conj_bits >> 2) ^ conj_bits) & 1 if cplx else 0
    Lc = np.conj(L) if cl else L
    Rc = np.conj(R) if cr else R
    spec = "".join(m[x] for x in sL) + "," + "".join(m[x] for x in sR) + "->" + "".join(m[x] for x in sD)
    return D0 + alpha * np.einsum(spec, Lc.astype(np.complex128 if cplx else np.float64),
                                  Rc.astype(np.complex128 if cplx else np.float64))


def test_stated_digital_patterns():
    g = gold("patterns.json")
    for key in ("nvtal_digital", "c1", "c1_transpose"):
        e, dig, dr, lr, rr, cj = O.str2dig(g[key]["pattern"])
        assert e == 0 and dig == g[key]["digital"], key


def test_stated_c1_matricizations():
    g = gold("patterns.json")["c1"]
    e, d, l, r, ncd, nlu, nru, nhu = O.permutations(g["digital"], 4, 4, variant="cpu")
    c = g["cpu"]
    assert e == 0 and (d, l, r, ncd, nlu, nru, nhu) == (c["dprm"], c["lprm"], c["rprm"], c["ncd"], c["nlu"], c["nru"], c["nhu"])
    e, d, l, r, ncd, nlu, nru, _ = O.permutations(g["digital"], 4, 4, variant="gpu")
    c = g["gpu"]
    assert e == 0 and (d, l, r, ncd, nlu, nru) == (c["dprm"], c["lprm"], c["rprm"], c["ncd"], c["nlu"], c["nru"])


def test_reference_benchmark_patterns_parse():
    for case in gold("tensor_contractions.json"):
        e, dig, dr, lr, rr, cj = O.str2dig(case["pattern"])
        assert e == 0, case
        assert (dr, lr, rr) == (len(case["D"]), len(case["L"]), len(case["R"]))
        for i, v in enumerate(dig[:lr]):  # extents agree with the pattern
            if v > 0:
                assert case["L"][i] == case["D"][v - 1]
            else:
                assert case["L"][i] == case["R"][-v - 1]


@pytest.mark.parametrize("pattern,code", [
    ("D(a,a)+=L(a)*R(a)", 10), ("D(a)+=L(a,b)", 11), ("D(a,,b)+=L(a,b)", 2),
    ("D(a,b)+=L(a,c)*R(c,b)*S(d)", 1), ("D(a,b,c)+=L(a,c,c)*R(b)", 8), ("", 15), ("*", -2),
    ("D(a|b+,)=L(a,b)", 3), ("D(a#,b)=L(a#,b)", 2)])
def test_malformed_patterns(pattern, code):
    assert O.str2dig(pattern)[0] == code


@pytest.mark.parametrize("dims", [(3, 4, 5), (17, 31, 2), (2, 3, 4, 5), (5, 1, 7, 3), (97, 2)])
def test_permute_matches_numpy(dims):
    rng = np.random.default_rng(1)
    a = np.asfortranarray(rng.standard_normal(dims))
    for o2n in itertools.permutations(range(1, len(dims) + 1)):
        n2o = [o2n.index(k + 1) for k in range(len(dims))]
        ref = np.transpose(a, n2o)
        assert np.array_equal(O.permute(a, list(o2n)), ref)
        assert np.array_equal(O.permute(a, list(o2n), blocked=True, nthreads=4), ref)


def test_permute_conj_and_signed_zero():
    a = np.asfortranarray(np.array([[1 + 2j, -0.0 + 0.0j], [np.nan + 1j, 3 - 0.0j]], dtype=np.complex128))
    out = O.permute(a, [2, 1], conj=True)
    exp = np.ascontiguousarray(np.transpose(a))
    exp.imag = -exp.imag  # a sign flip, bit for bit (also on zeros and NaN payloads)
    assert np.ascontiguousarray(out).tobytes() == exp.tobytes()


def test_blocked_transpose_large_bit_identical():
    rng = np.random.default_rng(2)
    a = np.asfortranarray(rng.standard_normal((97, 31, 17, 5)).astype(np.float32))
    for o2n in [(4, 3, 2, 1), (2, 1, 4, 3), (3, 1, 4, 2), (1, 3, 2, 4)]:
        assert np.array_equal(O.permute(a, list(o2n), blocked=True, nthreads=8), O.permute(a, list(o2n)))


def test_add_rules():
    # real kinds scale by cmplx8_to_real8(alpha): modulus with the sign of Re(alpha)
    assert O.cmplx8_to_real8(3.0, 4.0) == 5.0
    assert O.cmplx8_to_real8(-3.0, 4.0) == -5.0
    assert O.cmplx8_to_real8(0.0, -2.0) == -2.0
    rng = np.random.default_rng(3)
    l = np.asfortranarray(rng.standard_normal((3, 4, 5)))
    d0 = np.asfortranarray(rng.standard_normal((5, 3, 4)))
    d = d0.copy(order="F")
    O.tensor_add(d, l, [2, 3, 1], 0.5, 0.0)
    assert np.array_equal(d, d0 + np.transpose(l, (2, 0, 1)) * 0.5)


CONTRACTIONS = [
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", (6, 7, 5, 4), (6, 3, 8, 5), (8, 7, 3, 4)),
    ("D()+=L(a,b)*R(b,a)", (), (4, 5), (5, 4)),
    ("D(a,b)+=L(a)*R(b)", (4, 5), (4,), (5,)),
    ("D(a,b,c)+=L(c,a)*R(b,c)", (3, 4, 5), (5, 3), (4, 5)),
    ("D(b,a)+=L(a,b)*R()", (4, 3), (3, 4), ()),
    ("D(b,a)+=L()*R(a,b)", (4, 3), (), (3, 4)),
    ("D()+=L()*R()", (), (), ()),
    ("D(i,j,k)+=L(k,a,i,b)*R(b,k,a,j)", (3, 4, 5), (5, 2, 3, 6), (6, 5, 2, 4)),
    ("D(a,b,c,d)+=L(d,c,i,j)*R(b,a,i,j)", (3, 4, 5, 6), (6, 5, 2, 3), (4, 3, 2, 3)),
]


@pytest.mark.parametrize("kind", [O.R8, O.C8])
@pytest.mark.parametrize("case", CONTRACTIONS, ids=[c[0] for c in CONTRACTIONS])
def test_contract_matches_einsum(case, kind):
    pat, dd, ld, rd = case
    rng = np.random.default_rng(4)
    e, dig, _, _, _, cj = O.str2dig(pat)
    assert e == 0

    def rnd(shape):
        x = rng.standard_normal(shape)
        if kind == O.C8:
            x = x + 1j * rng.standard_normal(shape)
        return O._fort(np.asarray(x, dtype=O.NP_DTYPE[kind]))

    L, R, D0 = rnd(ld), rnd(rd), rnd(dd)
    for conj in ([0, 2, 4, 1] if kind == O.C8 else [0]):
        D = D0.copy(order="F")
        assert O.tensor_contract(D, L, R, dig, -1.25, 0.0, conj, True) == 0
        ref = einsum_ref(pat, D0, L, R, -1.25, conj)
        assert np.linalg.norm(D - ref) <= 1e-13 * max(1.0, np.linalg.norm(ref))


def test_known_answer_talsh_c():
    # test.cpp:38-165: D(a,b,i,j)+=L(c,b,d,a)*R(j,d,i,c), L=0.001, R=0.01, alpha=2:
    # every element is 2*V*V*1e-5 and the 1-norm is gflops*1e-5*1e9 (scaled-down V, O).
    V, Odim = 8, 4
    e, dig, _, _, _, _ = O.str2dig(gold("patterns.json")["talsh_c_pattern"])
    D = np.zeros((V, V, Odim, Odim), order="F")
    L = np.full((V, V, V, V), 0.001, order="F")
    R = np.full((Odim, V, Odim, V), 0.01, order="F")
    assert O.tensor_contract(D, L, R, dig, 2.0, 0.0, 0, True) == 0
    flops = np.sqrt(D.size * L.size * R.size) * 2.0
    assert np.allclose(D, 2.0 * V * V * 1e-5, rtol=1e-14)
    assert abs(O.norm1(D) - flops * 0.01 * 0.001) <= 1e-12 * flops * 1e-5


def test_known_answer_nwchem_residual():
    # test.cpp:895-1013: two contractions (alpha -2 then +1) plus the explicit loop give 0.
    rng = np.random.default_rng(5)
    Vd, Od = 5, 2
    e, dig, _, _, _, _ = O.str2dig(gold("patterns.json")["nwchem_pattern"])
    D = np.zeros((Od, Vd), order="F")
    L = np.asfortranarray(1e6 / (rng.integers(0, 2 ** 31, (Vd, Od)) + 1.0))
    R = np.asfortranarray(1e5 / (rng.integers(0, 2 ** 31, (Od, Od, Vd, Vd)) + 1.0))
    assert O.tensor_contract(D, L, R, dig, -2.0, 0.0, 0, True) == 0
    assert O.tensor_contract(D, L, R, dig, 1.0, 0.0, 0, True) == 0
    for ib in range(Vd):
        for ia in range(Od):
            for idd in range(Od):
                for ic in range(Vd):
                    D[ia, ib] += L[ic, idd] * R[idd, ia, ib, ic]
    assert O.norm1(D) <= 1e-12 * O.norm1(np.abs(L)) * O.norm1(np.abs(R))


def test_accumulative_false_overwrites():
    rng = np.random.default_rng(6)
    e, dig, _, _, _, _ = O.str2dig("D(a,b)+=L(a,c)*R(c,b)")
    L = np.asfortranarray(rng.standard_normal((3, 4)))
    R = np.asfortranarray(rng.standard_normal((4, 5)))
    D = np.asfortranarray(np.full((3, 5), np.nan))
    assert O.tensor_contract(D, L, R, dig, 1.0, 0.0, 0, False) == 0
    assert np.allclose(D, L @ R, rtol=1e-14)


def test_generator_is_deterministic():
    a = O.uniform((5, 7), O.R8, 0)
    b = O.uniform((5, 7), O.R8, 0)
    assert np.array_equal(a, b) and a.min() >= -1 and a.max() <= 1 and a.std() > 0.3


def test_slice_insert_match_numpy():
    """tensor_block_slice / tensor_block_insert restated: sub-block reads and writes
    equal numpy slicing (accumulating and overwriting), every kind, ranks 1-6."""
    rng = np.random.default_rng(0)
    for _ in range(60):
        r = int(rng.integers(1, 7))
        full = [int(rng.integers(1, 9)) for _ in range(r)]
        sl = [int(rng.integers(1, f + 1)) for f in full]
        off = [int(rng.integers(0, f - s + 1)) for f, s in zip(full, sl)]
        idx = tuple(slice(o, o + s) for o, s in zip(off, sl))
        for dt in (np.float32, np.float64, np.complex64, np.complex128):
            F = np.asfortranarray((rng.uniform(-1, 1, full) + 1j * rng.uniform(-1, 1, full)).astype(dt)
                                  if np.dtype(dt).kind == "c" else rng.uniform(-1, 1, full).astype(dt))
            S0 = np.asfortranarray(rng.uniform(-1, 1, sl).astype(dt))
            S = S0.copy(order="F")
            assert O.tensor_slice(S, F, off, False) == 0 and np.array_equal(S, F[idx])
            S = S0.copy(order="F")
            assert O.tensor_slice(S, F, off, True) == 0 and np.array_equal(S, S0 + F[idx])
            G, W = F.copy(order="F"), F.copy()
            W[idx] = S0
            assert O.tensor_insert(G, S0, off, False) == 0 and np.array_equal(G, W)
            G, W = F.copy(order="F"), F.copy()
            W[idx] += S0
            assert O.tensor_insert(G, S0, off, True) == 0 and np.array_equal(G, W)
    bad = np.asfortranarray(np.zeros((3, 3)))
    assert O.tensor_slice(bad, np.zeros((4, 4), order="F"), [2, 0], False) != 0  # 2 + 3 > 4


def test_split_precision_model_error_bound():
    """The split-precision arithmetic, modelled in numpy: the digits reconstruct
    each scaled entry to 2^-42 (6 slices), and the product error against float64
    stays below the 1e-10 bound stated for 6 slices, above it for 5."""
    from oracle.ozaki import slice_rows, split_gemm
    rng = np.random.default_rng(3)
    A = rng.standard_normal((64, 768))
    Bt = rng.standard_normal((48, 768))
    e, d = slice_rows(A, 6)
    rec = sum(np.ldexp(d[s].astype(np.float64), -7 * (s + 1)) for s in range(6))
    assert np.abs(np.ldexp(A, -e[:, None]) - rec).max() < 2.0 ** -42
    assert all(np.abs(x).max() <= 127 for x in d)
    ref = A @ Bt.T
    err = lambda S: np.linalg.norm(split_gemm(A, Bt, S) - ref) / np.linalg.norm(ref)
    assert err(6) < 1e-10
    assert err(5) > 1e-10
    assert err(3) > err(4) > err(5) > err(6)


def test_split_precision_model_complex_form():
    """The complex form's error, modelled: a complex product rewritten as the real
    product [Lr Li] x [[Yr Zr], [Yi Zi]] (Y = conj(R), Z = i conj(R)) and run through
    the slice model stays under 1e-10 with 6 slices at the complex test shapes."""
    from oracle.ozaki import split_gemm
    rng = np.random.default_rng(4)
    for M, N, K in ((130, 70, 200), (256, 256, 256), (77, 33, 95)):
        A = rng.standard_normal((M, K)) + 1j * rng.standard_normal((M, K))
        B = rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))
        Ar = np.stack([A.real, A.imag], axis=-1).reshape(M, 2 * K)        # k' = (k, c), c fastest
        Y, Z = np.conj(B).T, (1j * np.conj(B)).T                            # N x K each
        Bt = np.concatenate([np.stack([Y.real, Y.imag], axis=-1).reshape(N, 2 * K),
                             np.stack([Z.real, Z.imag], axis=-1).reshape(N, 2 * K)])
        C = split_gemm(Ar, Bt, 6)
        got = C[:, :N] + 1j * C[:, N:]
        ref = A @ B
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-10
