"""The BF16x3, TF32x3 and FP8 split forms of the tensor-core contraction
(tcTensorContractSplitForm: floating-point slices on tcgen05 kind::f16,
kind::tf32 and kind::f8f6f4, one fp32 accumulator per slice diagonal, FP64
recombination) against the FP64 oracle, and the numpy model of their arithmetic
(oracle/ozaki.py) on the CPU.

Stated bounds (relative Frobenius error of the contraction term, random normal
operands, contracted volumes up to 1600 here): three bf16 slices 5e-6, three
tf32 slices 1e-5 -- the fp32 sums dominate, and they grow with the number of
tensor-core K steps (16 bf16 or 8 tf32 elements each): measured 1e-6 and
2.4e-6 at K = 1024, up to 3.8e-6 for tf32 at K = 1600, 1.4e-5 to 8.6e-5 at the
coupled-cluster sizes (K = 12288 and 36864), several times the round-to-nearest
model of oracle/ozaki.py, which the CPU tests hold to its own quarter bounds;
three e4m3 slices 1e-4 and four 1e-5 -- the dropped pairs dominate, about
2^-12 and 2^-16 per product (3.5e-5 and 1.4e-6 in the model, 3.3e-5 to 3.6e-5
measured for three)."""
import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort
from oracle import ozaki as Z

BOUND = {("bf16", 3): 5e-6, ("tf32", 3): 1e-5, ("fp8", 3): 1e-4, ("fp8", 4): 1e-5, ("bf16", 2): 2e-5}
# the round-to-nearest model's own bounds at K = 1024
MODEL_BOUND = {("bf16", 3): 5e-7, ("tf32", 3): 5e-7, ("fp8", 3): 1e-4, ("fp8", 4): 5e-6, ("bf16", 2): 2e-5}
FORM = {"bf16": T.TC_SPLIT_BF16, "tf32": T.TC_SPLIT_TF32, "fp8": T.TC_SPLIT_FP8}


@pytest.mark.parametrize("form,S", sorted(BOUND))
def test_model_within_stated_bound(built, form, S):
    rng = np.random.default_rng(5)
    K = 1024
    A = rng.standard_normal((64, K)) / np.sqrt(K)
    B = rng.standard_normal((40, K)) / np.sqrt(K)
    ref = A @ B.T
    err = np.linalg.norm(Z.split_gemm_float(A, B, S, form) - ref) / np.linalg.norm(ref)
    assert err <= MODEL_BOUND[(form, S)], (form, S, err)


def test_model_slices_are_exact_decomposition(built):
    """The slices sum back to the row-scaled input up to the last residual."""
    rng = np.random.default_rng(6)
    X = rng.standard_normal((8, 100)) * np.exp2(rng.integers(-20, 20, size=(8, 100)))
    for form, b in Z.FORM_BITS.items():
        e, ys = Z.slice_rows_float(X, 6, form)
        back = sum(np.ldexp(y, -b * s) for s, y in enumerate(ys))
        rel = np.abs(np.ldexp(back, e[:, None]) - X) / np.abs(X).max(axis=1, keepdims=True)
        assert rel.max() < 2.0 ** (-6 * b + 1) * 4, (form, rel.max())


CASES = [
    ("D(a,b)+=L(a,k)*R(k,b)", dict(a=200, b=100, k=300)),
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=48, b=48, c=48, i=16, j=16, k=16)),
    ("D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", dict(a=40, b=40, c=40, d=40, i=12, j=12)),
]


def _run(torch, pattern, ext, form, S, kind=T.R8, alpha=1.0, acc=True, seed=0):
    import re
    m = re.fullmatch(r"D\(([a-z,]*)\)\+?=L\(([a-z,]*)\)\*R\(([a-z,]*)\)", pattern)
    dl, ll, rl = [[x for x in g.split(",") if x] for g in m.groups()]
    dd, ld, rd = ([ext[x] for x in g] for g in (dl, ll, rl))
    e, dig, dr, lr, rr, _ = T.parse_pattern(pattern)
    rng = np.random.default_rng(seed)
    cvol = np.sqrt(np.prod(ld) * np.prod(rd) / np.prod(dd))
    if kind == T.R8:
        Lh = fort(rng.standard_normal(ld) / np.sqrt(cvol))
        Rh = fort(rng.standard_normal(rd) / np.sqrt(cvol))
        D0 = fort(rng.standard_normal(dd))
    else:
        c = lambda d: rng.standard_normal(d) + 1j * rng.standard_normal(d)
        Lh, Rh, D0 = fort(c(ld) / np.sqrt(cvol)), fort(c(rd) / np.sqrt(cvol)), fort(c(dd))
    L = T.lib()
    args = (kind, T.ivec(dig), dr, T.ivec(dd), lr, T.ivec(ld), rr, T.ivec(rd))
    need = L.tcTensorContractSplitFormScratch(*args, FORM[form], S)
    assert need > 0
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    d, l, r = dev(D0), dev(Lh), dev(Rh)
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    rc = L.tcTensorContractSplitForm(*args, d.data_ptr(), l.data_ptr(), r.data_ptr(), alpha, 0.0, 0, 1 if acc else 0,
                                     FORM[form], S, scratch.data_ptr(), need, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()
    got = d.cpu().numpy().reshape(dd, order="F")
    ref = D0.copy(order="F")
    O.contract_ttgt_blas(ref, Lh, Rh, dig, alpha, 0.0, accumulative=acc)
    term = ref - (D0 if acc else 0)
    return np.linalg.norm((got - ref).ravel()) / np.linalg.norm(term.ravel())


@pytest.mark.gpu
@pytest.mark.parametrize("pattern,ext", CASES)
@pytest.mark.parametrize("form,S", [("bf16", 3), ("tf32", 3), ("fp8", 3), ("fp8", 4)])
def test_split_form_accuracy(talsh, pattern, ext, form, S):
    torch = pytest.importorskip("torch")
    err = _run(torch, pattern, ext, form, S)
    assert err <= BOUND[(form, S)], (pattern, form, S, err)


@pytest.mark.gpu
def test_split_form_overwrite_alpha_and_complex(talsh):
    torch = pytest.importorskip("torch")
    err = _run(torch, "D(a,b)+=L(a,k)*R(k,b)", dict(a=130, b=70, k=200), "bf16", 3, alpha=-0.75, acc=False)
    assert err <= BOUND[("bf16", 3)], err
    err = _run(torch, "D(a,b,i)+=L(a,k,i)*R(k,b)", dict(a=30, b=20, k=50, i=6), "tf32", 3, kind=T.C8, seed=3)
    assert err <= BOUND[("tf32", 3)], err


@pytest.mark.gpu
def test_split_form_invalid_arguments(talsh):
    L = T.lib()
    dig = T.ivec([1, -1, -2, 2])
    dims = T.ivec([4, 4])
    assert L.tcTensorContractSplitFormScratch(T.R8, dig, 2, dims, 2, dims, 2, dims, 7, 3) == 0
    assert L.tcTensorContractSplitFormScratch(T.R8, dig, 2, dims, 2, dims, 2, dims, T.TC_SPLIT_BF16, 1) == 0
    assert L.tcTensorContractSplitFormScratch(T.R8, dig, 2, dims, 2, dims, 2, dims, T.TC_SPLIT_BF16, 3) > 0
    assert L.tcTensorContractSplitScratch(T.R8, dig, 2, dims, 2, dims, 2, dims, 19) == 0
