"""Split-precision R8 and C8 contractions (tcTensorContractSplit: int8 slices on
the tensor cores, recombined in FP64; C8 rewritten as one real contraction)
against the FP64 oracle, through the C ABI."""
import ctypes as C
import re

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, rel_err

pytestmark = pytest.mark.gpu

TOL_SPLIT6 = 1e-10  # bound stated for the 6-slice form


def _labels(pattern):
    m = re.fullmatch(r"D\(([a-z,]*)\)\+?=L\(([a-z,]*)\)\*R\(([a-z,]*)\)", pattern)
    return [[x for x in g.split(",") if x] for g in m.groups()]


def _run(torch, pattern, ext, slices, alpha=1.0, acc=True, seed=0, scale_rows=False):
    e, dig, dr, lr, rr, _ = T.parse_pattern(pattern)
    assert e == 0
    dl, ll, rl = _labels(pattern)
    dd, ld, rd = ([ext[x] for x in g] for g in (dl, ll, rl))
    rng = np.random.default_rng(seed)
    Lh = fort(rng.standard_normal(ld))
    Rh = fort(rng.standard_normal(rd))
    if scale_rows:  # entries spanning many binades
        Lh = fort(Lh * np.exp2(rng.integers(-30, 30, size=ld)))
    D0 = fort(rng.standard_normal(dd))
    L = T.lib()
    args = (T.R8, T.ivec(dig), dr, T.ivec(dd), lr, T.ivec(ld), rr, T.ivec(rd))
    need = L.tcTensorContractSplitScratch(*args, slices)
    assert need > 0
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    d, l, r = dev(D0), dev(Lh), dev(Rh)
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    rc = L.tcTensorContractSplit(*args, d.data_ptr(), l.data_ptr(), r.data_ptr(), alpha, 0.0, 0, 1 if acc else 0,
                                 slices, scratch.data_ptr(), need, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()
    got = d.cpu().numpy().reshape(dd, order="F")
    ref = D0.copy(order="F")
    assert O.tensor_contract(ref, Lh, Rh, dig, alpha, 0.0, 0, acc) == 0
    # error relative to the contraction term (D0 excluded so accumulation cannot hide it)
    term = ref - (D0 if acc else 0)
    return np.linalg.norm((got - ref).ravel()) / np.linalg.norm(term.ravel())


CASES = [
    ("D(a,b)+=L(a,k)*R(k,b)", dict(a=200, b=100, k=300)),
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=32, b=32, c=32, i=32, j=32, k=32)),
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=48, b=48, c=48, i=16, j=16, k=16)),
    ("D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", dict(a=40, b=40, c=40, d=40, i=12, j=12)),
    ("D(i,a)+=L(k,a,j)*R(j,i,k)", dict(a=77, i=33, j=19, k=5)),
]


@pytest.mark.parametrize("pattern,ext", CASES)
def test_split_contraction_accuracy(talsh, pattern, ext):
    torch = pytest.importorskip("torch")
    err = _run(torch, pattern, ext, 6)
    assert err <= TOL_SPLIT6, (pattern, err)


def test_split_slices_trade_accuracy(talsh):
    """Fewer slices: larger error, still bounded by the dropped-term estimate."""
    torch = pytest.importorskip("torch")
    errs = [_run(torch, "D(a,b)+=L(a,k)*R(k,b)", dict(a=128, b=64, k=512), s) for s in (3, 4, 6)]
    assert errs[0] > errs[1] > errs[2]
    assert errs[0] < 1e-4 and errs[2] < TOL_SPLIT6


def test_split_overwrite_alpha_and_row_scales(talsh):
    torch = pytest.importorskip("torch")
    err = _run(torch, "D(a,b)+=L(a,k)*R(k,b)", dict(a=130, b=70, k=200), 6, alpha=-0.75, acc=False,
               scale_rows=True)
    assert err <= TOL_SPLIT6, err


def test_split_long_contraction_chunks(talsh):
    """K beyond the int32-exact bound is split into chunks that accumulate in D."""
    torch = pytest.importorskip("torch")
    err = _run(torch, "D(a,b)+=L(a,k)*R(k,b)", dict(a=64, b=64, k=30000), 6)
    assert err <= TOL_SPLIT6, err


def _run_complex(torch, pattern, ext, slices, alpha, conj, acc=True, seed=0):
    """Complex(8) through the split form (rewritten as one real contraction)
    against the oracle's complex contraction; error relative to the term."""
    e, dig, dr, lr, rr, _ = T.parse_pattern(pattern)
    assert e == 0
    dl, ll, rl = _labels(pattern)
    dd, ld, rd = ([ext[x] for x in g] for g in (dl, ll, rl))
    rng = np.random.default_rng(seed)
    cplx = lambda sh: fort(rng.standard_normal(sh) + 1j * rng.standard_normal(sh))
    Lh, Rh, D0 = cplx(ld), cplx(rd), cplx(dd)
    L = T.lib()
    args = (T.C8, T.ivec(dig), dr, T.ivec(dd), lr, T.ivec(ld), rr, T.ivec(rd))
    need = L.tcTensorContractSplitScratch(*args, slices)
    assert need > 0
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    d, l, r = dev(D0), dev(Lh), dev(Rh)
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    rc = L.tcTensorContractSplit(*args, d.data_ptr(), l.data_ptr(), r.data_ptr(), alpha[0], alpha[1], conj,
                                 1 if acc else 0, slices, scratch.data_ptr(), need,
                                 torch.cuda.current_stream().cuda_stream)
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()
    got = d.cpu().numpy().reshape(dd, order="F")
    ref = D0.copy(order="F")
    assert O.tensor_contract(ref, Lh, Rh, dig, alpha[0], alpha[1], conj, acc) == 0
    term = ref - (D0 if acc else 0)
    return np.linalg.norm((got - ref).ravel()) / np.linalg.norm(term.ravel())


COMPLEX_CASES = [
    ("D(a,b)+=L(a,k)*R(k,b)", dict(a=130, b=70, k=200)),
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=16, b=16, c=16, i=16, j=16, k=16)),
    ("D(i,a)+=L(k,a,j)*R(j,i,k)", dict(a=77, i=33, j=19, k=5)),
]


@pytest.mark.parametrize("conj", range(8))
def test_split_complex_conjugation_flags(talsh, conj):
    """Complex(8) split precision for every conjugation flag, complex alpha."""
    torch = pytest.importorskip("torch")
    pattern, ext = COMPLEX_CASES[0]
    err = _run_complex(torch, pattern, ext, 6, (0.75, -0.5), conj)
    assert err <= TOL_SPLIT6, (conj, err)


@pytest.mark.parametrize("pattern,ext", COMPLEX_CASES)
def test_split_complex_accuracy(talsh, pattern, ext):
    torch = pytest.importorskip("torch")
    err = _run_complex(torch, pattern, ext, 6, (1.0, 0.0), 0)
    assert err <= TOL_SPLIT6, (pattern, err)
    err = _run_complex(torch, pattern, ext, 6, (-0.5, 0.25), 6, acc=False, seed=1)
    assert err <= TOL_SPLIT6, (pattern, err)


def test_split_rejects_other_forms(talsh):
    L = T.lib()
    e, dig, dr, lr, rr, _ = T.parse_pattern("D(a,b)+=L(a,k)*R(k,b)")
    args = (T.ivec(dig), dr, T.ivec([4, 4]), lr, T.ivec([4, 4]), rr, T.ivec([4, 4]))
    assert L.tcTensorContractSplitScratch(T.C4, *args, 6) == 0
    assert L.tcTensorContractSplit(T.C4, *args, None, None, None, 1.0, 0.0, 0, 1, 6, None, 0, None) == \
        T.TALSH_NOT_IMPLEMENTED
    assert L.tcTensorContractSplit(T.R8, *args, None, None, None, 1.0, 0.0, 0, 1, 9, None, 0, None) == \
        T.TALSH_INVALID_ARGS


def test_split_through_talsh_contract(talsh):
    """talshContractSlicesSet routes R8 talshTensorContract through the split form."""
    from gpu_util import gpu_contract
    L = talsh
    assert L.talshContractSlicesGet() == 0  # the drop-in default is plain FP64
    assert L.talshContractSlicesSet(9) == T.TALSH_INVALID_ARGS
    rng = np.random.default_rng(11)
    A, B = fort(rng.standard_normal((40, 30, 20))), fort(rng.standard_normal((20, 30, 50)))
    D0 = fort(rng.standard_normal((40, 50)))
    ref = D0.copy(order="F")
    assert O.tensor_contract(ref, A, B, [1, -2, -1, -3, -2, 2], 0.5, 0.0, 0, True) == 0
    assert L.talshContractSlicesSet(6) == 0
    try:
        D = D0.copy(order="F")
        assert gpu_contract("D(a,b)+=L(a,k,c)*R(c,k,b)", D, A, B, 0.5) == 0
    finally:
        assert L.talshContractSlicesSet(0) == 0
    assert rel_err(D - D0, ref - D0) <= TOL_SPLIT6


def test_split_single_loop_kernel():
    """The single-loop kernel (used when tensor maps cannot be encoded) gives the
    same accuracy; forced in a child process."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = r"""
import sys
sys.path.insert(0, %r); sys.path.insert(0, %r)
import torch
import test_split_gpu as t
for pat, ext in t.CASES[:3]:
    err = t._run(torch, pat, ext, 6)
    assert err <= t.TOL_SPLIT6, (pat, err)
print("OK")
""" % (root, os.path.join(root, "tests"))
    env = dict(os.environ, TALSH_B200_SPLIT_SIMPLE="1")
    p = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=600)
    assert p.returncode == 0 and "OK" in p.stdout, p.stdout


def test_split_complex_through_talsh_contract(talsh):
    """talshContractSlicesSet also routes C8 talshTensorContract (with
    conjugation flags) through the split form."""
    from gpu_util import gpu_contract
    L = talsh
    rng = np.random.default_rng(12)
    cplx = lambda sh: fort(rng.standard_normal(sh) + 1j * rng.standard_normal(sh))
    A, B, D0 = cplx((40, 30, 20)), cplx((20, 30, 50)), cplx((40, 50))
    ref = D0.copy(order="F")
    assert O.tensor_contract(ref, A, B, [1, -2, -1, -3, -2, 2], 0.5, -0.25, 4, True) == 0
    assert L.talshContractSlicesSet(6) == 0
    try:
        D = D0.copy(order="F")
        assert gpu_contract("D(a,b)+=L(a,k,c)*R+(c,k,b)", D, A, B, 0.5, -0.25) == 0
    finally:
        assert L.talshContractSlicesSet(0) == 0
    assert rel_err(D - D0, ref - D0) <= TOL_SPLIT6


def test_cta_pair_kernel_accuracy(talsh):
    """The CTA-pair kernel (TALSH_B200_SPLIT_PAIR=1: cta_group::2 MMAs of
    256 x 256 over a 2-CTA cluster), in a child process, meets the same bound
    on every case, real and complex."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = r"""
import sys
sys.path.insert(0, %r); sys.path.insert(0, %r)
import torch
import test_split_gpu as t
for pat, ext in t.CASES:
    print("ERR", t._run(torch, pat, ext, 6))
for pat, ext in t.COMPLEX_CASES:
    print("ERR", t._run_complex(torch, pat, ext, 6, (0.75, -0.5), 5))
print("ERR", t._run(torch, "D(a,b)+=L(a,k)*R(k,b)", dict(a=130, b=70, k=200), 6, alpha=-0.75, acc=False,
                    scale_rows=True))
""" % (root, os.path.join(root, "tests"))
    env = dict(os.environ, TALSH_B200_SPLIT_PAIR="1")
    p = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stdout
    errs = [float(line.split()[1]) for line in p.stdout.splitlines() if line.startswith("ERR ")]
    assert len(errs) == len(CASES) + len(COMPLEX_CASES) + 1, p.stdout
    assert max(errs) <= TOL_SPLIT6, errs
