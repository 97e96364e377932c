"""Coupled-cluster-shaped contractions at v=96, o=32 against the oracle.

The two patterns of the coupled-cluster workload, at half its extents (v=96
virtual, o=32 occupied) so that the oracle finishes in about a second:
  C3a  D(a,b,i,j) += L(a,b,c,d) * R(c,d,i,j)   (a,b,c,d in v; i,j in o)
  C3b  D(a,b,i,j) += L(a,k,c,i) * R(c,b,k,j)   (a,b,c in v; i,j,k in o)
with normal(0,1) values scaled by 1/sqrt(contracted volume), D nonzero and
accumulated into.  The oracle is the reference's CPU contraction as it runs with
a BLAS library (tensor_block_contract, tensor_algebra_cpu.F90:3675-4358: the CPU
matricization, blocked transposes, one DGEMM('T','N'), the back-transpose).
Plain FP64 through talshTensorContract: relative Frobenius error <= 1e-12;
split precision (6 int8 slices, tcTensorContractSplit): <= 1e-10.  The error is
taken relative to the contraction term (D's old value excluded)."""
import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort

pytestmark = pytest.mark.gpu

V, OCC = 96, 32
CASES = {
    "C3a": ("D(a,b,i,j)+=L(a,b,c,d)*R(c,d,i,j)", (V, V, V, V), (V, V, OCC, OCC), (V, V, OCC, OCC), V * V),
    "C3b": ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", (V, OCC, V, OCC), (V, V, OCC, OCC), (V, V, OCC, OCC), V * OCC),
}
TOL_PLAIN, TOL_SPLIT6 = 1e-12, 1e-10


def _operands(name):
    pat, ld, rd, dd, cvol = CASES[name]
    rng = np.random.default_rng(3 if name == "C3a" else 4)
    s = 1.0 / np.sqrt(cvol)
    Lh = fort(rng.standard_normal(ld) * s)
    Rh = fort(rng.standard_normal(rd) * s)
    D0 = fort(rng.standard_normal(dd))
    e, dig, dr, lr, rr, _ = T.parse_pattern(pat)
    assert e == 0
    ref = D0.copy(order="F")
    O.contract_ttgt_blas(ref, Lh, Rh, dig, 1.0, 0.0)
    return pat, dig, (dr, lr, rr), (dd, ld, rd), Lh, Rh, D0, ref


def _err(got, ref, D0):
    return np.linalg.norm((got - ref).ravel()) / np.linalg.norm((ref - D0).ravel())


@pytest.mark.parametrize("name", ["C3a", "C3b"])
def test_cc_plain_fp64(talsh, name):
    torch = pytest.importorskip("torch")
    pat, dig, (dr, lr, rr), (dd, ld, rd), Lh, Rh, D0, ref = _operands(name)
    L = T.lib()
    args = (T.R8, T.ivec(dig), dr, T.ivec(dd), lr, T.ivec(ld), rr, T.ivec(rd))
    need = L.tcTensorContractScratch(*args)
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    d, l, r = dev(D0), dev(Lh), dev(Rh)
    scratch = torch.empty(max(1, need), dtype=torch.uint8, device="cuda")
    rc = L.tcTensorContract(*args, d.data_ptr(), l.data_ptr(), r.data_ptr(), 1.0, 0.0, 0, 1,
                            scratch.data_ptr(), need, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()
    err = _err(d.cpu().numpy().reshape(dd, order="F"), ref, D0)
    assert err <= TOL_PLAIN, (name, err)


@pytest.mark.parametrize("name", ["C3a", "C3b"])
def test_cc_split_precision(talsh, name):
    torch = pytest.importorskip("torch")
    pat, dig, (dr, lr, rr), (dd, ld, rd), Lh, Rh, D0, ref = _operands(name)
    L = T.lib()
    args = (T.R8, T.ivec(dig), dr, T.ivec(dd), lr, T.ivec(ld), rr, T.ivec(rd))
    need = L.tcTensorContractSplitScratch(*args, 6)
    assert need > 0
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    d, l, r = dev(D0), dev(Lh), dev(Rh)
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    rc = L.tcTensorContractSplit(*args, d.data_ptr(), l.data_ptr(), r.data_ptr(), 1.0, 0.0, 0, 1, 6,
                                 scratch.data_ptr(), need, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()
    err = _err(d.cpu().numpy().reshape(dd, order="F"), ref, D0)
    assert err <= TOL_SPLIT6, (name, err)
