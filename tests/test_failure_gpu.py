"""Failure detection on the GPU without a fault: the split-precision GEMM's
bounded waits.

With the test hook tcTestSplitStall(1) the GEMM's copy warp issues nothing, so
the MMA warp's first wait on a full stage runs out after 4096 polls.  Each CTA
then marks itself aborted (counted in the device error counter that
gpu_get_error_count reads, as the reference's gpu_error_count is,
tensor_algebra_gpu_nvidia.cu:189, :2315), lets the other warps finish their
bounded waits, frees its tensor memory and returns.  The tests check that the
launch ends on its own, that the counter rose, that a talshTensorContract task
in split precision reports TALSH_TASK_ERROR, and that the context stays usable:
the same contraction run afterwards is correct."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, host_tensor, rel_err

pytestmark = pytest.mark.gpu

PAT = "D(a,b)+=L(a,k)*R(k,b)"
DD, LD, RD = [100, 90], [100, 64], [64, 90]


def _operands(seed=0):
    rng = np.random.default_rng(seed)
    return fort(rng.standard_normal(LD)), fort(rng.standard_normal(RD)), fort(np.zeros(DD))


def _split_call(torch, Lh, Rh, D0):
    L = T.lib()
    e, dig, dr, lr, rr, _ = T.parse_pattern(PAT)
    args = (T.R8, T.ivec(dig), dr, T.ivec(DD), lr, T.ivec(LD), rr, T.ivec(RD))
    need = L.tcTensorContractSplitScratch(*args, 6)
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    d, l, r = dev(D0), dev(Lh), dev(Rh)
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    rc = L.tcTensorContractSplit(*args, d.data_ptr(), l.data_ptr(), r.data_ptr(), 1.0, 0.0, 0, 0, 6,
                                 scratch.data_ptr(), need, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()  # returns: every wait in the kernel is bounded
    return d.cpu().numpy().reshape(DD, order="F")


def test_bounded_wait_runs_out_and_context_survives(talsh):
    torch = pytest.importorskip("torch")
    L = T.lib()
    Lh, Rh, D0 = _operands()
    n0 = L.gpu_get_error_count()
    assert n0 >= 0
    assert L.tcTestSplitStall(1) == 0
    try:
        _split_call(torch, Lh, Rh, D0)
    finally:
        assert L.tcTestSplitStall(0) == 0
    n1 = L.gpu_get_error_count()
    assert n1 > n0, (n0, n1)
    # the context is intact: the same contraction without the hook is right
    got = _split_call(torch, Lh, Rh, D0)
    ref = D0.copy(order="F")
    e, dig, *_ = O.str2dig(PAT)
    O.contract_ttgt_blas(ref, Lh, Rh, dig)
    assert rel_err(got, ref) <= 1e-10
    assert L.gpu_get_error_count() == n1


def test_task_reports_error_then_recovers(talsh):
    L = T.lib()
    Lh, Rh, D0 = _operands(1)
    Dh = D0.copy(order="F")
    d, l, r = host_tensor(Dh), host_tensor(Lh), host_tensor(Rh)
    assert L.talshContractSlicesSet(6) == 0
    try:
        assert L.tcTestSplitStall(1) == 0
        task = T.Task()
        assert L.talshTaskClean(C.byref(task)) == 0
        rc = L.talshTensorContract(PAT.encode(), d.ref, l.ref, r.ref, 1.0, 0.0, 0, T.DEV_NVIDIA_GPU, T.COPY_TTT,
                                   T.NOPE, C.byref(task))
        assert rc == 0, rc
        st = C.c_int(0)
        L.talshTaskWait(C.byref(task), C.byref(st))
        assert st.value == T.TALSH_TASK_ERROR, st.value
        L.talshTaskDestruct(C.byref(task))
        assert L.tcTestSplitStall(0) == 0
        # the next task on the same tensors completes and is right
        rc = L.talshTensorContract(PAT.encode(), d.ref, l.ref, r.ref, 1.0, 0.0, 0, T.DEV_NVIDIA_GPU, T.COPY_TTT,
                                   T.NOPE, None)
        assert rc == 0, rc
    finally:
        L.tcTestSplitStall(0)
        L.talshContractSlicesSet(0)
    ref = np.zeros(DD, order="F")
    e, dig, *_ = O.str2dig(PAT)
    O.contract_ttgt_blas(ref, Lh, Rh, dig)
    assert rel_err(Dh, ref) <= 1e-10
    for t in (d, l, r):
        t.destruct()
