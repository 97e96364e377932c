"""tcTensorContractNoAlloc: the contraction entry point for callers that cannot
allocate device memory (code inside an allocator or memory-pool callback, a
process whose device budget belongs to another runtime, a loop that may not
take cudaMalloc's implicit synchronisation).  It runs the tcTensorContract
kernels with their scratch in one fixed array inside the library, so its
results must match tcTensorContract given caller scratch.

The device buffers below are the caller's inputs and outputs (allocated here
by torch, as any caller would); the entry point itself allocates nothing.
This file is collected last on purpose."""
import ctypes as C
import re

import numpy as np
import pytest

import tal_sh_b200 as T
from gpu_util import rand, rel_err

pytestmark = pytest.mark.gpu

TOL = {T.R8: 1e-12, T.C8: 1e-12, T.R4: 2e-5, T.C4: 2e-5}

# (kind, pattern, extents, alpha, accumulative): a gather-GEMM on the FP64
# tensor-core path, a full contraction (partial sums in the scratch too), and
# SIMT paths with conjugation.
CASES = [
    (T.R8, "D(a,b,c)+=L(a,k,c)*R(k,b)", dict(a=48, b=40, c=20, k=36), (0.75, 0.0), True),
    (T.C8, "D()+=L+(a,b)*R(b,a)", dict(a=300, b=200), (1.0, 0.5), False),
    (T.R4, "D(a,b)+=L(k,a)*R(b,k)", dict(a=130, b=70, k=50), (1.0, 0.0), True),
    (T.C4, "D(b,a)+=L(a,k,j)*R+(j,k,b)", dict(a=33, b=29, j=7, k=11), (0.5, -0.25), True),
    (T.R8, "D(i,j)+=L(i,k)*R(k,j)", dict(i=320, j=288, k=96), (1.0, 0.0), False),
]


def _labels(pattern):
    m = re.fullmatch(r"D\+?\(([a-z,]*)\)\+?=L\+?\(([a-z,]*)\)\*R\+?\(([a-z,]*)\)", pattern)
    return [[x for x in g.split(",") if x] for g in m.groups()]


class _Case:
    def __init__(self, torch, kind, pattern, ext, seed):
        e, self.dig, self.dr, self.lr, self.rr, self.conj = T.parse_pattern(pattern)
        assert e == 0, (pattern, e)
        dl, ll, rl = _labels(pattern)
        self.ddims, self.ldims, self.rdims = ([ext[x] for x in g] for g in (dl, ll, rl))
        rng = np.random.default_rng(seed)
        to_dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
        self.d0 = to_dev(rand(self.ddims, kind, rng))
        self.l = to_dev(rand(self.ldims, kind, rng))
        self.r = to_dev(rand(self.rdims, kind, rng))
        self.kind = kind

    def shape_args(self):
        return (self.kind, T.ivec(self.dig), self.dr, T.ivec(self.ddims), self.lr, T.ivec(self.ldims),
                self.rr, T.ivec(self.rdims))


def _stream(torch):
    return torch.cuda.current_stream().cuda_stream


def _with_scratch(L, torch, c, alpha, acc):
    d = c.d0.clone()
    need = L.tcTensorContractScratch(*c.shape_args())
    scratch = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda")
    rc = L.tcTensorContract(*c.shape_args(), d.data_ptr(), c.l.data_ptr(), c.r.data_ptr(), alpha[0], alpha[1],
                            c.conj, 1 if acc else 0, scratch.data_ptr(), need, _stream(torch))
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()
    return d.cpu().numpy()


def _no_alloc(L, torch, c, alpha, acc):
    d = c.d0.clone()
    rc = L.tcTensorContractNoAlloc(*c.shape_args(), d.data_ptr(), c.l.data_ptr(), c.r.data_ptr(), alpha[0],
                                   alpha[1], c.conj, 1 if acc else 0, _stream(torch))
    assert rc == 0, (rc, L.tcLastErrorString())
    torch.cuda.synchronize()
    return d.cpu().numpy()


def test_no_alloc_matches_caller_scratch(built):
    """Two calls in a row per case, and every case after another one, so each
    call finds the previous call's contents in the shared array."""
    torch = pytest.importorskip("torch")
    L = T.lib()
    assert L.tcTensorContractNoAllocMaxScratch() == 8 << 20
    for n, (kind, pattern, ext, alpha, acc) in enumerate(CASES):
        c = _Case(torch, kind, pattern, ext, seed=100 + n)
        assert 0 < L.tcTensorContractScratch(*c.shape_args()) <= 8 << 20
        want = _with_scratch(L, torch, c, alpha, acc)
        before = L.tcKernelLaunchCount()
        first = _no_alloc(L, torch, c, alpha, acc)
        assert L.tcKernelLaunchCount() > before
        second = _no_alloc(L, torch, c, alpha, acc)
        for got in (first, second):
            err = rel_err(got, want)
            assert err <= TOL[kind], (pattern, kind, err)


def test_no_alloc_rejects_oversized_shapes(built):
    """A shape whose offset tables exceed the fixed array is refused before any launch."""
    L = T.lib()
    ext = 200000  # tables of 16 bytes per index value: 9.6 MB > 8 MiB
    args = (T.R8, T.ivec([1, -1, -2, 2]), 2, T.ivec([ext, ext]), 2, T.ivec([ext, ext]), 2, T.ivec([ext, ext]))
    assert L.tcTensorContractScratch(*args) > L.tcTensorContractNoAllocMaxScratch()
    before = L.tcKernelLaunchCount()
    rc = L.tcTensorContractNoAlloc(*args, None, None, None, 1.0, 0.0, 0, 1, None)
    assert rc == T.TALSH_LIMIT_EXCEEDED
    assert L.tcKernelLaunchCount() == before
    assert b"tcTensorContractNoAlloc" in L.tcLastErrorString()
    assert L.tcTensorContractNoAlloc(99, T.ivec([1, -1, -2, 2]), 2, T.ivec([4, 4]), 2, T.ivec([4, 4]), 2,
                                     T.ivec([4, 4]), None, None, None, 1.0, 0.0, 0, 1, None) == T.TALSH_INVALID_ARGS
