"""Batched transposes (tcPermuteBatch*): small tasks in one persistent launch
over device-side descriptors, larger ones with their tiled plan, all replayed
from one CUDA graph; every task of a batch of uneven ranks, extents and kinds
equals the oracle bit for bit after each replay."""
import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, rand

pytestmark = pytest.mark.gpu


def _task(rng):
    kind = [T.R4, T.R8, T.C4, T.C8][int(rng.integers(0, 4))]
    r = int(rng.integers(1, 6))
    top = max(2, int(round((1 << 16) ** (1.0 / r))))
    dims = [int(rng.integers(1, top + 1)) for _ in range(r)]
    o2n = [int(x) + 1 for x in rng.permutation(r)]
    add = bool(rng.integers(0, 2))
    conj = bool(rng.integers(0, 2)) and kind in (T.C4, T.C8)
    alpha = (float(rng.choice([1.0, 0.5, -1.25])), float(rng.choice([0.0, 0.75])))
    return kind, dims, o2n, add, conj, alpha


# Two tasks above the persistent launch's size limit (2^18 elements), which
# keep their tiled plan in a branch of the same graph.
LARGE = [(T.R8, [65, 3, 1500], [3, 1, 2], True, False, (0.5, 0.0)),
         (T.C4, [700, 2, 300], [2, 3, 1], False, True, (1.0, 0.0))]


@pytest.mark.parametrize("with_large", [False, True])
def test_batched_transposes_bit_exact(talsh, with_large):
    torch = pytest.importorskip("torch")
    lib = T.lib()
    rng = np.random.default_rng(77)
    n = 40 + (len(LARGE) if with_large else 0)
    arr = (T.PermuteTask * n)()
    keep = []
    for t, x in zip(arr, range(n)):
        kind, dims, o2n, add, conj, alpha = LARGE[x - 40] if x >= 40 else _task(rng)
        src = rand(dims, kind, rng)
        d0 = rand(O.out_dims(dims, o2n), kind, rng)
        s = torch.from_numpy(src.ravel(order="F").copy()).cuda()
        d = torch.from_numpy(d0.ravel(order="F").copy()).cuda()
        keep.append((kind, dims, o2n, add, conj, alpha, src, d0, s, d))
        t.data_kind, t.rank = kind, len(dims)
        for i, v in enumerate(dims):
            t.dims[i] = v
        for i, v in enumerate(o2n):
            t.o2n[i] = v
        t.src, t.dst = s.data_ptr(), d.data_ptr()
        t.add, t.alpha_re, t.alpha_im, t.conj = int(add), alpha[0], alpha[1], int(conj)
    h = C_void()
    assert lib.tcPermuteBatchCreate(n, arr, 8, C_ref(h)) == 0
    stream = torch.cuda.current_stream().cuda_stream
    try:
        for rep in (1, 2):
            assert lib.tcPermuteBatchLaunch(h, stream) == 0
            torch.cuda.synchronize()
            for kind, dims, o2n, add, conj, alpha, src, d0, s, d in keep:
                if add:
                    want = d0.copy(order="F")
                    for _ in range(rep):
                        O.tensor_add(want, src, o2n, alpha[0], alpha[1], 2 if conj else 0)
                else:
                    want = O.permute(src, o2n, conj=conj)
                got = d.cpu().numpy().reshape(want.shape, order="F")
                assert got.tobytes() == want.tobytes(), (kind, dims, o2n, add, conj, rep)
    finally:
        assert lib.tcPermuteBatchDestroy(h) == 0


def test_batched_transposes_reject_bad_task(talsh):
    lib = T.lib()
    arr = (T.PermuteTask * 1)()
    arr[0].data_kind, arr[0].rank = T.R8, 2
    arr[0].dims[0], arr[0].dims[1] = 4, 4
    arr[0].o2n[0], arr[0].o2n[1] = 1, 1  # not a permutation
    arr[0].src, arr[0].dst = 256, 512
    h = C_void()
    assert lib.tcPermuteBatchCreate(1, arr, 1, C_ref(h)) == T.TALSH_INVALID_ARGS
    assert lib.tcPermuteBatchCreate(0, arr, 1, C_ref(h)) == T.TALSH_INVALID_ARGS


def C_void():
    import ctypes
    return ctypes.c_void_p()


def C_ref(x):
    import ctypes
    return ctypes.byref(x)
