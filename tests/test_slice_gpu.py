"""Tensor slicing and insertion on the GPU (tcTensorSlice / tcTensorInsert and
talshTensorSlice / talshTensorInsert) against the oracle's restatement of
tensor_block_slice / tensor_block_insert: bit-exact, every kind."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, host_tensor, rand

pytestmark = pytest.mark.gpu

KINDS = [T.R4, T.R8, T.C4, T.C8]


def _case(rng, r, long_run=False):
    """Full extents with a volume of at most about 2^20 elements."""
    top = max(2, int(round((1 << 20) ** (1.0 / r))))
    full = [int(rng.integers(1, top + 1)) for _ in range(r)]
    if long_run:
        full[0] = 300
        for i in range(1, r):
            full[i] = min(full[i], max(1, int(((1 << 20) / 300) ** (1.0 / max(r - 1, 1)))))
    sl = [int(rng.integers(1, f + 1)) for f in full]
    if long_run:
        sl[0] = full[0]  # a fully covered leading dimension fuses into the run
    off = [int(rng.integers(0, f - s + 1)) for f, s in zip(full, sl)]
    return full, sl, off


def _dev(torch, a):
    return torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("r", [1, 2, 3, 4, 6])
def test_device_slice_insert_bit_exact(talsh, kind, r):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(r * 31 + kind)
    L = T.lib()
    s = torch.cuda.current_stream().cuda_stream
    for long_run in (False, True):
        full, sl, off = _case(rng, r, long_run)
        F, S0 = rand(full, kind, rng), rand(sl, kind, rng)
        for acc in (0, 1):
            # slice
            f, d = _dev(torch, F), _dev(torch, S0)
            assert L.tcTensorSlice(kind, r, T.ivec(full), T.ivec(sl), T.ivec(off), f.data_ptr(), d.data_ptr(),
                                   acc, s) == 0
            want = S0.copy(order="F")
            assert O.tensor_slice(want, F, off, bool(acc)) == 0
            torch.cuda.synchronize()
            assert np.array_equal(d.cpu().numpy().reshape(sl, order="F"), want), (full, sl, off, acc)
            # insert
            f = _dev(torch, F)
            d = _dev(torch, S0)
            assert L.tcTensorInsert(kind, r, T.ivec(full), T.ivec(sl), T.ivec(off), d.data_ptr(), f.data_ptr(),
                                    acc, s) == 0
            want = F.copy(order="F")
            assert O.tensor_insert(want, S0, off, bool(acc)) == 0
            torch.cuda.synchronize()
            assert np.array_equal(f.cpu().numpy().reshape(full, order="F"), want), (full, sl, off, acc)


def test_device_slice_rejects_out_of_range(talsh):
    L = T.lib()
    args = (T.R8, 2, T.ivec([4, 4]), T.ivec([3, 3]))
    assert L.tcTensorSlice(*args, T.ivec([2, 0]), 1, 1, 0, None) == T.TALSH_INVALID_ARGS
    assert L.tcTensorInsert(*args, T.ivec([0, -1]), 1, 1, 0, None) == T.TALSH_INVALID_ARGS


@pytest.mark.parametrize("kind", [T.R8, T.C8])
def test_talsh_slice_and_insert(talsh, kind):
    """talshTensorSlice / talshTensorInsert (talsh.h API, Host tensors staged to GPU 0)."""
    rng = np.random.default_rng(4)
    full, sl, off = [17, 9, 23], [5, 9, 11], [3, 0, 7]
    F, S0 = rand(full, kind, rng), rand(sl, kind, rng)
    Lb = T.lib()
    for acc in (T.NOPE, T.YEP):
        S = S0.copy(order="F")
        dt, lt = host_tensor(S), host_tensor(F)
        assert Lb.talshTensorSlice(dt.ref, lt.ref, T.ivec(off), 0, T.DEV_NVIDIA_GPU, T.COPY_TT, acc, None) == 0
        dt.destruct(); lt.destruct()
        want = S0.copy(order="F")
        assert O.tensor_slice(want, F, off, acc == T.YEP) == 0
        assert np.array_equal(S, want)
        G = F.copy(order="F")
        dt, lt = host_tensor(G), host_tensor(S0)
        assert Lb.talshTensorInsert(dt.ref, lt.ref, T.ivec(off), 0, T.DEV_NVIDIA_GPU, T.COPY_TT, acc, None) == 0
        dt.destruct(); lt.destruct()
        want = F.copy(order="F")
        assert O.tensor_insert(want, S0, off, acc == T.YEP) == 0
        assert np.array_equal(G, want)
    # a slice that does not fit is refused before any work
    S = fort(np.zeros([5, 9, 11], dtype=F.dtype))
    dt, lt = host_tensor(S), host_tensor(F)
    assert Lb.talshTensorSlice(dt.ref, lt.ref, T.ivec([13, 0, 0]), 0, T.DEV_NVIDIA_GPU, T.COPY_TT, T.NOPE,
                               None) == T.TALSH_INVALID_ARGS
    dt.destruct(); lt.destruct()
