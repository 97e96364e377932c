"""The transpose autotuner (tcTensorPermuteTune / Tuned / TuneSet / TuneReset).

Every plan choice the tuner can record must give the same bytes as the oracle
(the reference's tensor_block_copy / tensor_block_add,
tensor_algebra_cpu.F90:3151-3310, :3312-3673): the choices change the tile
shape, the read path and the tile order, never the element arithmetic.  The
GPU tests pin every choice on sweep-like cases (odd, unit and power-of-two
extents, ranks 2-6, R4/R8/C8) and compare copy and add byte for byte; a tuned
run must record a valid choice for the case's class.  The CPU test covers the
table itself (it needs no device)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

CASES = [
    (T.R4, [44, 17, 18, 39, 2, 3], [4, 3, 6, 1, 2, 5]),
    (T.R4, [4, 6, 3, 571, 41], [3, 5, 2, 4, 1]),
    (T.R4, [1088, 1280], [2, 1]),
    (T.R8, [279, 2, 37, 19, 31], [2, 1, 5, 4, 3]),
    (T.R8, [25, 598, 13, 9], [4, 2, 3, 1]),
    (T.R8, [64, 32, 16, 8], [3, 4, 1, 2]),
    (T.C8, [17, 31, 3, 5], [3, 1, 4, 2]),
    (T.R8, [2, 1383, 2, 213], [1, 2, 3, 4]),  # fuses to a straight copy: one plan only
]


def test_tune_table_without_gpu(built):
    """TuneSet / Tuned / TuneReset keep a per-class table on the host."""
    L = T.lib()
    L.tcTensorPermuteTuneReset()
    ch = C.c_int(7)
    kind, dims, o2n = CASES[0]
    args = (kind, len(dims), T.ivec(dims), T.ivec(o2n))
    assert L.tcTensorPermuteTuned(*args, 0, C.byref(ch)) == 0 and ch.value == -1
    for choice in range(216):
        rc = L.tcTensorPermuteTuneSet(*args, 1, choice)
        assert rc in (0, T.TALSH_INVALID_ARGS)
        if rc == 0:
            assert L.tcTensorPermuteTuned(*args, 1, C.byref(ch)) == 0 and ch.value == choice
    # the copy class is separate from the add class
    assert L.tcTensorPermuteTuned(*args, 0, C.byref(ch)) == 0 and ch.value == -1
    # a case of the same class (same fused permutation and buckets) shares the entry
    assert L.tcTensorPermuteTuneSet(*args, 0, 2) == 0
    dims2 = list(dims)
    dims2[3] += 2  # 39 -> 41: same log2 buckets, same alignment
    assert L.tcTensorPermuteTuned(kind, len(dims2), T.ivec(dims2), T.ivec(o2n), 0, C.byref(ch)) == 0
    assert ch.value == 2
    assert L.tcTensorPermuteTuneSet(*args, 0, -1) == 0
    assert L.tcTensorPermuteTuned(*args, 0, C.byref(ch)) == 0 and ch.value == -1
    # invalid arguments
    assert L.tcTensorPermuteTuneSet(*args, 0, 216) == T.TALSH_INVALID_ARGS
    assert L.tcTensorPermuteTuneSet(*args, 0, -2) == T.TALSH_INVALID_ARGS
    assert L.tcTensorPermuteTuned(kind, len(dims), T.ivec(dims), T.ivec([1, 1, 2, 3, 4, 5]), 0,
                                  C.byref(ch)) == T.TALSH_INVALID_ARGS
    # straight copies have one plan: nothing is recorded
    kind, dims, o2n = CASES[-1]
    assert L.tcTensorPermuteTuneSet(kind, len(dims), T.ivec(dims), T.ivec(o2n), 0, 1) == 0
    assert L.tcTensorPermuteTuned(kind, len(dims), T.ivec(dims), T.ivec(o2n), 0, C.byref(ch)) == 0
    assert ch.value == -1
    L.tcTensorPermuteTuneReset()


def _dtype(kind):
    return {T.R4: np.float32, T.R8: np.float64, T.C4: np.complex64, T.C8: np.complex128}[kind]


def _rand(shape, kind, rng):
    x = rng.uniform(-1, 1, shape)
    if kind in (T.C4, T.C8):
        x = x + 1j * rng.uniform(-1, 1, shape)
    return np.asfortranarray(x.astype(_dtype(kind)))


def _run(torch, L, kind, dims, o2n, Lh, D0, alpha):
    """(copy bytes, add bytes) of the device path for one case."""
    s = torch.cuda.current_stream().cuda_stream
    lt = torch.from_numpy(Lh.ravel(order="F").view(np.uint8).copy()).cuda()
    dt = torch.from_numpy(D0.ravel(order="F").view(np.uint8).copy()).cuda()
    rc = L.tcTensorPermuteAdd(kind, len(dims), T.ivec(dims), T.ivec(o2n), lt.data_ptr(), dt.data_ptr(),
                              alpha, 0.0, 0, s)
    assert rc == 0, L.tcLastErrorString()
    torch.cuda.synchronize()
    got_add = dt.cpu().numpy().tobytes()
    rc = L.tcTensorPermute(kind, len(dims), T.ivec(dims), T.ivec(o2n), lt.data_ptr(), dt.data_ptr(), 0, s)
    assert rc == 0, L.tcLastErrorString()
    torch.cuda.synchronize()
    return dt.cpu().numpy().tobytes(), got_add


@pytest.mark.gpu
def test_every_choice_bit_exact(talsh):
    torch = pytest.importorskip("torch")
    L = T.lib()
    rng = np.random.default_rng(31)
    tried = 0
    try:
        for kind, dims, o2n in CASES:
            Lh = _rand(dims, kind, rng)
            D0 = _rand(O.out_dims(dims, o2n), kind, rng)
            ref_copy = O.permute(Lh, o2n).tobytes(order="F")
            ref = D0.copy(order="F")
            O.tensor_add(ref, Lh, o2n, 0.5)
            for choice in range(216):
                for acc in (0, 1):
                    rc = L.tcTensorPermuteTuneSet(kind, len(dims), T.ivec(dims), T.ivec(o2n), acc, choice)
                    assert rc in (0, T.TALSH_INVALID_ARGS)
                got_copy, got_add = _run(torch, L, kind, dims, o2n, Lh, D0, 0.5)
                assert got_copy == ref_copy, (dims, o2n, choice)
                assert got_add == ref.tobytes(order="F"), (dims, o2n, choice)
                tried += 1
    finally:
        L.tcTensorPermuteTuneReset()
    assert tried == 216 * len(CASES)


@pytest.mark.gpu
def test_tune_records_a_choice(talsh):
    torch = pytest.importorskip("torch")
    L = T.lib()
    rng = np.random.default_rng(32)
    ch, ch2 = C.c_int(-5), C.c_int(-5)
    s = torch.cuda.current_stream().cuda_stream
    try:
        for kind, dims, o2n in CASES:
            Lh = _rand(dims, kind, rng)
            nb = Lh.nbytes
            lt = torch.from_numpy(Lh.ravel(order="F").view(np.uint8).copy()).cuda()
            dt = torch.zeros(nb, dtype=torch.uint8, device="cuda")
            args = (kind, len(dims), T.ivec(dims), T.ivec(o2n))
            for acc in (0, 1):
                rc = L.tcTensorPermuteTune(*args, acc, lt.data_ptr(), dt.data_ptr(), s, 2, C.byref(ch))
                assert rc == 0, L.tcLastErrorString()
                assert 0 <= ch.value <= 215
                assert L.tcTensorPermuteTuned(*args, acc, C.byref(ch2)) == 0
                straight = len(o2n) > 1 and list(o2n) == sorted(o2n)
                assert ch2.value == (-1 if straight else ch.value)
            # after tuning, both operations still match the oracle
            D0 = _rand(O.out_dims(dims, o2n), kind, rng)
            got_copy, got_add = _run(torch, L, kind, dims, o2n, Lh, D0, -1.25)
            assert got_copy == O.permute(Lh, o2n).tobytes(order="F")
            ref = D0.copy(order="F")
            O.tensor_add(ref, Lh, o2n, -1.25)
            assert got_add == ref.tobytes(order="F")
        kind, dims, o2n = CASES[0]
        assert L.tcTensorPermuteTune(kind, len(dims), T.ivec(dims), T.ivec(o2n), 0, lt.data_ptr(),
                                     dt.data_ptr(), s, 0, C.byref(ch)) == T.TALSH_INVALID_ARGS
    finally:
        L.tcTensorPermuteTuneReset()


@pytest.mark.gpu
def test_tuned_sweep_slice_bit_exact(talsh):
    """Tune every 8th case of the benchmark sweep (capped at 2^21 elements), then
    run all of them through the tuned table against the oracle."""
    torch = pytest.importorskip("torch")
    L = T.lib()
    rng = np.random.default_rng(33)
    s = torch.cuda.current_stream().cuda_stream
    ch = C.c_int(0)
    bad = []
    try:
        for i, (kind, dims, o2n) in enumerate(bench.c2_cases()):
            if i % 8:
                continue
            dims = list(dims)
            while int(np.prod(dims, dtype=np.int64)) > (1 << 21):
                dims[int(np.argmax(dims))] //= 2
            Lh = _rand(dims, kind, rng)
            lt = torch.from_numpy(Lh.ravel(order="F").view(np.uint8).copy()).cuda()
            dt = torch.zeros(Lh.nbytes, dtype=torch.uint8, device="cuda")
            for acc in (0, 1):
                assert L.tcTensorPermuteTune(kind, len(dims), T.ivec(dims), T.ivec(o2n), acc, lt.data_ptr(),
                                             dt.data_ptr(), s, 1, C.byref(ch)) == 0
            D0 = _rand(O.out_dims(dims, o2n), kind, rng)
            sr = bench.ALPHAS[i % len(bench.ALPHAS)][0]
            got_copy, got_add = _run(torch, L, kind, dims, o2n, Lh, D0, sr)
            ref = D0.copy(order="F")
            O.tensor_add(ref, Lh, o2n, sr)
            if got_copy != O.permute(Lh, o2n).tobytes(order="F"):
                bad.append(("copy", i, dims, o2n))
            if got_add != ref.tobytes(order="F"):
                bad.append(("add", i, dims, o2n))
    finally:
        L.tcTensorPermuteTuneReset()
    assert not bad, bad[:8]
