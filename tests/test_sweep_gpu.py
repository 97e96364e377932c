"""The transpose/add sweep's every case, bit-exact on the GPU.

All 320 cases of the seeded sweep the benchmark times (ranks 2-6, every
permutation of ranks 2-4, 64 seeded permutations each of ranks 5 and 6, R4 and
R8, odd and unit extents), with each case's volume capped at 2^22 elements by
halving its largest extent (the shape's character -- rank, permutation, odd and
unit extents -- is kept).  Each case runs one transpose and one transpose-add
(alpha cycling through 1, 0.5, -1.25, as the benchmark does) through the device
C ABI (tcTensorPermute / tcTensorPermuteAdd) and is compared byte for byte with
the oracle: the reference's cache-blocked transpose (tensor_block_copy_dlf,
tensor_algebra_cpu.F90:7699-7940) and its add flow (cpu_tensor_block_add,
talshf.F90:1857-1904 -> tensor_block_add, tensor_algebra_cpu.F90:3312-3673).
A CPU test pins those multi-threaded oracle routines to the oracle's scatter
definitions on every case."""
import os
import sys

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

CAP = 1 << 22


def capped(dims, cap):
    dims = list(dims)
    while int(np.prod(dims, dtype=np.int64)) > cap:
        dims[int(np.argmax(dims))] //= 2
    return dims


def test_sweep_blocked_oracle_matches_definition(built):
    """The oracle's blocked transpose and blocked add equal its scatter definitions
    on every sweep case (capped at 2^14 elements), so the GPU test below may use them."""
    rng = np.random.default_rng(7)
    for i, (kind, dims, o2n) in enumerate(bench.c2_cases()):
        dims = capped(dims, 1 << 14)
        dt = np.float32 if kind == T.R4 else np.float64
        L = np.asfortranarray(rng.uniform(-1, 1, dims).astype(dt))
        assert O.permute(L, o2n, blocked=True, nthreads=4).tobytes(order="F") == \
            O.permute(L, o2n).tobytes(order="F"), (i, dims, o2n)
        D = np.asfortranarray(rng.uniform(-1, 1, O.out_dims(dims, o2n)).astype(dt))
        a, b = D.copy(order="F"), D.copy(order="F")
        sr = bench.ALPHAS[i % len(bench.ALPHAS)][0]
        O.tensor_add(a, L, o2n, sr)
        O.tensor_add_blocked(b, L, o2n, sr, nthreads=4)
        assert a.tobytes(order="F") == b.tobytes(order="F"), (i, dims, o2n)


@pytest.mark.gpu
def test_sweep_every_case_bit_exact(talsh):
    torch = pytest.importorskip("torch")
    L = T.lib()
    cases = bench.c2_cases()
    assert len(cases) == 320
    rng = np.random.default_rng(2024)
    nt = os.cpu_count() or 1
    stream = torch.cuda.current_stream().cuda_stream
    bad = []
    for i, (kind, dims, o2n) in enumerate(cases):
        dims = capped(dims, CAP)
        dt = np.float32 if kind == T.R4 else np.float64
        Lh = np.asfortranarray(rng.uniform(-1, 1, dims).astype(dt))
        D0 = np.asfortranarray(rng.uniform(-1, 1, O.out_dims(dims, o2n)).astype(dt))
        l = torch.from_numpy(Lh.ravel(order="F")).cuda()
        d = torch.from_numpy(D0.ravel(order="F")).cuda()
        sr = bench.ALPHAS[i % len(bench.ALPHAS)][0]
        # transpose-add into D0, then the transpose over it
        rc = L.tcTensorPermuteAdd(kind, len(dims), T.ivec(dims), T.ivec(o2n), l.data_ptr(), d.data_ptr(),
                                  sr, 0.0, 0, stream)
        assert rc == 0, (i, rc, L.tcLastErrorString())
        torch.cuda.synchronize()
        got_add = d.cpu().numpy().tobytes()
        ref = D0.copy(order="F")
        O.tensor_add_blocked(ref, Lh, o2n, sr, nthreads=nt)
        if got_add != ref.tobytes(order="F"):
            bad.append(("add", i, dims, o2n))
        rc = L.tcTensorPermute(kind, len(dims), T.ivec(dims), T.ivec(o2n), l.data_ptr(), d.data_ptr(), 0, stream)
        assert rc == 0, (i, rc, L.tcLastErrorString())
        torch.cuda.synchronize()
        if d.cpu().numpy().tobytes() != O.permute(Lh, o2n, blocked=True, nthreads=nt).tobytes(order="F"):
            bad.append(("copy", i, dims, o2n))
    assert not bad, bad[:8]
