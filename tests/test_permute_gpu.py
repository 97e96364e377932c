"""Transpose and transpose-add on the GPU through talshTensorCopy / talshTensorAdd,
bit-exact against the oracle (reference tensor_block_copy / tensor_block_add)."""
import ctypes as C
import itertools
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, gpu_add, gpu_copy, rand, same_bits

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KINDS = [T.R4, T.R8, T.C4, T.C8]
LAB = "abcdefgh"


def patterns(rank, o2n):
    """Copy pattern string for O2N: D's index at position o2n[i] is L's index i."""
    dlab = [None] * rank
    for i, p in enumerate(o2n):
        dlab[p - 1] = LAB[i]
    return "D(%s)=L(%s)" % (",".join(dlab), ",".join(LAB[:rank]))


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("dims", [(17, 31), (7, 1, 5), (17, 31, 3), (5, 6, 7, 3), (2, 3, 97, 4), (31, 17, 2, 3)])
def test_copy_all_permutations_bit_exact(talsh, dims, kind):
    rng = np.random.default_rng(hash((dims, kind)) % 2 ** 32)
    L = rand(dims, kind, rng)
    for o2n in itertools.permutations(range(1, len(dims) + 1)):
        pat = patterns(len(dims), o2n)
        D = fort(np.full(O.out_dims(list(dims), o2n), np.nan, dtype=L.dtype))
        assert gpu_copy(pat, D, L) == 0, pat
        assert same_bits(D, O.permute(L, list(o2n))), pat


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("rank", [5, 6])
def test_copy_random_high_rank_bit_exact(talsh, rank, kind):
    rng = np.random.default_rng(rank * 100 + kind)
    for _ in range(8):
        dims = [int(x) for x in rng.choice([2, 3, 5, 7, 11, 17], size=rank)]
        o2n = [int(x) + 1 for x in rng.permutation(rank)]
        L = rand(dims, kind, rng)
        D = fort(np.zeros(O.out_dims(dims, o2n), dtype=L.dtype))
        pat = patterns(rank, o2n)
        assert gpu_copy(pat, D, L) == 0
        assert same_bits(D, O.permute(L, o2n)), (dims, o2n)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("alpha", [(1.0, 0.0), (0.5, 0.0), (-1.25, 0.0), (0.3, 0.4), (0.0, -2.0)])
def test_add_bit_exact(talsh, kind, alpha):
    rng = np.random.default_rng(kind)
    for dims, o2n in [((17, 31, 3), (3, 1, 2)), ((5, 6, 7, 3), (4, 3, 2, 1)), ((64, 32), (1, 2)), ((33, 9, 4), (2, 1, 3))]:
        L = rand(dims, kind, rng)
        D0 = rand(O.out_dims(list(dims), o2n), kind, rng)
        D = D0.copy(order="F")
        pat = patterns(len(dims), o2n).replace(")=L", ")+=L")
        assert gpu_add(pat, D, L, *alpha) == 0
        ref = D0.copy(order="F")
        O.tensor_add(ref, L, list(o2n), *alpha)
        assert same_bits(D, ref), (dims, o2n, alpha)


@pytest.mark.parametrize("kind", [T.C4, T.C8])
def test_conjugated_copy_and_add(talsh, kind):
    rng = np.random.default_rng(11)
    L = rand((7, 9, 5), kind, rng)
    D = fort(np.zeros((5, 7, 9), dtype=L.dtype))
    assert gpu_copy("D(c,a,b)=L+(a,b,c)", D, L) == 0
    assert same_bits(D, O.permute(L, [2, 3, 1], conj=True))
    D0 = rand((5, 7, 9), kind, rng)
    D = D0.copy(order="F")
    assert gpu_add("D+(c,a,b)+=L(a,b,c)", D, L, 0.5, 0.25) == 0  # D conjugation flips the L bit
    ref = D0.copy(order="F")
    O.tensor_add(ref, L, [2, 3, 1], 0.5, 0.25, conj_bits=1)
    assert same_bits(D, ref)


def test_c1_transpose(talsh):
    """D(i,c,a,b)=L(a,b,c,i) on the 32^4 R8 tensor of the C1 workload."""
    L = O.uniform((32, 32, 32, 32), O.R8, 0)
    D = fort(np.zeros((32, 32, 32, 32)))
    assert gpu_copy("D(i,c,a,b)=L(a,b,c,i)", D, L) == 0
    assert same_bits(D, O.permute(L, [3, 4, 2, 1]))
    D2 = fort(np.zeros((32, 32, 32, 32)))
    assert gpu_add("D(i,c,a,b)+=L(a,b,c,i)", D2, L) == 0
    assert same_bits(D2, D)


@pytest.mark.parametrize("kind", [T.R4, T.R8])
def test_large_volumes_bit_exact(talsh, kind):
    """Volumes above L2 with aligned (vectorized) and odd (scalar) extents."""
    rng = np.random.default_rng(12)
    for dims, o2n in [((256, 128, 96), (3, 1, 2)), ((97, 31, 17, 40), (4, 2, 3, 1)), ((1024, 2048), (2, 1)),
                      ((40, 40, 20, 20, 20), (5, 4, 3, 2, 1)), ((512, 3, 700), (1, 3, 2))]:
        L = rand(dims, kind, rng)
        D = fort(np.zeros(O.out_dims(list(dims), o2n), dtype=L.dtype))
        assert gpu_copy(patterns(len(dims), o2n), D, L) == 0
        assert same_bits(D, O.permute(L, list(o2n))), (dims, o2n)


@pytest.mark.parametrize("kind", KINDS)
def test_table_path_bit_exact(talsh, kind):
    """Tensors large enough for the per-element tables, with extents that leave
    cut-short tiles along either split dimension or both (copy, add, conj)."""
    rng = np.random.default_rng(kind + 40)
    lib = T.lib()
    info = (C.c_int * 12)()
    cases = [((97, 131, 17, 23), (4, 3, 1, 2)), ((25, 9, 9, 10, 121), (3, 2, 1, 4, 5)),
             ((2, 347, 2, 241, 31), (1, 5, 4, 3, 2)), ((1321, 2, 31, 61), (3, 4, 1, 2)),
             ((30, 47, 2, 17, 113), (4, 3, 5, 2, 1)), ((17, 3, 40961), (1, 3, 2)),
             ((5, 7, 11, 13, 17, 3), (6, 4, 2, 5, 1, 3))]
    used = 0
    for dims, o2n in cases:
        assert lib.tcPermutePlanInfo(kind, len(dims), T.ivec(dims), T.ivec(o2n), info) == 0
        used += info[11]
        L = rand(dims, kind, rng)
        D = fort(np.full(O.out_dims(list(dims), o2n), np.nan, dtype=L.dtype))
        assert gpu_copy(patterns(len(dims), o2n), D, L) == 0
        assert same_bits(D, O.permute(L, list(o2n))), (dims, o2n)
        D0 = rand(O.out_dims(list(dims), o2n), kind, rng)
        D = D0.copy(order="F")
        assert gpu_add(patterns(len(dims), o2n).replace(")=L", ")+=L"), D, L, 0.75, 0.0) == 0
        ref = D0.copy(order="F")
        O.tensor_add(ref, L, list(o2n), 0.75, 0.0)
        assert same_bits(D, ref), ("add", dims, o2n)
    assert used >= len(cases) - 1  # the cases are meant to take the table path


def test_generic_kernel_bit_exact(built):
    """The generic kernel (64-bit run tables, used when a tile spans more than
    2^31 elements) is forced for every plan in a child process and checked on
    small and table-sized cases, copy and add, every kind."""
    code = r"""
import ctypes as C, itertools, sys
sys.path.insert(0, %r); sys.path.insert(0, %r)
import numpy as np
import oracle as O, tal_sh_b200 as T
from gpu_util import fort, rand, same_bits, gpu_copy, gpu_add
L = T.lib()
hb, ha = C.c_size_t(0), C.c_int(0)
assert L.talshInit(C.byref(hb), C.byref(ha), 1, T.ivec([0]), 0, None, 0, None) == 0
info = (C.c_int * 12)()
LAB = "abcdefgh"
def pat(o2n, add):
    d = [None] * len(o2n)
    for i, p in enumerate(o2n): d[p - 1] = LAB[i]
    return "D(%%s)%%s=L(%%s)" %% (",".join(d), "+" if add else "", ",".join(LAB[:len(o2n)]))
rng = np.random.default_rng(5)
cases = [((17, 31, 3), (3, 1, 2)), ((5, 6, 7, 3), (4, 3, 2, 1)), ((97, 131, 17, 23), (4, 3, 1, 2)),
         ((25, 9, 9, 10, 121), (3, 2, 1, 4, 5)), ((64, 32, 3), (2, 1, 3))]
for kind in (T.R4, T.R8, T.C4, T.C8):
    for dims, o2n in cases:
        assert L.tcPermutePlanInfo(kind, len(dims), T.ivec(dims), T.ivec(o2n), info) == 0
        assert info[11] == 0
        A = rand(dims, kind, rng)
        D = fort(np.full(O.out_dims(list(dims), o2n), np.nan, dtype=A.dtype))
        assert gpu_copy(pat(o2n, False), D, A) == 0
        assert same_bits(D, O.permute(A, list(o2n))), (kind, dims, o2n)
        D0 = rand(O.out_dims(list(dims), o2n), kind, rng)
        D = D0.copy(order="F")
        assert gpu_add(pat(o2n, True), D, A, -1.25, 0.0) == 0
        ref = D0.copy(order="F"); O.tensor_add(ref, A, list(o2n), -1.25, 0.0)
        assert same_bits(D, ref), ("add", kind, dims, o2n)
assert L.talshShutdown() == 0
print("OK")
""" % (ROOT, os.path.join(ROOT, "tests"))
    env = dict(os.environ, TALSH_B200_PERMUTE_GENERIC="1")
    p = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=600)
    assert p.returncode == 0 and "OK" in p.stdout, p.stdout


def test_plan_properties(talsh):
    L = T.lib()
    info = (C.c_int * 12)()
    assert L.tcPermutePlanInfo(T.R8, 4, T.ivec([32, 32, 32, 32]), T.ivec([3, 4, 2, 1]), info) == 0
    assert info[0] == 3 and info[1] == 0 and info[3] >= 32 and info[4] >= 32  # (a,b) fuse; coalesced runs
    assert info[8] == 2  # 16-byte vector stores on the output side
    assert L.tcPermutePlanInfo(T.R8, 3, T.ivec([4, 5, 6]), T.ivec([1, 2, 3]), info) == 0
    assert info[1] == 1  # identity fuses to a straight copy


def test_edge_cases(talsh):
    rng = np.random.default_rng(13)
    # rank 0 and volume-1 tensors
    for dims in [(), (1,), (1, 1, 1)]:
        L = fort(np.asarray(rng.standard_normal(dims)))
        D = fort(np.zeros(dims))
        pat = "D(%s)=L(%s)" % (",".join(LAB[:len(dims)]), ",".join(LAB[:len(dims)]))
        assert gpu_copy(pat, D, L) == 0 and same_bits(D, L)
    # extent mismatch and malformed patterns are rejected before any work
    L = fort(rng.standard_normal((3, 4)))
    D = fort(np.zeros((3, 4)))
    assert gpu_copy("D(a,b)=L(b,a)", D, L) == T.TALSH_INVALID_ARGS
    assert gpu_copy("D(a,b)=L(a,c)", D, L) == T.TALSH_INVALID_ARGS
