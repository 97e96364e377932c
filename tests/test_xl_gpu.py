"""Out-of-core contraction (talshTensorContractXL, reference talshc.cpp:5394-5648):
operands on the Host, decomposed by halving (talshTensorOpDecompose2 :3150-3294)
until the blocks fit the GPU budget, results against the oracle."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, host_tensor, rand

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [  # pattern, extents, kind, alpha, accumulative
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=24, b=20, c=18, i=9, j=8, k=7), T.R8, (0.5, 0.0), True),
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=24, b=20, c=18, i=9, j=8, k=7), T.R8, (1.0, 0.0), False),
    ("D(a,b)+=L(k,a,c)*R(c,k,b)", dict(a=70, b=60, c=40, k=30), T.C8, (0.5, -0.25), True),
    ("D(i,j,k)+=L(k,a,i,b)*R(b,k,a,j)", dict(i=30, j=20, k=16, a=12, b=10), T.C8, (0.5, 0.0), True),  # hyper k
    ("D()+=L(a,b,c)*R(c,b,a)", dict(a=60, b=50, c=40), T.R8, (1.0, 0.0), True),                      # full
]


def _dims(pattern, ext):
    import re
    return [[ext[x] for x in g.split(",") if x] for g in re.findall(r"\(([^)]*)\)", pattern)]


def _run(pattern, ext, kind, alpha, acc, seed=0):
    rng = np.random.default_rng(seed)
    dd, ld, rd = _dims(pattern, ext)
    D0 = rand(dd, kind, rng) if dd else np.asarray(rng.uniform(-1, 1), dtype=T.NP_DTYPE[kind])
    L, R = rand(ld, kind, rng), rand(rd, kind, rng)
    ref = np.array(D0, copy=True, order="F")
    e, dig, *_ = T.parse_pattern(pattern)
    assert O.tensor_contract(ref, L, R, dig, alpha[0], alpha[1], 0, acc) == 0
    got = np.array(D0, copy=True, order="F")
    dt, lt, rt = host_tensor(got), host_tensor(L), host_tensor(R)
    rc = T.lib().talshTensorContractXL(pattern.encode(), dt.ref, lt.ref, rt.ref, alpha[0], alpha[1], 0,
                                        T.DEV_NVIDIA_GPU, T.YEP if acc else T.NOPE)
    dt.destruct(); lt.destruct(); rt.destruct()
    assert rc == 0, rc
    base = D0 if acc else 0
    err = np.linalg.norm(np.ravel(got - ref)) / np.linalg.norm(np.ravel(ref - base))
    return err, T.lib().tcContractXLLastOps()


@pytest.mark.parametrize("pattern,ext,kind,alpha,acc", CASES)
def test_xl_whole_on_gpu(talsh, pattern, ext, kind, alpha, acc):
    """Operands that fit: one sub-contraction."""
    err, nops = _run(pattern, ext, kind, alpha, acc)
    assert err <= 1e-12 and nops == 1


def test_xl_decomposed_under_small_budget():
    """A 1 MiB device budget forces sub-contractions (D, L, R and
    contracted splits, the hyper and full forms)."""
    code = r"""
import ctypes as C, sys
sys.path.insert(0, %r); sys.path.insert(0, %r)
import tal_sh_b200 as T
import test_xl_gpu as t
L = T.lib()
hb, ha = C.c_size_t(0), C.c_int(0)
assert L.talshInit(C.byref(hb), C.byref(ha), 1, T.ivec([0]), 0, None, 0, None) == 0
for case in t.CASES:
    err, nops = t._run(*case)
    assert err <= 1e-12 and nops >= 2, (case[0], err, nops)
    print(case[0], nops, err)
assert L.talshShutdown() == 0
print("OK")
""" % (ROOT, os.path.join(ROOT, "tests"))
    env = dict(os.environ, TALSH_B200_GPU_BUDGET_BYTES=str(1 << 20))
    p = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=600)
    assert p.returncode == 0 and "OK" in p.stdout, p.stdout
