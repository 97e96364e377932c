"""TAL-SH runtime semantics on the GPU: asynchronous tasks and their status
ladder, coherence control (COPY_D/M/T/K), placement, GPU-resident tensors,
init/scale bit-exactness, the GPU 1-norm, and TRY_LATER under a memory budget."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, host_tensor, rand, rel_err, same_bits

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPU0 = 1  # flat device id of GPU 0


def test_async_task_and_timings(talsh):
    L = talsh
    rng = np.random.default_rng(0)
    A, B = rand((64, 48, 32), T.R8, rng), rand((32, 40), T.R8, rng)
    D = fort(np.zeros((64, 48, 40)))
    d, a, b = host_tensor(D), host_tensor(A), host_tensor(B)
    task = T.Task()
    L.talshTaskClean(C.byref(task))
    rc = L.talshTensorContract(b"D(x,y,z)+=L(x,y,k)*R(k,z)", d.ref, a.ref, b.ref, 1.0, 0.0, 0, T.DEV_NVIDIA_GPU,
                               T.COPY_TTT, T.YEP, C.byref(task))
    assert rc == 0
    seen = set()
    stats, ierr = C.c_int(), C.c_int()
    while L.talshTaskComplete(C.byref(task), C.byref(stats), C.byref(ierr)) != T.YEP:
        assert ierr.value == 0
        seen.add(stats.value)
    assert stats.value == T.TALSH_TASK_COMPLETED and task.task_error == 0
    assert seen <= {T.TALSH_TASK_SCHEDULED, T.TALSH_TASK_STARTED, T.TALSH_TASK_INPUT_READY, T.TALSH_TASK_OUTPUT_READY}
    tot, comp, inp, out, mm = (C.c_double() for _ in range(5))
    assert L.talshTaskTime(C.byref(task), C.byref(tot), C.byref(comp), C.byref(inp), C.byref(out), C.byref(mm)) == 0
    assert tot.value > 0 and comp.value > 0 and tot.value >= comp.value
    assert task.flops == 2.0 * 64 * 48 * 40 * 32
    assert L.talshTaskDestruct(C.byref(task)) == 0
    assert rel_err(D, np.einsum("xyk,kz->xyz", A, B)) < 1e-13
    for t in (d, a, b):
        t.destruct()


def test_coherence_move_and_place(talsh):
    """COPY_MTT (the default) moves D to the GPU; talshTensorPlace(COPY_M) brings it back
    (the flow of the reference's test_talsh_c); T-arguments keep their Host images."""
    L = talsh
    rng = np.random.default_rng(1)
    A, B = rand((20, 30), T.R8, rng), rand((30, 25), T.R8, rng)
    d = T.Tensor([20, 25], T.R8, dev_id=0, init=0.0)
    a, b = host_tensor(A), host_tensor(B)
    assert L.talshTensorContract(b"D(i,j)+=L(i,k)*R(k,j)", d.ref, a.ref, b.ref, 2.0, 0.0, 0, T.DEV_NVIDIA_GPU,
                                 T.COPY_MTT, T.YEP, None) == 0
    assert [img[0] for img in d.images()] == [GPU0]          # moved
    assert [img[0] for img in a.images()] == [0]             # temporary copy discarded
    assert L.talshTensorImageNorm1_cpu(d.ref) == -1.0        # no Host image any more
    assert L.talshTensorPlace(d.ref, 0, T.DEV_HOST, None, T.COPY_M, None) == 0
    assert [img[0] for img in d.images()] == [0]
    assert rel_err(d.host_array(), 2.0 * A @ B) < 1e-13
    # COPY_K keeps both images
    assert L.talshTensorPlace(d.ref, 0, T.DEV_NVIDIA_GPU, None, T.COPY_K, None) == 0
    assert sorted(img[0] for img in d.images()) == [0, GPU0]
    assert L.talshTensorDiscard(d.ref, 0, T.DEV_NVIDIA_GPU) == 0
    assert [img[0] for img in d.images()] == [0]
    for t in (d, a, b):
        assert t.destruct() == 0


def test_chain_with_asynchronous_place(talsh):
    """A transpose and a transpose-add that keep D on the GPU between them
    (COPY_MK, then COPY_KD), then an asynchronous talshTensorPlace(COPY_M) of D
    into its Host buffer: one upload of L, one copy back of D, bit-exact with
    the oracle; the moved GPU image is discarded when the place task completes,
    L's kept image by the add."""
    L = talsh
    rng = np.random.default_rng(5)
    for kind in (T.R4, T.R8, T.C8):
        A = rand((17, 31, 6), kind, rng)
        D = fort(np.zeros((6, 17, 31), dtype=A.dtype))
        d, a = host_tensor(D), host_tensor(A)
        tasks = [T.Task() for _ in range(3)]
        for tk in tasks:
            L.talshTaskClean(C.byref(tk))
        st = C.c_int()

        def wait(tk):
            assert L.talshTaskWait(C.byref(tk), C.byref(st)) == 0 and st.value == T.TALSH_TASK_COMPLETED
            assert L.talshTaskDestruct(C.byref(tk)) == 0

        # The copy's result (moved to the GPU) and L's kept GPU copy are images
        # as soon as the copy is scheduled, so the add and the placement are
        # accepted at once and run after it in stream order.
        assert L.talshTensorCopy(b"D(c,a,b)=L(a,b,c)", d.ref, a.ref, 0, T.DEV_NVIDIA_GPU, T.COPY_MK,
                                 C.byref(tasks[0])) == 0
        assert L.talshTensorAdd(b"D(c,a,b)+=L(a,b,c)", d.ref, a.ref, 0.5, 0.0, 0, T.DEV_NVIDIA_GPU, T.COPY_KD,
                                C.byref(tasks[1])) == 0
        assert L.talshTensorPlace(d.ref, 0, T.DEV_HOST, C.c_void_p(D.ctypes.data), T.COPY_M,
                                  C.byref(tasks[2])) == 0
        for tk in tasks:
            wait(tk)
        ref = O.permute(A, [2, 3, 1])
        O.tensor_add(ref, A, [2, 3, 1], 0.5)
        assert same_bits(D, ref), kind
        assert [img[0] for img in d.images()] == [0]
        assert [img[0] for img in a.images()] == [0]
        for t in (d, a):
            assert t.destruct() == 0
    # An output staged as a temporary (COPY_T) is held until its task completes.
    A = rand((17, 31, 6), T.R8, rng)
    D = fort(np.zeros((6, 17, 31)))
    d, a = host_tensor(D), host_tensor(A)
    tk, tk2 = T.Task(), T.Task()
    L.talshTaskClean(C.byref(tk)); L.talshTaskClean(C.byref(tk2))
    assert L.talshTensorCopy(b"D(c,a,b)=L(a,b,c)", d.ref, a.ref, 0, T.DEV_NVIDIA_GPU, T.COPY_TT, C.byref(tk)) == 0
    rc = L.talshTensorPlace(d.ref, 0, T.DEV_NVIDIA_GPU, None, T.COPY_K, C.byref(tk2))
    assert rc in (0, T.TRY_LATER)  # TRY_LATER unless the copy already completed
    st = C.c_int()
    assert L.talshTaskWait(C.byref(tk), C.byref(st)) == 0 and st.value == T.TALSH_TASK_COMPLETED
    if rc == 0:
        assert L.talshTaskWait(C.byref(tk2), C.byref(st)) == 0
    L.talshTaskDestruct(C.byref(tk)); L.talshTaskDestruct(C.byref(tk2))
    assert same_bits(D, O.permute(A, [2, 3, 1]))
    for t in (d, a):
        assert t.destruct() == 0


def test_gpu_resident_tensors(talsh):
    """Tensors constructed on the GPU stay there; chains of operations run without transfers."""
    L = talsh
    a = T.Tensor([16, 24], T.R8, dev_id=GPU0, init=0.5)
    b = T.Tensor([24, 8], T.R8, dev_id=GPU0, init=-2.0)
    c = T.Tensor([16, 8], T.R8, dev_id=GPU0, init=1.0)
    assert L.talshTensorContract(b"D(i,j)+=L(i,k)*R(k,j)", c.ref, a.ref, b.ref, 1.0, 0.0, -1, -1, T.COPY_MTT, T.YEP,
                                 None) == 0
    assert L.talshTensorScale(c.ref, 0.5, 0.0, -1, -1, T.COPY_M, None) == 0
    assert [img[0] for img in c.images()] == [GPU0]
    s = C.c_double()
    assert L.talshTensorNorm1(c.ref, -1, -1) == pytest.approx(16 * 8 * abs((1.0 - 24.0) * 0.5))
    h = fort(np.zeros((16, 8)))
    ht = host_tensor(h)
    assert L.talshTensorCopy(b"D(i,j)=L(i,j)", ht.ref, c.ref, 0, T.DEV_NVIDIA_GPU, T.COPY_TK, None) == 0
    assert np.all(h == (1.0 - 24.0) * 0.5)
    for t in (a, b, c, ht):
        assert t.destruct() == 0


@pytest.mark.parametrize("kind", [T.R4, T.R8, T.C4, T.C8])
def test_init_scale_norm(talsh, kind):
    L = talsh
    rng = np.random.default_rng(kind)
    X = rand((33, 17, 9), kind, rng)
    for alpha in [(0.5, 0.0), (-3.0, 4.0), (0.0, 1.5)]:
        Y = X.copy(order="F")
        y = host_tensor(Y)
        assert L.talshTensorScale(y.ref, alpha[0], alpha[1], 0, T.DEV_NVIDIA_GPU, T.COPY_T, None) == 0
        y.destruct()
        ref = X.copy(order="F")
        O.tensor_scale(ref, *alpha)
        assert same_bits(Y, ref), alpha
    Z = fort(np.zeros_like(X))
    z = host_tensor(Z)
    assert L.talshTensorInit(z.ref, 0.25, -0.5, 0, T.DEV_NVIDIA_GPU, T.COPY_T, None) == 0
    z.destruct()
    ref = fort(np.zeros_like(X))
    O.lib().orc_tensor_init(kind, ref.size, O._ptr(ref), 0.25, -0.5, 0)
    assert same_bits(Z, ref)
    x = host_tensor(X)
    n1 = L.talshTensorNorm1(x.ref, 0, T.DEV_NVIDIA_GPU)
    # moduli of C4 elements are single precision (last-ulp differences between libm and CUDA)
    tol = 1e-6 if kind == T.C4 else 1e-12
    assert abs(n1 - O.norm1(X)) <= tol * O.norm1(X)
    assert L.talshTensorNorm1(x.ref, 0, T.DEV_NVIDIA_GPU) == n1  # deterministic
    assert [img[0] for img in x.images()] == [0]  # the staged copy was temporary
    x.destruct()


def test_try_later_under_budget():
    """A device budget smaller than the operands makes the operation TRY_LATER
    (not an error); the tensors are left exactly as they were."""
    code = r"""
import ctypes as C, numpy as np, sys
sys.path.insert(0, %r)
import tal_sh_b200 as T
L = T.lib()
hb, ha = C.c_size_t(0), C.c_int(0)
assert L.talshInit(C.byref(hb), C.byref(ha), 1, T.ivec([0]), 0, None, 0, None) == 0
A = np.asfortranarray(np.ones((512, 512))); B = np.asfortranarray(np.ones((512, 512))); D = np.asfortranarray(np.zeros((512, 512)))
d, a, b = T.Tensor([512, 512], T.R8, 0, ext=D), T.Tensor([512, 512], T.R8, 0, ext=A), T.Tensor([512, 512], T.R8, 0, ext=B)
rc = L.talshTensorContract(b"D(i,j)+=L(i,k)*R(k,j)", d.ref, a.ref, b.ref, 1.0, 0.0, 0, T.DEV_NVIDIA_GPU, T.COPY_TTT, T.YEP, None)
assert rc == T.TRY_LATER, rc
assert d.images() == [(0, T.R8, 1)] and a.images() == [(0, T.R8, 1)] and np.all(D == 0)
for t in (d, a, b): assert t.destruct() == 0
assert L.talshShutdown() == 0
print("OK")
""" % ROOT
    env = dict(os.environ, TALSH_B200_GPU_BUDGET_BYTES=str(3 * 1024 * 1024))
    p = subprocess.run([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True, timeout=300)
    assert p.returncode == 0 and "OK" in p.stdout, p.stdout


def test_device_abi_direct(talsh):
    """tcTensorPermute / tcTensorContract on device buffers and a caller's stream."""
    torch = pytest.importorskip("torch")
    L = talsh
    rng = np.random.default_rng(3)
    A = rand((40, 30, 20), T.R8, rng)
    src = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    dst = torch.empty_like(src)
    stream = torch.cuda.current_stream().cuda_stream
    assert L.tcTensorPermute(T.R8, 3, T.ivec([40, 30, 20]), T.ivec([2, 3, 1]), src.data_ptr(), dst.data_ptr(), 0,
                             stream) == 0
    torch.cuda.synchronize()
    out = dst.cpu().numpy().reshape((20, 40, 30), order="F")
    assert same_bits(out, O.permute(A, [2, 3, 1]))
    before = L.tcKernelLaunchCount()
    assert L.tcTensorPermute(T.R8, 3, T.ivec([40, 30, 20]), T.ivec([1, 1, 2]), src.data_ptr(), dst.data_ptr(), 0,
                             stream) == T.TALSH_INVALID_ARGS
    assert L.tcKernelLaunchCount() == before


def test_host_mem_register_pins_caller_memory(talsh):
    """host_mem_register / host_mem_unregister (mem_manager.h; the reference C++
    layer's pinHostMemory / unpinHostMemory): 0 on success, 1 for a second
    registration or an unregistration of memory that is not pinned."""
    L = talsh
    buf = np.zeros(1 << 16)
    p = C.c_void_p(buf.ctypes.data)
    assert L.host_mem_register(p, buf.nbytes) == 0
    try:
        assert L.host_mem_register(p, buf.nbytes) == 1
    finally:
        assert L.host_mem_unregister(p) == 0
    assert L.host_mem_unregister(p) == 1


class _DeviceBlock:
    """A device pointer seen by torch through the CUDA array interface (no copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "strides": None,
                                          "version": 2}


def test_device_resource_memory_from_caller_streams(talsh):
    """tensDevRsc_allocate_mem on GPU 0 (flat device 1) returns a block that is ready
    when the call returns, as the reference's synchronous gpu_mem_alloc
    (mem_manager.cpp:779) is: a caller fills it at once from a stream of its own and
    reads it back, the library permutes into it, and tensDevRsc_free_mem takes it back
    only after the device has finished with it, over several allocate / free cycles."""
    import torch
    L = talsh
    pp = C.POINTER(T.DevRsc)()
    assert L.tensDevRsc_create(C.byref(pp)) == 0
    d = pp
    n = 1 << 20
    rng = np.random.default_rng(17)
    A = rand((128, 64, 128), T.R8, rng)
    src = torch.from_numpy(A.ravel(order="F").copy()).cuda()
    ref = O.permute(A, [3, 1, 2])
    side = torch.cuda.Stream()
    try:
        for it in range(4):
            assert L.tensDevRsc_allocate_mem(d, 1, n * 8, T.NOPE) == 0
            assert L.tensDevRsc_device_id(d) == 1
            g = C.c_void_p()
            assert L.tensDevRsc_get_gmem_ptr(d, C.byref(g)) == 0 and g.value
            blk = torch.as_tensor(_DeviceBlock(g.value, n), device="cuda")
            with torch.cuda.stream(side):
                blk.fill_(it + 0.5)
                assert bool((blk == it + 0.5).all().item())
            side.synchronize()
            s = torch.cuda.current_stream().cuda_stream
            assert L.tcTensorPermute(T.R8, 3, T.ivec([128, 64, 128]), T.ivec([3, 1, 2]), src.data_ptr(), g.value,
                                     0, s) == 0
            torch.cuda.synchronize()
            got = blk.cpu().numpy().reshape((64, 128, 128), order="F")
            assert same_bits(got, ref), it
            del blk
            assert L.tensDevRsc_free_mem(d) == 0 and L.tensDevRsc_is_empty(d) == T.YEP
    finally:
        L.tensDevRsc_release_all(d)
        assert L.tensDevRsc_destroy(d) == 0
