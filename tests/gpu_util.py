"""Helpers for the GPU parity tests: run TAL-SH operations on GPU 0 over Host
tensors whose bodies are numpy arrays (caller memory attached with ext_mem)."""
import ctypes as C

import numpy as np

import oracle as O
import tal_sh_b200 as T


def fort(a):
    a = np.asarray(a)
    return a if a.flags["F_CONTIGUOUS"] else np.asfortranarray(a)


def rand(dims, kind, rng, scale=1.0):
    dt = T.NP_DTYPE[kind]
    x = rng.uniform(-1, 1, dims)
    if kind in (T.C4, T.C8):
        x = x + 1j * rng.uniform(-1, 1, dims)
    return fort(np.asarray(x * scale).astype(dt))


def host_tensor(arr):
    arr = fort(arr)
    return T.Tensor(list(arr.shape), T.KIND_OF[arr.dtype], dev_id=0, ext=arr)


def gpu_copy(pattern, D, L, coh=None):
    dt, lt = host_tensor(D), host_tensor(L)
    rc = T.lib().talshTensorCopy(pattern.encode(), dt.ref, lt.ref, 0, T.DEV_NVIDIA_GPU,
                                 T.COPY_TT if coh is None else coh, None)
    dt.destruct(); lt.destruct()
    return rc


def gpu_add(pattern, D, L, sr=1.0, si=0.0):
    dt, lt = host_tensor(D), host_tensor(L)
    rc = T.lib().talshTensorAdd(pattern.encode(), dt.ref, lt.ref, sr, si, 0, T.DEV_NVIDIA_GPU, T.COPY_TT, None)
    dt.destruct(); lt.destruct()
    return rc


def gpu_contract(pattern, D, L, R, sr=1.0, si=0.0, accumulative=True):
    dt, lt, rt = host_tensor(D), host_tensor(L), host_tensor(R)
    rc = T.lib().talshTensorContract(pattern.encode(), dt.ref, lt.ref, rt.ref, sr, si, 0, T.DEV_NVIDIA_GPU,
                                     T.COPY_TTT, T.YEP if accumulative else T.NOPE, None)
    dt.destruct(); lt.destruct(); rt.destruct()
    return rc


def rel_err(a, b):
    nb = np.linalg.norm(np.asarray(b, dtype=np.complex128).ravel())
    return np.linalg.norm((np.asarray(a, dtype=np.complex128) - np.asarray(b, dtype=np.complex128)).ravel()) / max(nb, 1e-300)


def same_bits(a, b):
    return fort(a).tobytes(order="F") == fort(b).tobytes(order="F")
