"""Oracle for the talsh-b200 hot path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over liboracle.so, the plain-C restatement of the reference
TAL-SH CPU path (see oracle.h for the reference file:line each routine
follows).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg import this package, as the checker or as the timed CPU baseline; the
product library never uses it.

Parity status: pinned.  The restatement is checked against every known answer
the reference's own tests and documents hold for this path (digital patterns
and matricizations quoted from the reference, the analytic norms of
test.cpp's test_talsh_c, the explicit-loop residual of test_nwchem_c, the
patterns of tensor_contractions.txt) and against numpy's independent einsum /
transpose (tests/test_oracle.py).  The reference's own CPU library is Fortran
and cannot be compiled here (no Fortran compiler in the image).
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
R4, R8, C4, C8 = 4, 8, 14, 18
NP_DTYPE = {R4: np.float32, R8: np.float64, C4: np.complex64, C8: np.complex128}
KIND_OF = {np.dtype(np.float32): R4, np.dtype(np.float64): R8,
           np.dtype(np.complex64): C4, np.dtype(np.complex128): C8}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from .build import build_oracle
            build_oracle()
        L = C.CDLL(LIB_PATH)
        P, I, D, V, Z = C.POINTER, C.c_int, C.c_double, C.c_void_p, C.c_size_t
        L.orc_str2dig.argtypes = [C.c_char_p, P(I), P(I), P(I), P(I), P(I)]
        L.orc_contraction_permutations.argtypes = [I, I, I, I, P(I), I, P(I), P(I), P(I), P(I), P(I), P(I), P(I)]
        L.orc_contr_permutations.argtypes = [I, I, I, I, P(I), I, P(I), P(I), P(I), P(I), P(I), P(I)]
        L.orc_permute.argtypes = [I, I, P(I), P(I), V, V, I]
        L.orc_permute_blocked.argtypes = [I, I, P(I), P(I), V, V, I]
        L.orc_tensor_copy.argtypes = [I, P(I), I, P(I), V, V, I]
        L.orc_tensor_add.argtypes = [I, P(I), I, P(I), V, V, D, D, I]
        L.orc_tensor_add_blocked.argtypes = [I, I, P(I), P(I), V, V, D, D, I]
        L.orc_tensor_scale.argtypes = [I, Z, V, D, D, I]
        L.orc_tensor_init.argtypes = [I, Z, V, D, D, I]
        L.orc_norm1.argtypes = [I, Z, V]
        L.orc_norm1.restype = D
        L.orc_tensor_contract.argtypes = [I, P(I), I, P(I), I, P(I), I, P(I), V, V, V, D, D, I, I]
        L.orc_cmplx8_to_real8.argtypes = [D, D]
        L.orc_cmplx8_to_real8.restype = D
        L.orc_fill_uniform.argtypes = [I, Z, V, C.c_ulonglong]
        L.orc_tensor_slice.argtypes = [I, I, P(I), P(I), P(I), V, V, I]
        L.orc_tensor_insert.argtypes = [I, I, P(I), P(I), P(I), V, V, I]
        _lib = L
    return _lib


def _iv(seq):
    seq = list(seq)
    return (C.c_int * max(1, len(seq)))(*seq)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def _fort(a):
    """Fortran-ordered view/copy that keeps 0-d arrays 0-d (np.asfortranarray would not)."""
    a = np.asarray(a)
    return a if a.flags["F_CONTIGUOUS"] else np.asfortranarray(a)


def str2dig(pattern):
    """Returns (errc, digital, drank, lrank, rrank, conj_bits)."""
    dig = (C.c_int * 256)()
    dr, lr, rr, cj = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    e = lib().orc_str2dig(pattern.encode(), dig, C.byref(dr), C.byref(lr), C.byref(rr), C.byref(cj))
    n = max(0, lr.value + rr.value) if e == 0 else 0
    return e, list(dig[:n]), dr.value, lr.value, rr.value, cj.value


def pattern_sym(cptrn, lrank, rrank, conj_bits=0):
    """Digital -> symbolic pattern: (ierr, string)."""
    buf = C.create_string_buffer(16 + 4 * (max(lrank, 0) + max(rrank, 0)))
    cpl = C.c_int()
    e = lib().orc_pattern_sym(lrank, rrank, conj_bits, _iv(list(cptrn) or [0]), buf, C.byref(cpl))
    return e, buf.raw[:cpl.value].decode("latin-1")


def permutations(cptrn, lrank, rrank, conj=0, variant="cpu", gemm_tl=1, gemm_tr=0):
    """Matricization: (ierr, dprm[1:], lprm[1:], rprm[1:], ncd, nlu, nru, nhu)."""
    a = _iv(cptrn)
    d, l, r = (C.c_int * 64)(), (C.c_int * 64)(), (C.c_int * 64)()
    ncd, nlu, nru, nhu = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    if variant == "cpu":
        e = lib().orc_contraction_permutations(gemm_tl, gemm_tr, lrank, rrank, a, conj, d, l, r,
                                               C.byref(ncd), C.byref(nlu), C.byref(nru), C.byref(nhu))
    else:
        e = lib().orc_contr_permutations(gemm_tl, gemm_tr, lrank, rrank, a, conj, d, l, r,
                                         C.byref(ncd), C.byref(nlu), C.byref(nru))
    dr = sum(1 for x in cptrn if x > 0) - nhu.value
    return e, list(d[1:1 + dr]), list(l[1:1 + lrank]), list(r[1:1 + rrank]), ncd.value, nlu.value, nru.value, nhu.value


def out_dims(dims_in, o2n):
    out = [0] * len(dims_in)
    for i, p in enumerate(o2n):
        out[p - 1] = dims_in[i]
    return out


def permute(a, o2n, conj=False, blocked=False, nthreads=1):
    """Returns permute(a) as a Fortran-ordered array; a is Fortran-ordered with dims a.shape."""
    a = _fort(a)
    dims = list(a.shape)
    out = np.empty(out_dims(dims, o2n), dtype=a.dtype, order="F")
    kind = KIND_OF[a.dtype]
    if blocked:
        e = lib().orc_permute_blocked(kind, len(dims), _iv(dims), _iv(o2n), _ptr(a), _ptr(out), nthreads)
    else:
        e = lib().orc_permute(kind, len(dims), _iv(dims), _iv(o2n), _ptr(a), _ptr(out), 1 if conj else 0)
    assert e == 0, e
    return out


def tensor_add(d, l, cptrn, sr=1.0, si=0.0, conj_bits=0):
    """In place: d += permute(l) * s (reference cpu_tensor_block_add)."""
    l = _fort(l)
    assert d.flags["F_CONTIGUOUS"] and d.dtype == l.dtype
    e = lib().orc_tensor_add(KIND_OF[d.dtype], _iv(cptrn), l.ndim, _iv(l.shape), _ptr(l), _ptr(d), sr, si, conj_bits)
    assert e == 0, e
    return d


def tensor_add_blocked(d, l, o2n, sr=1.0, si=0.0, nthreads=None):
    """In place: d += permute(l) * s through the reference's multi-threaded flow
    (blocked transpose into a temporary, then an OpenMP add); bit-identical to tensor_add."""
    l = _fort(l)
    assert d.flags["F_CONTIGUOUS"] and d.dtype == l.dtype
    e = lib().orc_tensor_add_blocked(KIND_OF[l.dtype], l.ndim, _iv(l.shape), _iv(o2n), _ptr(l), _ptr(d), sr, si,
                                     nthreads or os.cpu_count() or 1)
    assert e == 0, e


def contract_ttgt_blas(d, l, r, cptrn, sr=1.0, si=0.0, accumulative=True, nthreads=None):
    """In place on d: the reference CPU contraction as it runs with a BLAS library
    (tensor_block_contract, tensor_algebra_cpu.F90:3675-4358): L and R permuted by the
    CPU matricization (get_contraction_permutations, :5757-5956) with the cache-blocked
    transpose, D permuted unless its order is already the matrix order, one
    ?GEMM('T','N', ll, lr, lc, alpha, L, lc, R, lc, beta=1, D, ll) (:3987-4044, the call at
    :4005) from the BLAS scipy links (OpenBLAS, the reference's default BLASLIB), and the
    back-transpose.  No hyper-indices and no conjugation flags.  Returns seconds spent."""
    import time
    from scipy.linalg import blas
    nt = nthreads or os.cpu_count() or 1
    l, r = _fort(l), _fort(r)
    assert d.flags["F_CONTIGUOUS"] and d.dtype == l.dtype == r.dtype
    t0 = time.perf_counter()
    e, dprm, lprm, rprm, ncd, nlu, nru, nhu = permutations(cptrn, l.ndim, r.ndim, 0, "cpu")
    assert e == 0 and nhu == 0, (e, nhu)
    ident = lambda p: all(x == i + 1 for i, x in enumerate(p))
    lt = l if ident(lprm) else permute(l, lprm, blocked=True, nthreads=nt)
    rt = r if ident(rprm) else permute(r, rprm, blocked=True, nthreads=nt)
    lc = int(np.prod(lt.shape[:ncd], dtype=np.int64))
    ll = lt.size // max(1, lc)
    lr = rt.size // max(1, lc)
    if not accumulative:
        d[...] = 0
    dinv = [0] * len(dprm)
    for k, p in enumerate(dprm):
        dinv[p - 1] = k + 1
    dt = d if ident(dinv) else permute(d, dinv, blocked=True, nthreads=nt)
    A = lt.reshape((lc, ll), order="F")
    B = rt.reshape((lc, lr), order="F")
    Dm = dt.reshape((ll, lr), order="F")
    gemm = {np.dtype(np.float32): blas.sgemm, np.dtype(np.float64): blas.dgemm,
            np.dtype(np.complex64): blas.cgemm, np.dtype(np.complex128): blas.zgemm}[d.dtype]
    alpha = complex(sr, si) if np.iscomplexobj(d) else sr
    out = gemm(alpha, A, B, beta=1.0, c=Dm, trans_a=1, overwrite_c=1)
    if out is not Dm and not np.shares_memory(out, Dm):
        Dm[...] = out
    if dt is not d:
        e = lib().orc_permute_blocked(KIND_OF[d.dtype], dt.ndim, _iv(dt.shape), _iv(dprm), _ptr(dt), _ptr(d), nt)
        assert e == 0, e
    return time.perf_counter() - t0


def tensor_copy(d, l, cptrn, conj_bits=0):
    l = _fort(l)
    e = lib().orc_tensor_copy(KIND_OF[d.dtype], _iv(cptrn), l.ndim, _iv(l.shape), _ptr(l), _ptr(d), conj_bits)
    assert e == 0, e
    return d


def tensor_scale(d, sr, si=0.0, conj_bits=0):
    e = lib().orc_tensor_scale(KIND_OF[d.dtype], d.size, _ptr(d), sr, si, conj_bits)
    assert e == 0, e
    return d


def norm1(a):
    a = np.ascontiguousarray(a.ravel(order="F"))
    return lib().orc_norm1(KIND_OF[a.dtype], a.size, _ptr(a))


def tensor_contract(d, l, r, cptrn, sr=1.0, si=0.0, conj_bits=0, accumulative=True):
    """In place on d (Fortran-ordered): reference tensor_block_contract. Returns ierr."""
    l = _fort(l)
    r = _fort(r)
    assert d.flags["F_CONTIGUOUS"]
    return lib().orc_tensor_contract(KIND_OF[d.dtype], _iv(cptrn), d.ndim, _iv(d.shape), l.ndim, _iv(l.shape),
                                     r.ndim, _iv(r.shape), _ptr(d), _ptr(l), _ptr(r), sr, si, conj_bits,
                                     1 if accumulative else 0)


def tensor_slice(slice_, full, offsets, accumulative=False):
    """In place on slice_ (Fortran-ordered): reference tensor_block_slice. Returns ierr."""
    full = _fort(full)
    assert slice_.flags["F_CONTIGUOUS"] and slice_.ndim == full.ndim
    return lib().orc_tensor_slice(KIND_OF[full.dtype], full.ndim, _iv(full.shape), _iv(slice_.shape), _iv(offsets),
                                  _ptr(full), _ptr(slice_), 1 if accumulative else 0)


def tensor_insert(full, slice_, offsets, accumulative=False):
    """In place on full (Fortran-ordered): reference tensor_block_insert. Returns ierr."""
    slice_ = _fort(slice_)
    assert full.flags["F_CONTIGUOUS"] and slice_.ndim == full.ndim
    return lib().orc_tensor_insert(KIND_OF[full.dtype], full.ndim, _iv(full.shape), _iv(slice_.shape),
                                   _iv(offsets), _ptr(slice_), _ptr(full), 1 if accumulative else 0)


def cmplx8_to_real8(re, im):
    return lib().orc_cmplx8_to_real8(re, im)


def uniform(dims, kind, seed):
    """Seeded mt19937_64 uniform[-1,1] tensor (complex: re then im per element)."""
    n = int(np.prod(dims)) if len(dims) else 1
    a = np.empty(n, dtype=NP_DTYPE[kind])
    lib().orc_fill_uniform(kind, n, _ptr(a), seed)
    return a.reshape(dims, order="F") if len(dims) else a.reshape(())
