"""talsh-b200: a B200-native TAL-SH tensor-algebra core.

The product is the shared library ``libtalsh.so`` built from ``csrc/`` for
sm_100a; it exports the TAL-SH C API (``include/talsh.h``) and a device-level
C ABI (``include/talsh_b200.h``).  This module is the Python mirror of that
API: it loads the library with ctypes, declares the interoperable structs with
the reference layouts (talsh.h:84-121, tensor_algebra.h:205-249) and the
prototypes, and offers a thin ``Tensor`` helper.  There is no Python or CPU
fallback: if the library is missing, importing ``lib()`` raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtalsh.so")

# ---- constants (tensor_algebra.h / talsh.h) ----
NO_TYPE, R4, R8, C4, C8 = 0, 4, 8, 14, 18
DEV_NULL = DEV_DEFAULT = -1
DEV_HOST, DEV_NVIDIA_GPU, DEV_INTEL_MIC, DEV_AMD_GPU = 0, 1, 2, 3
MAX_TENSOR_RANK, MAX_TENSOR_OPERANDS = 56, 4
NOPE, YEP = 0, 1
TRY_LATER, DEVICE_UNABLE, NOT_CLEAN = -918273645, -546372819, -192837465
TALSH_SUCCESS, TALSH_FAILURE, TALSH_NOT_AVAILABLE, TALSH_NOT_IMPLEMENTED = 0, -666, -888, -999
TALSH_NOT_INITIALIZED, TALSH_ALREADY_INITIALIZED, TALSH_INVALID_ARGS = 1000000, 1000001, 1000002
TALSH_INTEGER_OVERFLOW, TALSH_OBJECT_NOT_EMPTY, TALSH_OBJECT_IS_EMPTY = 1000003, 1000004, 1000005
TALSH_IN_PROGRESS, TALSH_NOT_ALLOWED, TALSH_LIMIT_EXCEEDED = 1000006, 1000007, 1000008
TALSH_NOT_FOUND, TALSH_OBJECT_BROKEN, TALSH_INVALID_REQUEST = 1000009, 1000010, 1000011
TALSH_TASK_ERROR, TALSH_TASK_EMPTY, TALSH_TASK_SCHEDULED = 1999999, 2000000, 2000001
TALSH_TASK_STARTED, TALSH_TASK_INPUT_READY = 2000002, 2000003
TALSH_TASK_OUTPUT_READY, TALSH_TASK_COMPLETED = 2000004, 2000005
COPY_D, COPY_M, COPY_T, COPY_K = 0, 1, 2, 3
TC_SPLIT_INT8, TC_SPLIT_BF16, TC_SPLIT_TF32, TC_SPLIT_FP8 = 0, 1, 2, 3


def copy_ctrl(*codes):
    """Composite coherence code, e.g. copy_ctrl('M','T','T') == COPY_MTT == 26."""
    v = 0
    for c in codes:
        v = v * 4 + "DMTK".index(c)
    return v


for _a in "DMTK":
    for _b in "DMTK":
        globals()["COPY_" + _a + _b] = copy_ctrl(_a, _b)
        for _c in "DMTK":
            globals()["COPY_" + _a + _b + _c] = copy_ctrl(_a, _b, _c)
del _a, _b, _c

NP_DTYPE = {R4: np.float32, R8: np.float64, C4: np.complex64, C8: np.complex128}
KIND_OF = {np.dtype(np.float32): R4, np.dtype(np.float64): R8,
           np.dtype(np.complex64): C4, np.dtype(np.complex128): C8}


# ---- interoperable structs ----
class TensShape(C.Structure):
    _fields_ = [("num_dim", C.c_int), ("dims", C.POINTER(C.c_int)),
                ("divs", C.POINTER(C.c_int)), ("grps", C.POINTER(C.c_int))]


class DevRsc(C.Structure):
    _fields_ = [("dev_id", C.c_int), ("gmem_p", C.c_void_p), ("buf_entry", C.c_int),
                ("mem_attached", C.c_int)]


class Tens(C.Structure):
    _fields_ = [("shape_p", C.POINTER(TensShape)), ("dev_rsc", C.POINTER(DevRsc)),
                ("data_kind", C.POINTER(C.c_int)), ("avail", C.POINTER(C.c_int)),
                ("dev_rsc_len", C.c_int), ("ndev", C.c_int)]


class TensArg(C.Structure):
    _fields_ = [("tens_p", C.POINTER(Tens)), ("source_image", C.c_int)]


class Task(C.Structure):
    _fields_ = [("task_p", C.c_void_p), ("task_error", C.c_int), ("dev_kind", C.c_int),
                ("data_kind", C.c_int), ("coherence", C.c_int), ("num_args", C.c_int),
                ("tens_args", TensArg * MAX_TENSOR_OPERANDS), ("data_vol", C.c_double),
                ("flops", C.c_double), ("exec_time", C.c_double)]


TC_BATCH_MAX_RANK = 8


class ContractTask(C.Structure):
    """tcContractTask (talsh_b200.h): one contraction of a batch, device pointers."""
    _fields_ = [("data_kind", C.c_int), ("drank", C.c_int), ("lrank", C.c_int), ("rrank", C.c_int),
                ("cptrn", C.c_int * (2 * TC_BATCH_MAX_RANK)), ("ddims", C.c_int * TC_BATCH_MAX_RANK),
                ("ldims", C.c_int * TC_BATCH_MAX_RANK), ("rdims", C.c_int * TC_BATCH_MAX_RANK),
                ("D", C.c_void_p), ("L", C.c_void_p), ("R", C.c_void_p),
                ("alpha_re", C.c_double), ("alpha_im", C.c_double),
                ("conj_bits", C.c_int), ("accumulative", C.c_int)]


class PermuteTask(C.Structure):
    """tcPermuteTask (talsh_b200.h): one transpose of a graph-captured batch."""
    _fields_ = [("data_kind", C.c_int), ("rank", C.c_int), ("dims", C.c_int * TC_BATCH_MAX_RANK),
                ("o2n", C.c_int * TC_BATCH_MAX_RANK), ("src", C.c_void_p), ("dst", C.c_void_p),
                ("add", C.c_int), ("alpha_re", C.c_double), ("alpha_im", C.c_double), ("conj", C.c_int)]


class ServeConfig(C.Structure):
    """tcServeConfig (talsh_b200.h)."""
    _fields_ = [("budget_bytes", C.c_size_t), ("r8_slices", C.c_int), ("max_batch", C.c_int),
                ("max_inflight", C.c_int), ("large_flop", C.c_double), ("prealloc_bytes", C.c_size_t)]


class ServeTask(C.Structure):
    """tcServeTask (talsh_b200.h): a task for the contraction server."""
    _fields_ = [("op", ContractTask), ("l_from", C.c_uint64), ("r_from", C.c_uint64),
                ("consumers", C.c_int), ("keep_output", C.c_int)]


class ServeStats(C.Structure):
    """tcServeStats (talsh_b200.h)."""
    _fields_ = [("submitted", C.c_ulonglong), ("completed", C.c_ulonglong), ("failed", C.c_ulonglong),
                ("batches", C.c_ulonglong), ("batched_tasks", C.c_ulonglong), ("large_tasks", C.c_ulonglong),
                ("admission_waits", C.c_ulonglong), ("bytes_in_use", C.c_size_t), ("bytes_peak", C.c_size_t),
                ("budget_bytes", C.c_size_t), ("sched_s", C.c_double), ("max_step_s", C.c_double)]


_P = C.POINTER
_I, _D, _V, _S, _Z = C.c_int, C.c_double, C.c_void_p, C.c_char_p, C.c_size_t
_PROTOS = {
    "talshValidDataKind": (_I, [_I, _P(_I)]),
    "talshInit": (_I, [_P(_Z), _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I)]),
    "talshShutdown": (_I, []),
    "talshDeviceCount": (_I, [_I, _P(_I)]),
    "talshFlatDevId": (_I, [_I, _I]),
    "talshKindDevId": (_I, [_I, _P(_I)]),
    "talshDeviceBufferSize": (_Z, [_I, _I]),
    "talshDeviceBufferFreeSize": (_Z, [_I, _I]),
    "talshStats": (_I, [_I, _I]),
    "talshTensorCreate": (_I, [_P(_P(Tens))]),
    "talshTensorClean": (_I, [_P(Tens)]),
    "talshTensorIsEmpty": (_I, [_P(Tens)]),
    "talshTensorConstruct": (_I, [_P(Tens), _I, _I, _P(_I), _I, _V, _I, _V, _D, _D]),
    "talshTensorImportData": (_I, [_P(Tens), _I, _V]),
    "talshTensorDestruct": (_I, [_P(Tens)]),
    "talshTensorDestroy": (_I, [_P(Tens)]),
    "talshTensorRank": (_I, [_P(Tens)]),
    "talshTensorVolume": (_Z, [_P(Tens)]),
    "talshTensorPresence": (_I, [_P(Tens), _P(_I), _P(_I), _P(_I), _I, _I]),
    "talshTensorGetBodyAccess": (_I, [_P(Tens), _P(_V), _I, _I, _I]),
    "talshTensorGetScalar": (_I, [_P(Tens), _P(_D), _P(_D)]),
    "talshTensorInUse": (_I, [_P(Tens)]),
    "talshTaskCreate": (_I, [_P(_P(Task))]),
    "talshTaskClean": (_I, [_P(Task)]),
    "talshTaskIsEmpty": (_I, [_P(Task)]),
    "talshTaskDestruct": (_I, [_P(Task)]),
    "talshTaskDestroy": (_I, [_P(Task)]),
    "talshTaskStatus": (_I, [_P(Task)]),
    "talshTaskComplete": (_I, [_P(Task), _P(_I), _P(_I)]),
    "talshTaskWait": (_I, [_P(Task), _P(_I)]),
    "talshTaskTime": (_I, [_P(Task), _P(_D), _P(_D), _P(_D), _P(_D), _P(_D)]),
    "talshTensorPlace": (_I, [_P(Tens), _I, _I, _V, _I, _P(Task)]),
    "talshTensorDiscard": (_I, [_P(Tens), _I, _I]),
    "talshTensorDiscardOther": (_I, [_P(Tens), _I, _I]),
    "talshTensorInit": (_I, [_P(Tens), _D, _D, _I, _I, _I, _P(Task)]),
    "talshTensorScale": (_I, [_P(Tens), _D, _D, _I, _I, _I, _P(Task)]),
    "talshTensorSlice": (_I, [_P(Tens), _P(Tens), _P(_I), _I, _I, _I, _I, _P(Task)]),
    "talshTensorInsert": (_I, [_P(Tens), _P(Tens), _P(_I), _I, _I, _I, _I, _P(Task)]),
    "talshTensorCopy": (_I, [_S, _P(Tens), _P(Tens), _I, _I, _I, _P(Task)]),
    "talshTensorAdd": (_I, [_S, _P(Tens), _P(Tens), _D, _D, _I, _I, _I, _P(Task)]),
    "talshTensorContract": (_I, [_S, _P(Tens), _P(Tens), _P(Tens), _D, _D, _I, _I, _I, _I, _P(Task)]),
    "talshTensorContractXL": (_I, [_S, _P(Tens), _P(Tens), _P(Tens), _D, _D, _I, _I, _I]),
    "talshTensorImageNorm1_cpu": (_D, [_P(Tens)]),
    "talshTensorNorm1": (_D, [_P(Tens), _I, _I]),
    "talshContractSlicesSet": (_I, [_I]),
    "talshContractSlicesGet": (_I, []),
    "talshContractSplitFormSet": (_I, [_I, _I]),
    "talshContractSplitFormGet": (_I, [_P(_I), _P(_I)]),
    "talsh_get_contr_ptrn_str2dig": (_I, [_S, _P(_I), _P(_I), _P(_I), _P(_I), _P(_I)]),
    "get_contr_pattern_sym": (None, [_P(_I), _P(_I), _P(_I), _P(_I), C.c_char_p, _P(_I), _P(_I)]),
    "host_mem_register": (_I, [_V, _Z]),
    "host_mem_unregister": (_I, [_V]),
    "talsh_tensor_image_info": (_I, [_P(Tens), _I, _P(_I), _P(_I), _P(_V), _P(_I)]),
    "gpu_get_device_count": (_I, [_P(_I)]),
    "tensDevRsc_create": (_I, [_P(_P(DevRsc))]),
    "tensDevRsc_clean": (_I, [_P(DevRsc)]),
    "tensDevRsc_is_empty": (_I, [_P(DevRsc)]),
    "tensDevRsc_same": (_I, [_P(DevRsc), _P(DevRsc)]),
    "tensDevRsc_clone": (_I, [_P(DevRsc), _P(DevRsc)]),
    "tensDevRsc_attach_mem": (_I, [_P(DevRsc), _I, _V, _I]),
    "tensDevRsc_detach_mem": (_I, [_P(DevRsc)]),
    "tensDevRsc_allocate_mem": (_I, [_P(DevRsc), _I, _Z, _I]),
    "tensDevRsc_free_mem": (_I, [_P(DevRsc)]),
    "tensDevRsc_get_gmem_ptr": (_I, [_P(DevRsc), _P(_V)]),
    "tensDevRsc_device_id": (_I, [_P(DevRsc)]),
    "tensDevRsc_release_all": (_I, [_P(DevRsc)]),
    "tensDevRsc_destroy": (_I, [_P(DevRsc)]),
    "tensShape_create": (_I, [_P(_V)]),
    "tensShape_construct": (_I, [_V, _I, _I, _P(_I), _P(_I), _P(_I)]),
    "tensShape_volume": (_Z, [_V]),
    "tensShape_rank": (_I, [_V]),
    "tensShape_destroy": (_I, [_V]),
    "tensShape_reshape": (_I, [_V, _I, _P(_I), _P(_I), _P(_I)]),
    "tensShape_print": (None, [_V]),
    "tensSignature_create": (_I, [_P(_V)]),
    "tensSignature_clean": (_I, [_V]),
    "tensSignature_construct": (_I, [_V, _I, _P(_Z)]),
    "tensSignature_destruct": (_I, [_V]),
    "tensSignature_destroy": (_I, [_V]),
    "tens_elem_offset_f": (_Z, [C.c_uint, _P(C.c_uint), _P(C.c_uint)]),
    "fortran_cptr_int": (_Z, [_V]),
    "talshTensorSliceCreate": (_I, [_P(_V)]),
    "talshTensorSliceClean": (_I, [_V]),
    "talshTensorSliceConstruct": (_I, [_V, _P(Tens), _P(_Z), _P(_I), _P(_I), _P(_I)]),
    "talshTensorSliceVolume": (_Z, [_V]),
    "talshTensorSliceDestruct": (_I, [_V]),
    "talshTensorSliceDestroy": (_I, [_V]),
    "tens_elem_mlndx_f": (None, [_Z, C.c_uint, _P(C.c_uint), _P(C.c_uint)]),
    "get_contr_permutations": (None, [_I, _I, _I, _I, _P(_I), _I, _P(_I), _P(_I), _P(_I),
                                      _P(_I), _P(_I), _P(_I), _P(_I)]),
    "get_contraction_permutations": (None, [_I, _I, _I, _I, _P(_I), _I, _P(_I), _P(_I), _P(_I),
                                            _P(_I), _P(_I), _P(_I), _P(_I), _P(_I)]),
    "argument_coherence_get_value": (C.c_uint, [C.c_uint, C.c_uint, C.c_uint]),
    "argument_coherence_set_value": (_I, [_P(C.c_uint), C.c_uint, C.c_uint, C.c_uint]),
    "encode_device_id": (_I, [_I, _I]),
    "decode_device_id": (_I, [_I, _P(_I)]),
    "tcTensorPermute": (_I, [_I, _I, _P(_I), _P(_I), _V, _V, _I, _V]),
    "tcTensorPermuteAdd": (_I, [_I, _I, _P(_I), _P(_I), _V, _V, _D, _D, _I, _V]),
    "tcTensorPermuteTune": (_I, [_I, _I, _P(_I), _P(_I), _I, _V, _V, _V, _I, _P(_I)]),
    "tcTensorPermuteTuned": (_I, [_I, _I, _P(_I), _P(_I), _I, _P(_I)]),
    "tcTensorPermuteTuneSet": (_I, [_I, _I, _P(_I), _P(_I), _I, _I]),
    "tcTensorPermuteTuneReset": (None, []),
    "tcTensorInit": (_I, [_I, _Z, _V, _D, _D, _V]),
    "tcTensorScale": (_I, [_I, _Z, _V, _D, _D, _V]),
    "tcTensorNorm1Scratch": (_Z, [_Z]),
    "tcTensorNorm1": (_I, [_I, _Z, _V, _V, _V, _Z, _V]),
    "tcTensorContractScratch": (_Z, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I)]),
    "tcTensorContract": (_I, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I), _V, _V, _V, _D, _D,
                              _I, _I, _V, _Z, _V]),
    "tcTensorContractNoAlloc": (_I, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I), _V, _V, _V, _D,
                                     _D, _I, _I, _V]),
    "tcTensorContractNoAllocMaxScratch": (_Z, []),
    "tcTensorContractSplitScratch": (_Z, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I), _I]),
    "tcTensorContractBatchScratch": (_Z, [_I, _P(ContractTask)]),
    "tcTensorContractBatch": (_I, [_I, _P(ContractTask), _V, _Z, _V]),
    "tcContractBatchGraphCreate": (_I, [_I, _P(ContractTask), _V, _Z, _V, _P(_V)]),
    "tcContractBatchGraphLaunch": (_I, [_V, _V]),
    "tcContractBatchGraphDestroy": (_I, [_V]),
    "tcPermuteBatchCreate": (_I, [_I, _P(PermuteTask), _I, _P(_V)]),
    "tcPermuteBatchLaunch": (_I, [_V, _V]),
    "tcPermuteBatchDestroy": (_I, [_V]),
    "tcTensorContractBatchTune": (_I, [_I, _P(ContractTask), _V, _Z, _V, _I]),
    "tcTensorContractBatchTuned": (_I, [_I, _I, _I]),
    "tcTensorContractBatchTuneReset": (None, []),
    "tcContractXLLastOps": (_Z, []),
    "tcContractXLPlan": (_I, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I), _Z, _I, _P(_I), _P(_I)]),
    "tcTensorSlice": (_I, [_I, _I, _P(_I), _P(_I), _P(_I), _V, _V, _I, _V]),
    "tcTensorInsert": (_I, [_I, _I, _P(_I), _P(_I), _P(_I), _V, _V, _I, _V]),
    "tcServerCreate": (_I, [_P(ServeConfig), _P(_V)]),
    "tcServerDestroy": (_I, [_V]),
    "tcServerSubmit": (_I, [_V, _P(ServeTask), _P(C.c_uint64)]),
    "tcServerProgress": (_I, [_V]),
    "tcServerPoll": (_I, [_V, _I, _P(C.c_uint64), _P(_D), _P(_I)]),
    "tcServerDrain": (_I, [_V]),
    "tcServerOutput": (_I, [_V, C.c_uint64, _P(_V)]),
    "tcServerRelease": (_I, [_V, C.c_uint64]),
    "tcServerGetStats": (_I, [_V, _P(ServeStats)]),
    "tcServerResetStats": (_I, [_V]),
    "tcServerReplay": (_I, [_V, _I, _P(ServeTask), _P(_D), _P(C.c_uint64), _P(_D)]),
    "tcTensorContractSplit": (_I, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I), _V, _V, _V, _D, _D,
                                   _I, _I, _I, _V, _Z, _V]),
    "tcTensorContractSplitForm": (_I, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I), _V, _V, _V, _D, _D,
                                       _I, _I, _I, _I, _V, _Z, _V]),
    "tcTensorContractSplitFormScratch": (_Z, [_I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _P(_I), _I, _I]),
    "tcPermutePlanInfo": (_I, [_I, _I, _P(_I), _P(_I), _P(_I)]),
    "gpu_get_error_count": (_I, []),
    "tcTestSplitStall": (_I, [_I]),
    "tcKernelLaunchCount": (C.c_ulonglong, []),
    "tcLastErrorString": (_S, []),
}

_lib = None


def lib():
    """Loads libtalsh.so and returns the CDLL; raises RuntimeError when it has not been built
    (there is no fallback implementation)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "talsh-b200: %s is missing; build it with `python -m tal_sh_b200.build`" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def ivec(seq):
    """ctypes int array from a Python sequence (empty sequences give a 1-element array)."""
    seq = list(seq)
    arr = (C.c_int * max(1, len(seq)))(*seq)
    return arr


def pattern_sym(digital, lrank, rrank, conj_bits=0):
    """get_contr_pattern_sym: returns (ierr, symbolic pattern string)."""
    buf = C.create_string_buffer(16 + 4 * (max(lrank, 0) + max(rrank, 0)))
    cpl, ierr = C.c_int(0), C.c_int(0)
    lib().get_contr_pattern_sym(C.byref(C.c_int(lrank)), C.byref(C.c_int(rrank)), C.byref(C.c_int(conj_bits)),
                                ivec(digital), buf, C.byref(cpl), C.byref(ierr))
    return ierr.value, buf.raw[:cpl.value].decode("latin-1")


def parse_pattern(pattern):
    """talsh_get_contr_ptrn_str2dig: returns (errc, digital, drank, lrank, rrank, conj_bits)."""
    L = lib()
    dig = (C.c_int * (2 * MAX_TENSOR_RANK + 8))()
    dr, lr, rr, cj = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    e = L.talsh_get_contr_ptrn_str2dig(pattern.encode(), dig, C.byref(dr), C.byref(lr),
                                       C.byref(rr), C.byref(cj))
    n = max(0, lr.value + rr.value) if e == 0 else 0
    return e, list(dig[:n]), dr.value, lr.value, rr.value, cj.value


class Tensor:
    """Owns one talsh_tens_t (caller-owned object per the reference's rules)."""

    def __init__(self, dims, kind=R8, dev_id=0, ext=None, init=0.0, init_imag=0.0):
        self.L = lib()
        self.t = Tens()
        self._ext = ext  # keeps caller memory alive while attached
        self.dims = list(dims)
        self.kind = kind
        rc = self.L.talshTensorClean(C.byref(self.t))
        assert rc == 0
        ptr = None
        if ext is not None:
            assert ext.flags["F_CONTIGUOUS"] or ext.ndim <= 1
            ptr = ext.ctypes.data
        rc = self.L.talshTensorConstruct(C.byref(self.t), kind, len(self.dims), ivec(self.dims),
                                         dev_id, ptr, -1, None, init, init_imag)
        if rc != 0:
            raise RuntimeError("talshTensorConstruct failed: %d" % rc)

    @property
    def ref(self):
        return C.byref(self.t)

    def volume(self):
        return int(self.L.talshTensorVolume(self.ref))

    def host_array(self):
        """numpy view (Fortran order) of the Host image, or None."""
        for i in range(self.t.ndev):
            if self.t.dev_rsc[i].dev_id == 0:
                dt = NP_DTYPE[self.t.data_kind[i]]
                n = self.volume()
                buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(self.t.dev_rsc[i].gmem_p)
                a = np.frombuffer(buf, dtype=dt, count=n)
                return a.reshape(self.dims, order="F") if self.dims else a.reshape(())
        return None

    def images(self):
        return [(self.t.dev_rsc[i].dev_id, self.t.data_kind[i], self.t.avail[i]) for i in range(self.t.ndev)]

    def destruct(self):
        if self.t.shape_p:
            return self.L.talshTensorDestruct(self.ref)
        return 0
