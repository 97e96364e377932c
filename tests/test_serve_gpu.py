"""Contraction server (tcServer*, talsh_b200.h) against the oracle: chains of
tasks through server-held outputs across the batch and large-task streams,
results identical alone and in a mix, admission under a device-memory budget,
error paths, and the arrival-replay loop."""
import ctypes as C
import re

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, rand

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12    # plain FP64 paths, relative Frobenius error
TOL_SPLIT6 = 1e-10  # split-precision R8 (6 slices)


def _labels(pattern):
    m = re.fullmatch(r"D\(([a-z,]*)\)\+?=L\(([a-z,]*)\)\*R\(([a-z,]*)\)", pattern)
    return [[x for x in g.split(",") if x] for g in m.groups()]


def _dims(pattern, ext):
    return [[ext[x] for x in g] for g in _labels(pattern)]


class _Dev:
    """Device memory as a numpy-shaped view (__cuda_array_interface__)."""

    def __init__(self, ptr, n, kind):
        ts = {T.R8: "<f8", T.C8: "<c16", T.R4: "<f4", T.C4: "<c8"}[kind]
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": ts, "data": (ptr, False), "version": 3}


def _task(kind, pattern, ext, L=0, R=0, D=0, l_from=0, r_from=0, consumers=0, keep=0, alpha=(1.0, 0.0), acc=0):
    e, dig, dr, lr, rr, _ = T.parse_pattern(pattern)
    dd, ld, rd = _dims(pattern, ext)
    st = T.ServeTask()
    t = st.op
    t.data_kind, t.drank, t.lrank, t.rrank = kind, len(dd), len(ld), len(rd)
    for i, v in enumerate(dig):
        t.cptrn[i] = v
    for arr, name in ((dd, "ddims"), (ld, "ldims"), (rd, "rdims")):
        for i, v in enumerate(arr):
            getattr(t, name)[i] = v
    t.D, t.L, t.R = D or None, L or None, R or None
    t.alpha_re, t.alpha_im = alpha
    t.conj_bits, t.accumulative = 0, acc
    st.l_from, st.r_from, st.consumers, st.keep_output = l_from, r_from, consumers, keep
    return st


class Server:
    def __init__(self, **cfg):
        self.L = T.lib()
        c = T.ServeConfig(**cfg)
        self.h = C.c_void_p()
        assert self.L.tcServerCreate(C.byref(c), C.byref(self.h)) == 0

    def submit(self, st):
        i = C.c_uint64(0)
        rc = self.L.tcServerSubmit(self.h, C.byref(st), C.byref(i))
        return rc, i.value

    def drain(self):
        assert self.L.tcServerDrain(self.h) == 0

    def poll(self):
        out = {}
        ids, lat, stt = (C.c_uint64 * 4096)(), (C.c_double * 4096)(), (C.c_int * 4096)()
        while True:
            n = self.L.tcServerPoll(self.h, 4096, ids, lat, stt)
            if n <= 0:
                return out
            for j in range(n):
                out[ids[j]] = (lat[j], stt[j])

    def stats(self):
        s = T.ServeStats()
        assert self.L.tcServerGetStats(self.h, C.byref(s)) == 0
        return s

    def close(self):
        assert self.L.tcServerDestroy(self.h) == 0


def _cuda(torch, a):
    a = np.asarray(a)
    return torch.from_numpy(a.ravel(order="F").copy()).cuda()


def _host(t, shape):
    return t.cpu().numpy().reshape(shape, order="F")


def _oracle(D, Lh, Rh, pattern, alpha=(1.0, 0.0), acc=False):
    e, dig, *_ = T.parse_pattern(pattern)
    assert O.tensor_contract(D, Lh, Rh, dig, alpha[0], alpha[1], 0, acc) == 0
    return D


def _rel(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


CHAIN = [  # (pattern, extents): t2 and t4 are large at large_flop=1e6, t1 small, t3 small for R8
    ("D(a,b)+=L(a,k)*R(k,b)", dict(a=20, k=30, b=25)),
    ("D(a,c)+=L(a,b)*R(b,c)", dict(a=20, b=25, c=2100)),
    ("D(c,d)+=L(a,c)*R(a,d)", dict(a=20, c=2100, d=5)),
    ("D(c,e)+=L(c,d)*R(d,e)", dict(c=2100, d=5, e=60)),
]


def _run_chain(torch, kind, slices, seed=0):
    rng = np.random.default_rng(seed)
    srv = Server(large_flop=1e6, r8_slices=slices)
    alpha = (0.5, 0.25) if kind == T.C8 else (0.5, 0.0)
    keep = []
    L1 = rand(_dims(*CHAIN[0])[1], kind, rng)
    Rs = [rand(_dims(p, e)[2], kind, rng) for p, e in CHAIN]
    D0 = rand(_dims(*CHAIN[3])[0], kind, rng)
    l1 = _cuda(torch, L1)
    rs = [_cuda(torch, r) for r in Rs]
    d4 = _cuda(torch, D0)
    keep += [l1, rs, d4]
    prev = 0
    for i, (p, e) in enumerate(CHAIN):
        last = i == len(CHAIN) - 1
        st = _task(kind, p, e, L=l1.data_ptr() if i == 0 else 0, R=rs[i].data_ptr(), l_from=prev,
                   D=d4.data_ptr() if last else 0, consumers=0 if last else 1,
                   alpha=alpha if last else (1.0, 0.0), acc=1 if last else 0)
        rc, prev = srv.submit(st)
        assert rc == 0, rc
    srv.drain()
    done = srv.poll()
    assert len(done) == 4 and all(s == 0 for _, s in done.values()), done
    st = srv.stats()
    n_large = 2 if kind == T.R8 else 3  # complex t3 counts 8 MNK = 1.68e6 flops
    assert st.large_tasks == n_large and st.batched_tasks == 4 - n_large and st.bytes_in_use == 0
    got = _host(d4, D0.shape)
    srv.close()
    # oracle chain
    x = L1
    for i, (p, e) in enumerate(CHAIN[:-1]):
        x = _oracle(fort(np.zeros(_dims(p, e)[0], dtype=L1.dtype)), x, Rs[i], p)
    ref = _oracle(D0.copy(order="F"), x, Rs[3], CHAIN[3][0], alpha, True)
    return _rel(got - D0, ref - D0)


@pytest.mark.parametrize("kind", [T.R8, T.C8])
def test_chain_across_streams_plain(talsh, kind):
    torch = pytest.importorskip("torch")
    assert _run_chain(torch, kind, 0) <= TOL_FP64


def test_chain_split_precision(talsh):
    torch = pytest.importorskip("torch")
    assert _run_chain(torch, T.R8, 6) <= TOL_SPLIT6


def _random_small(rng, kind):
    """A random small contraction (C4-like shapes, operands <= 2^15 elements)."""
    while True:
        nc = int(rng.integers(1, 3))
        lu, ru = int(rng.integers(0, 3)), int(rng.integers(1, 3))
        names = "abcdefgh"[: nc + lu + ru]
        ext = {x: int(rng.integers(2, 24)) for x in names}
        c, lo, ro = list(names[:nc]), list(names[nc:nc + lu]), list(names[nc + lu:])
        Li, Ri, Di = list(rng.permutation(c + lo)), list(rng.permutation(c + ro)), list(rng.permutation(lo + ro))
        pat = "D(%s)+=L(%s)*R(%s)" % (",".join(Di), ",".join(Li), ",".join(Ri))
        dd, ld, rd = _dims(pat, ext)
        if max(np.prod(dd), np.prod(ld), np.prod(rd)) <= 1 << 15:
            return pat, ext


def test_results_same_alone_and_in_mix(talsh):
    """Probe tasks give bit-identical results run alone and inside a mix of
    fillers (batches of other sizes, chains, a large task on the other stream)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    probes = []
    for i in range(16):
        kind = T.R8 if i % 2 == 0 else T.C8
        pat, ext = _random_small(rng, kind)
        dd, ld, rd = _dims(pat, ext)
        probes.append((kind, pat, ext, rand(ld, kind, rng), rand(rd, kind, rng), rand(dd, kind, rng)))
    big = ("D(a,c)+=L(a,b)*R(b,c)", dict(a=96, b=80, c=700))  # large at large_flop=1e6
    dd, ld, rd = _dims(*big)
    probes.append((T.R8, big[0], big[1], rand(ld, T.R8, rng), rand(rd, T.R8, rng), rand(dd, T.R8, rng)))
    dev = [(_cuda(torch, a), _cuda(torch, b)) for _, _, _, a, b, _ in probes]

    def probe_task(i, d):
        kind, pat, ext, _, _, _ = probes[i]
        return _task(kind, pat, ext, L=dev[i][0].data_ptr(), R=dev[i][1].data_ptr(), D=d.data_ptr(),
                     alpha=(0.75, -0.5) if kind == T.C8 else (0.75, 0.0), acc=1)

    alone = []
    for i, p in enumerate(probes):
        d = _cuda(torch, p[5])
        srv = Server(large_flop=1e6, r8_slices=6)
        assert srv.submit(probe_task(i, d))[0] == 0
        srv.drain()
        srv.close()
        alone.append(_host(d, p[5].shape))
    # the mix: fillers from a shared random pool, some chained, in random order
    pool = torch.empty(1 << 17, dtype=torch.float64, device="cuda").uniform_(-1, 1)
    srv = Server(large_flop=1e6, r8_slices=6, max_batch=64)
    mixd = [_cuda(torch, p[5]) for p in probes]
    order = list(range(len(probes)))
    rng.shuffle(order)
    prev = None
    for j in range(240):
        kind = T.R8 if j % 3 else T.C8
        if prev is not None and prev[0] == kind and j % 5 == 0:
            # chain: the filler's L is the previous filler's output
            pk, ppat, pext, pid = prev
            dd = _dims(ppat, pext)[0]
            names = "pqrstu"[: len(dd)]
            ext = dict(zip(names, dd))
            ext["z"] = max(1, min(7, (1 << 15) // int(np.prod(dd[1:]))))  # R stays inside the pool
            pat = "D(z,%s)+=L(%s)*R(%s,z)" % (names[0], ",".join(names), ",".join(names[1:]) or "")
            pat = pat.replace("R(,z)", "R(z)")
            st = _task(kind, pat, ext, R=pool.data_ptr(), l_from=pid)
            prev = None
        else:
            pat, ext = _random_small(rng, kind)
            st = _task(kind, pat, ext, L=pool.data_ptr(), R=pool.data_ptr() + 8 * (1 << 16), consumers=1)
        rc, fid = srv.submit(st)
        assert rc == 0, (rc, pat)
        if st.consumers:
            prev = (kind, pat, ext, fid)
        if j % 15 == 0 and order:
            i = order.pop()
            assert srv.submit(probe_task(i, mixd[i]))[0] == 0
        if j % 7 == 0:
            srv.L.tcServerProgress(srv.h)
    for i in order:
        assert srv.submit(probe_task(i, mixd[i]))[0] == 0
    srv.drain()
    st = srv.stats()
    assert st.failed == 0 and st.batches > 1 and st.large_tasks >= 1
    srv.close()
    for i, p in enumerate(probes):
        got = _host(mixd[i], p[5].shape)
        assert np.array_equal(got, alone[i]), (i, p[1])
        kind, pat, ext, Lh, Rh, D0 = p
        ref = _oracle(D0.copy(order="F"), Lh, Rh, pat, (0.75, -0.5) if kind == T.C8 else (0.75, 0.0), True)
        tol = TOL_SPLIT6 if i == len(probes) - 1 else TOL_FP64
        assert _rel(got - D0, ref - D0) <= tol, (i, pat)


def test_admission_under_budget(talsh):
    """Server-held intermediates under a 2 MiB budget: tasks wait at admission,
    the peak stays within the budget, every chain result is right."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(9)
    budget = 2 << 20
    srv = Server(budget_bytes=budget, max_batch=8)
    p1, e1 = "D(a,b)+=L(a,k)*R(k,b)", dict(a=256, k=16, b=256)  # 512 KiB intermediate
    p2, e2 = "D(a,c)+=L(a,b)*R(b,c)", dict(a=256, b=256, c=4)
    chains = []
    for i in range(12):
        Lh, R1 = rand(_dims(p1, e1)[1], T.R8, rng), rand(_dims(p1, e1)[2], T.R8, rng)
        R2 = rand(_dims(p2, e2)[2], T.R8, rng)
        l, r1, r2 = _cuda(torch, Lh), _cuda(torch, R1), _cuda(torch, R2)
        d = torch.zeros(256 * 4, dtype=torch.float64, device="cuda")
        rc, a = srv.submit(_task(T.R8, p1, e1, L=l.data_ptr(), R=r1.data_ptr(), consumers=1))
        assert rc == 0
        rc, b = srv.submit(_task(T.R8, p2, e2, R=r2.data_ptr(), l_from=a, D=d.data_ptr(), acc=0))
        assert rc == 0
        chains.append((Lh, R1, R2, l, r1, r2, d))
    srv.drain()
    st = srv.stats()
    assert st.failed == 0 and st.admission_waits > 0
    assert 0 < st.bytes_peak <= budget and st.bytes_in_use == 0
    srv.close()
    for Lh, R1, R2, l, r1, r2, d in chains:
        x = _oracle(fort(np.zeros((256, 256))), Lh, R1, p1)
        ref = _oracle(fort(np.zeros((256, 4))), x, R2, p2)
        assert _rel(_host(d, (256, 4)), ref) <= TOL_FP64


def test_keep_output_and_release(talsh):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    p, e = "D(a,b)+=L(a,k)*R(k,b)", dict(a=33, k=17, b=29)
    Lh, Rh = rand([33, 17], T.C8, rng), rand([17, 29], T.C8, rng)
    l, r = _cuda(torch, Lh), _cuda(torch, Rh)
    srv = Server()
    rc, i = srv.submit(_task(T.C8, p, e, L=l.data_ptr(), R=r.data_ptr(), keep=1))
    assert rc == 0
    srv.drain()
    ptr = C.c_void_p()
    assert srv.L.tcServerOutput(srv.h, i, C.byref(ptr)) == 0
    got = torch.as_tensor(_Dev(ptr.value, 33 * 29, T.C8), device="cuda").cpu().numpy().reshape((33, 29), order="F")
    ref = _oracle(fort(np.zeros((33, 29), dtype=np.complex128)), Lh, Rh, p)
    assert _rel(got, ref) <= TOL_FP64
    assert srv.stats().bytes_in_use > 0
    assert srv.L.tcServerRelease(srv.h, i) == 0
    torch.cuda.synchronize()
    assert srv.stats().bytes_in_use == 0
    srv.close()


def test_error_paths(talsh):
    torch = pytest.importorskip("torch")
    buf = torch.zeros(1 << 16, dtype=torch.float64, device="cuda")
    srv = Server(budget_bytes=1 << 20)
    p, e = "D(a,b)+=L(a,k)*R(k,b)", dict(a=600, k=2, b=600)  # 2.9 MB output > 1 MiB budget
    rc, big = srv.submit(_task(T.R8, p, e, L=buf.data_ptr(), R=buf.data_ptr(), consumers=1))
    assert rc == 0
    # consumer of a task that will fail
    rc, c = srv.submit(_task(T.R8, "D(a,c)+=L(a,b)*R(b,c)", dict(a=600, b=600, c=1), R=buf.data_ptr(), l_from=big,
                             D=buf.data_ptr()))
    assert rc == 0
    # shape mismatch with the producer, unknown producer, inconsistent extents: refused at submit
    assert srv.submit(_task(T.R8, "D(a,c)+=L(a,b)*R(b,c)", dict(a=5, b=600, c=1), R=buf.data_ptr(), l_from=big,
                            D=buf.data_ptr()))[0] == T.TALSH_INVALID_ARGS
    assert srv.submit(_task(T.R8, p, dict(a=4, k=4, b=4), R=buf.data_ptr(), l_from=987654))[0] == T.TALSH_INVALID_ARGS
    bad = _task(T.R8, p, dict(a=4, k=4, b=4), L=buf.data_ptr(), R=buf.data_ptr(), D=buf.data_ptr())
    bad.op.rdims[0] = 5  # contracted extents differ
    assert srv.submit(bad)[0] == T.TALSH_INVALID_ARGS
    srv.drain()
    done = srv.poll()
    assert done[big][1] == T.TALSH_LIMIT_EXCEEDED
    assert done[c][1] != 0
    assert srv.stats().failed == 2
    srv.close()


def test_replay_arrivals(talsh):
    """tcServerReplay: Poisson arrivals at 2000 tasks/s with chains; every task
    completes, latencies are positive, chain ends match the oracle."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(17)
    n = 300
    arr = (T.ServeTask * n)()
    keep, checks = [], []
    i = 0
    while i < n:
        p1, e1 = "D(a,b)+=L(a,k)*R(k,b)", dict(a=int(rng.integers(4, 40)), k=int(rng.integers(2, 30)),
                                                 b=int(rng.integers(4, 40)))
        Lh, R1 = rand(_dims(p1, e1)[1], T.R8, rng), rand(_dims(p1, e1)[2], T.R8, rng)
        l, r1 = _cuda(torch, Lh), _cuda(torch, R1)
        if i + 1 < n:
            p2, e2 = "D(b,c)+=L(a,b)*R(a,c)", dict(a=e1["a"], b=e1["b"], c=int(rng.integers(1, 9)))
            R2 = rand(_dims(p2, e2)[2], T.R8, rng)
            r2 = _cuda(torch, R2)
            d = torch.zeros(e2["b"] * e2["c"], dtype=torch.float64, device="cuda")
            arr[i] = _task(T.R8, p1, e1, L=l.data_ptr(), R=r1.data_ptr(), consumers=1)
            arr[i + 1] = _task(T.R8, p2, e2, R=r2.data_ptr(), l_from=i + 1, D=d.data_ptr())
            keep += [l, r1, r2, d]
            if len(checks) < 10:
                checks.append((Lh, R1, R2, d, p1, e1, p2, e2))
            i += 2
        else:
            d = torch.zeros(e1["a"] * e1["b"], dtype=torch.float64, device="cuda")
            arr[i] = _task(T.R8, p1, e1, L=l.data_ptr(), R=r1.data_ptr(), D=d.data_ptr())
            keep += [l, r1, d]
            i += 1
    arrivals = np.cumsum(rng.exponential(1 / 2000.0, n))
    ids, lat = (C.c_uint64 * n)(), (C.c_double * n)()
    srv = Server()
    rc = srv.L.tcServerReplay(srv.h, n, arr, (C.c_double * n)(*arrivals), ids, lat)
    assert rc == 0
    st = srv.stats()
    assert st.completed == n and st.failed == 0 and st.bytes_in_use == 0
    assert all(ids[j] > 0 for j in range(n)) and min(lat) > 0
    srv.close()
    for Lh, R1, R2, d, p1, e1, p2, e2 in checks:
        x = _oracle(fort(np.zeros(_dims(p1, e1)[0])), Lh, R1, p1)
        ref = _oracle(fort(np.zeros(_dims(p2, e2)[0])), x, R2, p2)
        assert _rel(_host(d, ref.shape), ref) <= TOL_FP64
