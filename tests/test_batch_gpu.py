"""Batched contractions (tcTensorContractBatch): every task equals the same
contraction run alone through tcTensorContract, and the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T
from gpu_util import fort, rel_err

pytestmark = pytest.mark.gpu

NPT = {T.R4: np.float32, T.R8: np.float64, T.C4: np.complex64, T.C8: np.complex128}
TOL = {T.R8: 1e-12, T.C8: 1e-12, T.R4: 2e-5, T.C4: 2e-5}


def random_task(rng, kind, emax=24, vmax=1 << 16):
    """Random contraction: L and R share nc contracted indices; D holds the rest in a random order."""
    while True:
        nc = int(rng.integers(1, 4))
        lu = int(rng.integers(0, 4))
        ru = int(rng.integers(0, 4))
        if nc + lu < 1 or nc + ru < 1:
            continue
        ext = [int(x) for x in np.exp(rng.uniform(np.log(4), np.log(emax), nc + lu + ru)).round()]
        c, l, r = list(range(nc)), list(range(nc, nc + lu)), list(range(nc + lu, nc + lu + ru))
        Lidx = list(rng.permutation(c + l))
        Ridx = list(rng.permutation(c + r))
        Didx = list(rng.permutation(l + r))
        vol = lambda idx: int(np.prod([ext[i] for i in idx])) if idx else 1
        if max(vol(Lidx), vol(Ridx), vol(Didx)) <= vmax:
            break
    cptrn = []
    for i in Lidx:
        cptrn.append(Didx.index(i) + 1 if i not in c else -(Ridx.index(i) + 1))
    for i in Ridx:
        cptrn.append(Didx.index(i) + 1 if i not in c else -(Lidx.index(i) + 1))
    dims = lambda idx: [ext[i] for i in idx]
    return dict(kind=kind, cptrn=cptrn, dd=dims(Didx), ld=dims(Lidx), rd=dims(Ridx))


def rnd(rng, dims, kind):
    x = rng.uniform(-1, 1, dims) if dims else np.asarray(rng.uniform(-1, 1))
    if kind in (T.C4, T.C8):
        x = x + 1j * (rng.uniform(-1, 1, dims) if dims else rng.uniform(-1, 1))
    return fort(np.asarray(x).astype(NPT[kind]))


def test_batch_matches_single_and_oracle(talsh):
    torch = pytest.importorskip("torch")
    lib = T.lib()
    rng = np.random.default_rng(2024)
    kinds = [T.R8] * 60 + [T.C8] * 40 + [T.R4] * 10 + [T.C4] * 10
    specs = [random_task(rng, k) for k in kinds]
    # two more full contractions (1 x 1 tiles in the batch) and a scalar-by-tensor task (single-task path)
    specs.append(dict(kind=T.R8, cptrn=[-2, -1, -2, -1], dd=[], ld=[9, 7], rd=[7, 9]))
    specs.append(dict(kind=T.C8, cptrn=[-1, -1], dd=[], ld=[33], rd=[33]))
    specs.append(dict(kind=T.R8, cptrn=[2, 1], dd=[5, 6], ld=[6, 5], rd=[]))
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    tasks = (T.ContractTask * len(specs))()
    keep, singles = [], []
    for t, sp in zip(tasks, specs):
        kind = sp["kind"]
        Lh, Rh, D0 = rnd(rng, sp["ld"], kind), rnd(rng, sp["rd"], kind), rnd(rng, sp["dd"], kind)
        acc = bool(rng.integers(0, 2))
        alpha = (0.5, 0.0) if kind in (T.R4, T.R8) else (0.5, -0.25)
        d, l, r, d1 = dev(D0), dev(Lh), dev(Rh), dev(D0)
        keep.append((sp, Lh, Rh, D0, acc, alpha, d, l, r, d1))
        t.data_kind, t.drank, t.lrank, t.rrank = kind, len(sp["dd"]), len(sp["ld"]), len(sp["rd"])
        for i, v in enumerate(sp["cptrn"]):
            t.cptrn[i] = v
        for arr, name in ((sp["dd"], "ddims"), (sp["ld"], "ldims"), (sp["rd"], "rdims")):
            for i, v in enumerate(arr):
                getattr(t, name)[i] = v
        t.D, t.L, t.R = d.data_ptr(), l.data_ptr(), r.data_ptr()
        t.alpha_re, t.alpha_im = alpha
        t.conj_bits, t.accumulative = 0, 1 if acc else 0
    need = lib.tcTensorContractBatchScratch(len(specs), tasks)
    assert need > 0
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    launches = lib.tcKernelLaunchCount()
    assert lib.tcTensorContractBatch(len(specs), tasks, scratch.data_ptr(), need, s) == 0, lib.tcLastErrorString()
    torch.cuda.synchronize()
    batched_launches = lib.tcKernelLaunchCount() - launches
    # tables + one launch per tile configuration (six) + the scalar-by-tensor task
    assert batched_launches <= 1 + 6 + 1
    for sp, Lh, Rh, D0, acc, alpha, d, l, r, d1 in keep:
        kind = sp["kind"]
        args = (kind, T.ivec(sp["cptrn"]), len(sp["dd"]), T.ivec(sp["dd"]), len(sp["ld"]), T.ivec(sp["ld"]),
                len(sp["rd"]), T.ivec(sp["rd"]))
        ns = lib.tcTensorContractScratch(*args)
        sc = torch.empty(max(ns, 1), dtype=torch.uint8, device="cuda")
        assert lib.tcTensorContract(*args, d1.data_ptr(), l.data_ptr(), r.data_ptr(), alpha[0], alpha[1], 0,
                                    1 if acc else 0, sc.data_ptr(), ns, s) == 0
        torch.cuda.synchronize()
        got, single = d.cpu().numpy(), d1.cpu().numpy()
        if sp["dd"]:  # same tile arithmetic as the single-task path (its full contraction is a two-pass dot)
            assert got.tobytes() == single.tobytes(), sp
        ref = D0.copy(order="F")
        assert O.tensor_contract(ref, Lh, Rh, sp["cptrn"], alpha[0], alpha[1], 0, acc) == 0
        assert rel_err(got.reshape(ref.shape, order="F"), ref) <= TOL[kind], sp


def test_batch_rejects_bad_tasks(talsh):
    lib = T.lib()
    tasks = (T.ContractTask * 1)()
    tasks[0].data_kind, tasks[0].drank, tasks[0].lrank, tasks[0].rrank = T.R8, 9, 1, 1
    assert lib.tcTensorContractBatchScratch(1, tasks) == 0
    assert lib.tcTensorContractBatch(1, tasks, None, 0, None) == T.TALSH_INVALID_ARGS
    assert lib.tcTensorContractBatch(0, tasks, None, 0, None) == 0


def test_operands_must_be_element_aligned(talsh):
    """Device operands aligned to less than their element size (an 8-byte
    aligned complex(8) tensor) are refused before any launch, alone and batched."""
    torch = pytest.importorskip("torch")
    lib = T.lib()
    rng = np.random.default_rng(21)
    sp = random_task(rng, T.C8)
    buf = torch.zeros(1 << 16, dtype=torch.float64, device="cuda")
    args = (T.C8, T.ivec(sp["cptrn"]), len(sp["dd"]), T.ivec(sp["dd"]), len(sp["ld"]), T.ivec(sp["ld"]),
            len(sp["rd"]), T.ivec(sp["rd"]))
    ns = lib.tcTensorContractScratch(*args)
    sc = torch.empty(max(ns, 1), dtype=torch.uint8, device="cuda")
    base = buf.data_ptr()
    for dp, lp, rp in ((base + 8, base + 4096, base + 8192), (base, base + 4104, base + 8192),
                       (base, base + 4096, base + 8200)):
        assert lib.tcTensorContract(*args, dp, lp, rp, 1.0, 0.0, 0, 0, sc.data_ptr(), ns, None) == \
            T.TALSH_INVALID_ARGS
        t = (T.ContractTask * 1)()
        x = t[0]
        x.data_kind, x.drank, x.lrank, x.rrank = T.C8, len(sp["dd"]), len(sp["ld"]), len(sp["rd"])
        for i, v in enumerate(sp["cptrn"]):
            x.cptrn[i] = v
        for arr, name in ((sp["dd"], "ddims"), (sp["ld"], "ldims"), (sp["rd"], "rdims")):
            for i, v in enumerate(arr):
                getattr(x, name)[i] = v
        x.D, x.L, x.R = dp, lp, rp
        assert lib.tcTensorContractBatchScratch(1, t) == 0
        assert lib.tcTensorContractBatch(1, t, sc.data_ptr(), 1 << 20, None) == T.TALSH_INVALID_ARGS


def test_autotune_chooses_tiles_and_keeps_results(talsh):
    """tcTensorContractBatchTune records a tile per class present; batches run
    afterwards still match tcTensorContract bit for bit (the tile does not change
    any element's summation order)."""
    torch = pytest.importorskip("torch")
    lib = T.lib()
    rng = np.random.default_rng(33)
    specs = [random_task(rng, T.R8 if i % 2 == 0 else T.C8, emax=40, vmax=1 << 15) for i in range(48)]
    s = torch.cuda.current_stream().cuda_stream

    def build(specs, seed):
        r = np.random.default_rng(seed)
        tasks = (T.ContractTask * len(specs))()
        keep = []
        for t, sp in zip(tasks, specs):
            kind = sp["kind"]
            def mk(d):
                x = r.uniform(-1, 1, d)
                if kind == T.C8:
                    x = x + 1j * r.uniform(-1, 1, d)
                return torch.from_numpy(fort(x.astype(NPT[kind])).ravel(order="F").copy()).cuda()
            l, rr, d = mk(sp["ld"]), mk(sp["rd"]), mk(sp["dd"] if sp["dd"] else [1])
            keep.append((sp, l, rr, d))
            t.data_kind, t.drank, t.lrank, t.rrank = kind, len(sp["dd"]), len(sp["ld"]), len(sp["rd"])
            for i, v in enumerate(sp["cptrn"]):
                t.cptrn[i] = v
            for arr, name in ((sp["dd"], "ddims"), (sp["ld"], "ldims"), (sp["rd"], "rdims")):
                for i, v in enumerate(arr):
                    getattr(t, name)[i] = v
            t.D, t.L, t.R = d.data_ptr(), l.data_ptr(), rr.data_ptr()
            t.alpha_re, t.alpha_im, t.conj_bits, t.accumulative = 0.5, 0.0, 0, 0
        return tasks, keep

    lib.tcTensorContractBatchTuneReset()
    try:
        tasks, keep = build(specs, 1)
        need = lib.tcTensorContractBatchScratch(len(specs), tasks)
        sc = torch.empty(need, dtype=torch.uint8, device="cuda")
        assert lib.tcTensorContractBatchTune(len(specs), tasks, sc.data_ptr(), need, s, 1) == 0
        tuned = [lib.tcTensorContractBatchTuned(k, mb, nb) for k in (T.R8, T.C8) for mb in range(4) for nb in range(4)]
        assert set(tuned) <= {0, 32, 64} and any(t in (32, 64) for t in tuned), tuned
        assert lib.tcTensorContractBatchTuned(T.R4, 0, 0) == -1
        # a fresh batch after tuning equals one tcTensorContract per task (the
        # scratch size depends on the tiles chosen: query it again)
        tasks, keep = build(specs, 2)
        need = lib.tcTensorContractBatchScratch(len(specs), tasks)
        sc = torch.empty(need, dtype=torch.uint8, device="cuda")
        assert lib.tcTensorContractBatch(len(specs), tasks, sc.data_ptr(), need, s) == 0
        torch.cuda.synchronize()
        for sp, l, r, d in keep:
            if not sp["dd"]:
                continue
            args = (sp["kind"], T.ivec(sp["cptrn"]), len(sp["dd"]), T.ivec(sp["dd"]), len(sp["ld"]),
                    T.ivec(sp["ld"]), len(sp["rd"]), T.ivec(sp["rd"]))
            d1 = torch.empty_like(d)
            ns = lib.tcTensorContractScratch(*args)
            s1 = torch.empty(max(ns, 1), dtype=torch.uint8, device="cuda")
            assert lib.tcTensorContract(*args, d1.data_ptr(), l.data_ptr(), r.data_ptr(), 0.5, 0.0, 0, 0,
                                        s1.data_ptr(), ns, s) == 0
            torch.cuda.synchronize()
            assert torch.equal(d1, d), sp
    finally:
        lib.tcTensorContractBatchTuneReset()
    assert all(lib.tcTensorContractBatchTuned(k, mb, nb) == 0 for k in (T.R8, T.C8) for mb in range(4)
               for nb in range(4))


def test_batch_graph_replays_equal_the_batch(talsh):
    """tcContractBatchGraph: descriptors and tables set up once, the GEMM work
    captured in one CUDA graph with the tile configurations as concurrent
    branches; every replay equals tcTensorContractBatch bit for bit, also after
    the operands' contents change between replays."""
    torch = pytest.importorskip("torch")
    lib = T.lib()
    rng = np.random.default_rng(77)
    kinds = [T.R8] * 30 + [T.C8] * 20 + [T.R4] * 6 + [T.C4] * 6
    specs = [random_task(rng, k) for k in kinds]
    specs.append(dict(kind=T.R8, cptrn=[2, 1], dd=[5, 6], ld=[6, 5], rd=[]))  # scalar operand: single-task path
    dev = lambda a: torch.from_numpy(np.asarray(a).ravel(order="F").copy()).cuda()
    s = torch.cuda.current_stream().cuda_stream

    def make(out):
        tasks = (T.ContractTask * len(specs))()
        for t, sp, (l, r, d) in zip(tasks, specs, out):
            t.data_kind, t.drank, t.lrank, t.rrank = sp["kind"], len(sp["dd"]), len(sp["ld"]), len(sp["rd"])
            for i, v in enumerate(sp["cptrn"]):
                t.cptrn[i] = v
            for arr, name in ((sp["dd"], "ddims"), (sp["ld"], "ldims"), (sp["rd"], "rdims")):
                for i, v in enumerate(arr):
                    getattr(t, name)[i] = v
            t.D, t.L, t.R = d.data_ptr(), l.data_ptr(), r.data_ptr()
            t.alpha_re, t.alpha_im = (0.5, 0.0) if sp["kind"] in (T.R4, T.R8) else (0.5, -0.25)
            t.conj_bits, t.accumulative = 0, 0
        return tasks

    ops = [(dev(rnd(rng, sp["ld"], sp["kind"])), dev(rnd(rng, sp["rd"], sp["kind"])),
            dev(rnd(rng, sp["dd"] if sp["dd"] else [1], sp["kind"]))) for sp in specs]
    ref_d = [torch.empty_like(d) for _, _, d in ops]
    tasks_g = make(ops)
    tasks_r = make([(l, r, d2) for (l, r, _), d2 in zip(ops, ref_d)])
    need = lib.tcTensorContractBatchScratch(len(specs), tasks_g)
    sc_g = torch.empty(need, dtype=torch.uint8, device="cuda")
    sc_r = torch.empty(need, dtype=torch.uint8, device="cuda")
    g = C.c_void_p()
    assert lib.tcContractBatchGraphCreate(len(specs), tasks_g, sc_g.data_ptr(), need, s, C.byref(g)) == 0, \
        lib.tcLastErrorString()
    try:
        for rep in range(3):
            if rep == 2:  # new operand contents, same buffers
                for l, r, _ in ops:
                    l.mul_(-1.5)
            assert lib.tcContractBatchGraphLaunch(g, s) == 0
            assert lib.tcTensorContractBatch(len(specs), tasks_r, sc_r.data_ptr(), need, s) == 0
            torch.cuda.synchronize()
            for sp, (_, _, d), d2 in zip(specs, ops, ref_d):
                assert torch.equal(d, d2), (rep, sp)
    finally:
        assert lib.tcContractBatchGraphDestroy(g) == 0
    bad = C.c_void_p()
    assert lib.tcContractBatchGraphCreate(0, tasks_g, sc_g.data_ptr(), need, s, C.byref(bad)) == T.TALSH_INVALID_ARGS
    assert lib.tcContractBatchGraphCreate(len(specs), tasks_g, sc_g.data_ptr(), 16, s, C.byref(bad)) == \
        T.TALSH_INVALID_ARGS
