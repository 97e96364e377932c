"""CPU-only checks of the drop-in boundary: libtalsh.so loads and exports every
function include/*.h declares; the product's pattern parser and permutation
solvers agree with the oracle; the runtime's host logic works without a GPU."""
import ctypes as C
import itertools
import json
import os
import random
import re

import numpy as np
import pytest

import oracle as O
import tal_sh_b200 as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"^\s*#[^\n]*", "", text, flags=re.M)
    text = re.sub(r"typedef[^;]*;", "", text)
    names = set()
    for m in re.finditer(r"([A-Za-z_]\w*)\s*\(([^;{}]*)\)\s*;", text):
        if m.group(1) not in ("TALSH_DEFAULT", "int", "void", "double", "size_t"):
            names.add(m.group(1))
    return names


@pytest.mark.parametrize("header", ["talsh.h", "tensor_algebra.h", "talsh_b200.h", "mem_manager.h"])
def test_library_exports_every_declared_symbol(built, header):
    L = T.lib()
    names = declared_functions(os.path.join(ROOT, "include", header))
    assert len(names) >= (2 if header == "mem_manager.h" else 6)  # the declaration scan found them
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_headers_compile_as_c_and_cpp(built, tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "talsh.h"\n#include "talsh_b200.h"\n#include "mem_manager.h"\n'
                   'int main(void){talsh_tens_t t; talshTensorClean(&t); return 0;}\n')
    import subprocess
    for cc, ext in (("gcc", "c"), ("g++", "cpp")):
        f = tmp_path / ("t." + ext)
        f.write_text(src.read_text())
        subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-c", str(f), "-o", str(tmp_path / ("t_" + ext + ".o"))],
                       check=True)


def test_struct_layouts_match_reference_abi():
    # talsh.h:87-94 and :110-121 on LP64
    assert C.sizeof(T.Tens) == 40
    assert C.sizeof(T.DevRsc) == 24
    assert C.sizeof(T.Task) == 8 + 4 * 5 + 4 + 16 * 4 + 24


def _pattern_corpus():
    g = json.load(open(os.path.join(GOLD, "tensor_contractions.json")))
    pats = [c["pattern"] for c in g]
    pats += ["D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", "D(i,c,a,b)=L(a,b,c,i)", "D(a,a)+=L(a)*R(a)", "D(a)+=L(a,b)",
             "D(a,,b)+=L(a,b)", "D+(a)+=L(a,b)*R+(b)", "D(a,b)+=L(a,b)*2.0", "D()=L()", "X(a|b)+=Y(b|a)",
             "D(a,b)+=L(a,c)*R(c,b)*S(d)", "D(a,b+)+=L(b+,a)", "D(a,b", "D(1a,b2)=L(b2,1a)", "D(a)+=L(a)*R(a)",
             "D(a,b)+=L(a,c,c)*R(b)", "", "*", "D(a)*3", "D(a)+=L(a)*R()*", "  D(a)=L(a)  ", "D(a_b)=L(a_b)",
             "D(a,b)+=L+(a,c)*R(c,b)", "D(ab,cd)+=L(cd,ef)*R(ef,ab)", "D(a)+=L(a,b)*R(b)*2", "D(a)+=L(a,b)*R(c)"]
    rng = random.Random(7)
    for _ in range(300):  # random well-formed and perturbed patterns
        labels = list("abcdefghij")
        rng.shuffle(labels)
        nd, nc = rng.randint(0, 4), rng.randint(0, 3)
        dl, cl = labels[:nd], labels[nd:nd + nc]
        split = rng.randint(0, nd)
        lidx, ridx = dl[:split] + cl, dl[split:] + cl
        rng.shuffle(lidx)
        rng.shuffle(ridx)
        p = "D(%s)+=L%s(%s)*R%s(%s)" % (",".join(dl), rng.choice(["", "+"]), ",".join(lidx),
                                           rng.choice(["", "+"]), ",".join(ridx))
        if rng.random() < 0.3:
            i = rng.randrange(len(p))
            p = p[:i] + rng.choice(["a", ",", ")", "(", "+", "*", "|"]) + p[i + 1:]
        pats.append(p)
    return pats


def test_parser_matches_oracle(built):
    for p in _pattern_corpus():
        assert T.parse_pattern(p) == O.str2dig(p), p


def _product_permutations(fn, cptrn, lr, rr, conj, tl=1, tr=0):
    L = T.lib()
    d, l, r = (C.c_int * 64)(), (C.c_int * 64)(), (C.c_int * 64)()
    ncd, nlu, nru, nhu, ierr = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
    if fn == "cpu":
        L.get_contraction_permutations(tl, tr, lr, rr, T.ivec(cptrn), conj, d, l, r, C.byref(ncd), C.byref(nlu),
                                       C.byref(nru), C.byref(nhu), C.byref(ierr))
    else:
        L.get_contr_permutations(tl, tr, lr, rr, T.ivec(cptrn), conj, d, l, r, C.byref(ncd), C.byref(nlu),
                                 C.byref(nru), C.byref(ierr))
    dr = sum(1 for x in cptrn if x > 0) - nhu.value
    return ierr.value, list(d[1:1 + dr]), list(l[1:1 + lr]), list(r[1:1 + rr]), ncd.value, nlu.value, nru.value, nhu.value


def test_permutation_solvers_match_oracle(built):
    for p in _pattern_corpus():
        e, dig, dr, lr, rr, cj = O.str2dig(p)
        if e != 0:
            continue
        for conj in {0, cj, 2, 4, 1}:
            for tl, tr in ((1, 0), (0, 0), (1, 1)):
                a = _product_permutations("cpu", dig, lr, rr, conj, tl, tr)
                b = O.permutations(dig, lr, rr, conj, "cpu", tl, tr)
                assert a[0] == b[0] and (a[0] != 0 or a == b), (p, conj, a, b)
                a = _product_permutations("gpu", dig, lr, rr, conj, tl, tr)
                b = O.permutations(dig, lr, rr, conj, "gpu", tl, tr)
                assert (a[0] != 0) == (b[0] != 0) and (a[0] != 0 or a == b), (p, conj, a, b)


def test_device_id_codec_and_coherence(built):
    L = T.lib()
    k = C.c_int()
    assert L.encode_device_id(T.DEV_HOST, 0) == 0
    assert L.encode_device_id(T.DEV_NVIDIA_GPU, 3) == 4
    assert L.decode_device_id(4, C.byref(k)) == 3 and k.value == T.DEV_NVIDIA_GPU
    assert L.decode_device_id(0, C.byref(k)) == 0 and k.value == T.DEV_HOST
    assert L.talshFlatDevId(T.DEV_NVIDIA_GPU, 8) == 25  # DEV_MAX: out of range
    assert T.COPY_MTT == 26 and T.COPY_TT == 10
    for coh in range(64):
        vals = [L.argument_coherence_get_value(coh, 3, i) for i in range(3)]
        assert vals == [(coh >> 4) & 3, (coh >> 2) & 3, coh & 3]
        c = C.c_uint(0)
        for i, v in enumerate(vals):
            assert L.argument_coherence_set_value(C.byref(c), 3, i, v) == 0
        assert c.value == coh


def test_host_runtime_without_gpu(built):
    """Host-side object logic with no GPU in the session: construction, queries,
    Host 1-norm, and every compute request refused (no CPU compute path)."""
    L = T.lib()
    hb, ha = C.c_size_t(0), C.c_int(0)
    assert L.talshInit(C.byref(hb), C.byref(ha), 0, None, 0, None, 0, None) == 0
    try:
        assert L.talshInit(C.byref(hb), C.byref(ha), 0, None, 0, None, 0, None) == T.TALSH_ALREADY_INITIALIZED
        d = T.Tensor([3, 4, 5], T.R8, dev_id=0, init=0.5)
        assert d.volume() == 60 and L.talshTensorRank(d.ref) == 3
        assert np.all(d.host_array() == 0.5)
        assert L.talshTensorImageNorm1_cpu(d.ref) == pytest.approx(30.0)
        ext = np.asfortranarray(np.arange(12, dtype=np.complex128).reshape(3, 4, order="F") * (1 - 1j))
        c = T.Tensor([3, 4], T.C8, dev_id=0, ext=ext)
        assert L.talshTensorImageNorm1_cpu(c.ref) == pytest.approx(np.abs(ext).sum())
        body = C.c_void_p()
        assert L.talshTensorGetBodyAccess(c.ref, C.byref(body), T.C8, 0, T.DEV_HOST) == 0
        assert body.value == ext.ctypes.data
        n, copies, kinds = C.c_int(), (C.c_int * 16)(), (C.c_int * 16)()
        assert L.talshTensorPresence(c.ref, C.byref(n), copies, kinds, T.DEV_NULL, -1) == 0
        assert n.value == 1 and copies[0] == 0 and kinds[0] == T.C8
        l = T.Tensor([5, 3, 4], T.R8, dev_id=0, init=1.0)
        assert L.talshTensorAdd(b"D(a,b,c)+=L(c,a,b)", d.ref, l.ref, 1.0, 0.0, 0, T.DEV_HOST, T.COPY_MT, None) == T.TALSH_NOT_AVAILABLE
        assert L.talshTensorAdd(b"D(a,b,c)+=L(c,a,b)", d.ref, l.ref, 1.0, 0.0, -1, -1, T.COPY_MT, None) == T.TALSH_NOT_AVAILABLE
        assert L.talshTensorAdd(b"D(a,b,c)+=L(c,a,b", d.ref, l.ref, 1.0, 0.0, -1, -1, T.COPY_MT, None) == T.TALSH_INVALID_ARGS
        assert L.talshTensorNorm1(d.ref, -1, -1) == -1.0
        assert L.talshTensorContract(b"D(a,b,c)+=L(c,a,b)*R()", d.ref, l.ref, l.ref, 1.0, 0.0, 0, T.DEV_HOST,
                                     T.COPY_MTT, T.YEP, None) == T.TALSH_INVALID_ARGS  # rank mismatch of R
        sc = T.Tensor([], T.R8, dev_id=0, init=2.5)
        re_, im_ = C.c_double(), C.c_double()
        assert L.talshTensorGetScalar(sc.ref, C.byref(re_), C.byref(im_)) == 0 and re_.value == 2.5
        task = T.Task()
        assert L.talshTaskClean(C.byref(task)) == 0 and L.talshTaskIsEmpty(C.byref(task)) == T.YEP
        assert L.talshTaskStatus(C.byref(task)) == T.TALSH_TASK_EMPTY
        for t in (d, c, l, sc):
            assert t.destruct() == 0
        assert L.talshTensorIsEmpty(d.ref) == T.YEP
    finally:
        assert L.talshShutdown() == 0
    assert L.talshShutdown() == T.TALSH_NOT_INITIALIZED


def test_batch_and_serve_struct_layouts_match_c(built, tmp_path):
    """ctypes mirrors of tcContractTask / tcServe* agree with the C compiler's layout."""
    import subprocess
    fields = {"tcContractTask": (T.ContractTask, ["D", "L", "R", "alpha_re", "conj_bits", "accumulative"]),
              "tcPermuteTask": (T.PermuteTask, ["o2n", "src", "dst", "add", "alpha_re", "conj"]),
              "tcServeTask": (T.ServeTask, ["op", "l_from", "r_from", "consumers", "keep_output"]),
              "tcServeConfig": (T.ServeConfig, ["budget_bytes", "r8_slices", "max_batch", "max_inflight",
                                                "large_flop", "prealloc_bytes"]),
              "tcServeStats": (T.ServeStats, ["submitted", "admission_waits", "bytes_in_use", "budget_bytes",
                                               "max_step_s"])}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "talsh_b200.h"', "int main(void){"]
    for name, (_, fs) in fields.items():
        lines.append('printf("%%zu\\n", sizeof(%s));' % name)
        for f in fs:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (name, f))
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for name, (cls, fs) in fields.items():
        want.append(C.sizeof(cls))
        want += [getattr(cls, f).offset for f in fs]
    assert got == want


def test_batch_planner_on_the_host(built):
    """tcTensorContractBatchScratch plans on the host (no GPU): the scratch grows
    with the tasks, and bad tasks -- an invalid pattern, a pointer not aligned to
    the element size -- make the whole batch unplannable (0 bytes)."""
    L = T.lib()

    def task(kind, pattern, dd, ld, rd, ptr=1 << 20):
        e, dig, dr, lr, rr, _ = T.parse_pattern(pattern)
        t = T.ContractTask()
        t.data_kind, t.drank, t.lrank, t.rrank = kind, len(dd), len(ld), len(rd)
        for i, v in enumerate(dig):
            t.cptrn[i] = v
        for arr, name in ((dd, "ddims"), (ld, "ldims"), (rd, "rdims")):
            for i, v in enumerate(arr):
                getattr(t, name)[i] = v
        t.D, t.L, t.R = ptr, ptr + (1 << 20), ptr + (2 << 20)
        t.alpha_re = 1.0
        return t

    a = task(T.R8, "D(a,b)+=L(a,k)*R(k,b)", [40, 30], [40, 20], [20, 30])
    b = task(T.C8, "D(a,b,c)+=L(c,a)*R(b,c)", [4, 5, 6], [6, 4], [5, 6])  # hyper: single-task path inside
    one = (T.ContractTask * 1)(a)
    two = (T.ContractTask * 2)(a, b)
    s1, s2 = L.tcTensorContractBatchScratch(1, one), L.tcTensorContractBatchScratch(2, two)
    assert 0 < s1 < s2
    assert s1 >= 8 * 2 * (40 + 30 + 20)  # the offset tables at least
    bad = task(T.R8, "D(a,b)+=L(a,k)*R(k,b)", [40, 30], [40, 21], [20, 30])  # contracted extents differ
    assert L.tcTensorContractBatchScratch(2, (T.ContractTask * 2)(a, bad)) == 0
    mis = task(T.C8, "D(a,b)+=L(a,k)*R(k,b)", [4, 3], [4, 2], [2, 3], ptr=(1 << 20) + 8)  # 8-byte aligned complex
    assert L.tcTensorContractBatchScratch(1, (T.ContractTask * 1)(mis)) == 0


def test_contract_flop_count(tmp_path):
    """The core's flop count of a contraction (task flops, the server's large-task
    threshold) is 2 (8 complex) times the product of the extents of the distinct
    indices of L and R: a hyper index (in D, L and R) counts once."""
    import subprocess
    cases = [("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=6, b=7, i=4, j=5, k=3, c=8), O.R8),
             ("D(x,y,z)+=L(x,y,k)*R(k,z)", dict(x=64, y=48, z=40, k=32), O.C8),
             ("D(a,b,c)+=L(c,a)*R(b,c)", dict(a=3, b=4, c=5), O.R8),
             ("D(i,j,k)+=L(k,a,i,b)*R(b,k,a,j)", dict(i=12, j=10, k=7, a=6, b=5), O.C4),
             ("D(x,h,g)+=L(x,h,k,g)*R(g,k,h)", dict(h=4, g=3, x=33, k=17), O.R4),
             ("D(h)+=L(k,h)*R(h,k)", dict(h=9, k=40), O.R8),
             ("D()+=L(a,b)*R(b,a)", dict(a=4, b=5), O.R8),
             ("D(a,b)+=L(a)*R(b)", dict(a=4, b=5), O.R8),
             ("D(b,a)+=L()*R(a,b)", dict(a=3, b=4), O.R8),
             ("D()+=L()*R()", dict(), O.C8)]
    body, want = [], []
    for n, (pat, ext, kind) in enumerate(cases):
        e, dig, dr, lr, rr, _ = O.str2dig(pat)
        assert e == 0
        groups = [[x for x in g.split(",") if x] for g in re.findall(r"\(([^)]*)\)", pat)]
        ld, rd = [ext[x] for x in groups[1]], [ext[x] for x in groups[2]]
        arr = lambda v: "{%s}" % ",".join(str(x) for x in (list(v) or [0]))
        body.append("{ const int c[] = %s, l[] = %s, r[] = %s; std::printf(\"%%.17g\\n\", "
                    "tb::contract_flops(%d, c, %d, l, %d, r)); }"
                    % (arr(dig[:lr + rr]), arr(ld), arr(rd), kind, lr, rr))
        labels = set(groups[1]) | set(groups[2])
        want.append((8.0 if kind in (O.C4, O.C8) else 2.0) * float(np.prod([ext[x] for x in labels])))
    src = tmp_path / "flops.cpp"
    src.write_text('#include <cstdio>\n#include "common.h"\nint main() {\n%s\nreturn 0; }\n' % "\n".join(body))
    exe = tmp_path / "flops"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I",
                    os.path.join(ROOT, "tal_sh_b200", "csrc"), str(src), "-o", str(exe)], check=True)
    got = [float(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == want


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without the built library the package raises instead of falling back."""
    monkeypatch.setattr(T, "_lib", None)
    monkeypatch.setattr(T, "LIB_PATH", str(tmp_path / "libtalsh.so"))
    with pytest.raises(RuntimeError, match="missing"):
        T.lib()


SPLIT_COMPLEX_CASES = [
    ("D(a,b)+=L(a,k)*R(k,b)", dict(a=5, b=4, k=6)),
    ("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)", dict(a=3, b=4, c=2, i=3, j=2, k=5)),
    ("D(i,a)+=L(k,a,j)*R(j,i,k)", dict(a=7, i=3, j=4, k=2)),
    ("D(a,b,c)+=L(c,a)*R(b,c)", dict(a=3, b=4, c=5)),  # hyper index: the rewrite keeps it (the split form refuses it)
]


@pytest.mark.parametrize("pattern,ext", SPLIT_COMPLEX_CASES)
def test_complex_split_rewrite_matches_oracle(tmp_path, pattern, ext):
    """The real form of a complex contraction that the split-precision form runs
    (split_complex.h): L and D read as real tensors with a leading (re, im) index,
    R's conjugated and i-rotated copies (alpha folded in) stacked along a trailing
    index.  The oracle's real contraction of the rewritten problem equals its
    complex contraction of the original, for every conjugation flag."""
    import subprocess
    e, dig, dr, lr, rr, _ = O.str2dig(pattern)
    assert e == 0
    groups = [[x for x in g.split(",") if x] for g in re.findall(r"\(([^)]*)\)", pattern)]
    dd, ld, rd = ([ext[x] for x in g] for g in groups)
    arr = lambda v: "{%s}" % ",".join(str(x) for x in (list(v) or [0]))
    body = []
    for conj in range(8):
        body.append("{ const int c[] = %s, d[] = %s, l[] = %s, r[] = %s; tb::ComplexSplitForm f;"
                    " int rc = tb::complex_split_form(c, %d, d, %d, l, %d, r, %d, f);"
                    " std::printf(\"%%d %%d %%d %%d %%d %%g %%d\", rc, f.drank, f.lrank, f.rrank, f.y_conj, f.z_im,"
                    " f.alpha_conj);"
                    " for (int i = 0; i < f.lrank + f.rrank; ++i) std::printf(\" %%d\", f.cptrn[i]);"
                    " for (int i = 0; i < f.drank; ++i) std::printf(\" %%d\", f.ddims[i]);"
                    " for (int i = 0; i < f.lrank; ++i) std::printf(\" %%d\", f.ldims[i]);"
                    " for (int i = 0; i < f.rrank; ++i) std::printf(\" %%d\", f.rdims[i]);"
                    " std::printf(\"\\n\"); }" % (arr(dig[:lr + rr]), arr(dd), arr(ld), arr(rd), dr, lr, rr, conj))
    src = tmp_path / "cs.cpp"
    src.write_text('#include <cstdio>\n#include "split_complex.h"\nint main() {\n%s\nreturn 0; }\n' % "\n".join(body))
    exe = tmp_path / "cs"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I",
                    os.path.join(ROOT, "tal_sh_b200", "csrc"), str(src), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    rng = np.random.default_rng(17)
    cplx = lambda s: np.asfortranarray(rng.standard_normal(s) + 1j * rng.standard_normal(s))
    L, R, D0 = cplx(ld), cplx(rd), cplx(dd)
    alpha = (0.75, -0.5)
    as_real = lambda X: np.frombuffer(np.asarray(X).tobytes(order="F"), dtype=np.float64).reshape(
        [2] + list(X.shape), order="F")
    for conj, line in enumerate(lines):
        v = [float(x) for x in line.split()]
        rc, fdr, flr, frr, yconj, zim, aconj = (int(v[0]), int(v[1]), int(v[2]), int(v[3]), int(v[4]), v[5],
                                                int(v[6]))
        assert rc == 0 and (fdr, flr, frr) == (dr + 1, lr + 1, rr + 2)
        rest = [int(x) for x in v[7:]]
        fdig, rest = rest[:flr + frr], rest[flr + frr:]
        fdd, rest = rest[:fdr], rest[fdr:]
        fld, frd = rest[:flr], rest[flr:]
        assert fdd == [2] + dd and fld == [2] + ld and frd == [2] + rd + [2]
        a = complex(*alpha).conjugate() if aconj else complex(*alpha)
        Y = np.conj(R) if yconj else R
        Rx = np.asfortranarray(np.stack([Y * a, Y * (1j * zim * a)], axis=-1))
        Dr = np.asfortranarray(as_real(D0).copy(order="F"))
        assert O.tensor_contract(Dr, as_real(L), as_real(Rx), fdig, 1.0, 0.0, 0, True) == 0
        got = np.frombuffer(Dr.tobytes(order="F"), dtype=np.complex128).reshape(dd, order="F")
        ref = D0.copy(order="F")
        assert O.tensor_contract(ref, L, R, dig, alpha[0], alpha[1], conj, True) == 0
        assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref - D0), (pattern, conj)


def test_complex_split_host_checks(built):
    """Host side of the complex(8) split-precision form, without a GPU: its scratch
    is the stacked operand (2 vol(R) complex elements, 256-byte rounded) plus the
    scratch of the rewritten real contraction; hyper-indices, rank-0 operands and
    complex(4) are refused before anything is launched."""
    L = T.lib()
    e, dig, dr, lr, rr, _ = T.parse_pattern("D(a,b,i,j)+=L(a,k,c,i)*R(c,b,k,j)")
    dd, ld, rd = [3, 4, 3, 2], [3, 5, 2, 3], [2, 4, 5, 2]
    args = (T.ivec(dig), dr, T.ivec(dd), lr, T.ivec(ld), rr, T.ivec(rd))
    shift = lambda v: v + 1 if v > 0 else v - 1
    fdig = [-1] + [shift(v) for v in dig[:lr]] + [-1] + [shift(v) for v in dig[lr:lr + rr]] + [1]
    for slices in (3, 6):
        real = L.tcTensorContractSplitScratch(T.R8, T.ivec(fdig), dr + 1, T.ivec([2] + dd), lr + 1,
                                              T.ivec([2] + ld), rr + 2, T.ivec([2] + rd + [2]), slices)
        rx = (2 * int(np.prod(rd)) * 16 + 255) // 256 * 256
        assert real > 0 and L.tcTensorContractSplitScratch(T.C8, *args, slices) == real + rx
    assert L.tcTensorContractSplit(T.C8, *args, None, None, None, 1.0, 0.0, 0, 1, 6, None, 0, None) == \
        T.TALSH_INVALID_ARGS
    assert L.tcTensorContractSplit(T.C8, *args, None, None, None, 1.0, 0.0, 0, 1, 9, None, 0, None) == \
        T.TALSH_INVALID_ARGS
    assert L.tcTensorContractSplitScratch(T.C4, *args, 6) == 0
    assert L.tcTensorContractSplit(T.C4, *args, None, None, None, 1.0, 0.0, 0, 1, 6, None, 0, None) == \
        T.TALSH_NOT_IMPLEMENTED
    e, hd, hdr, hlr, hrr, _ = T.parse_pattern("D(a,b,c)+=L(c,a)*R(b,c)")
    hargs = (T.ivec(hd), hdr, T.ivec([3, 4, 5]), hlr, T.ivec([5, 3]), hrr, T.ivec([4, 5]))
    assert L.tcTensorContractSplitScratch(T.C8, *hargs, 6) == 0
    assert L.tcTensorContractSplit(T.C8, *hargs, None, None, None, 1.0, 0.0, 0, 1, 6, None, 0, None) == \
        T.TALSH_NOT_IMPLEMENTED
    e, sd, sdr, slr, srr, _ = T.parse_pattern("D()+=L(a,b)*R(b,a)")
    sargs = (T.ivec(sd), sdr, T.ivec([]), slr, T.ivec([4, 5]), srr, T.ivec([5, 4]))
    assert L.tcTensorContractSplitScratch(T.C8, *sargs, 6) == 0
    assert L.tcTensorContractSplit(T.C8, *sargs, None, None, None, 1.0, 0.0, 0, 1, 6, None, 0, None) == \
        T.TALSH_NOT_IMPLEMENTED


def test_transpose_plan_invariants(built):
    """The transpose planner (host only) over thousands of random shapes: every tile
    fits the per-thread register tables (at most 8 elements per thread of a
    256-thread CTA, 4 for complex(8)), the tile splits into whole input runs and whole
    output runs, vector accesses are at most 16 bytes, the tiles cover the tensor,
    and identity permutations become a straight copy."""
    L = T.lib()
    rng = np.random.default_rng(2024)
    esize = {T.R4: 4, T.R8: 8, T.C4: 8, T.C8: 16}
    info = (C.c_int * 12)()
    n_tiled = 0
    for it in range(3000):
        kind = [T.R4, T.R8, T.C4, T.C8][it % 4]
        rank = int(rng.integers(1, 7))
        dims = [int(x) for x in rng.choice([1, 2, 3, 5, 7, 16, 17, 31, 32, 64, 97, 100, 128, 333], size=rank)]
        while np.prod(dims, dtype=np.int64) > 1 << 31:
            dims[int(np.argmax(dims))] //= 2
        o2n = [int(x) + 1 for x in rng.permutation(rank)]
        assert L.tcPermutePlanInfo(kind, rank, T.ivec(dims), T.ivec(o2n), info) == 0, (kind, dims, o2n)
        vol = int(np.prod(dims, dtype=np.int64))
        assert 0 <= info[0] <= rank
        if o2n == list(range(1, rank + 1)):
            assert info[1] == 1, (dims, o2n)
        if info[1]:
            continue
        n_tiled += 1
        V, Li, Lo, Ri, Ro, vin, vout, smem, ntiles = (info[i] for i in range(2, 11))
        per_thread = 4 if kind == T.C8 else 8
        assert 1 <= V <= 256 * per_thread, (kind, dims, o2n, V)
        assert Li * Ri == V and Lo * Ro == V, (dims, o2n, V, Li, Ri, Lo, Ro)
        assert vin >= 1 and vout >= 1 and vin * esize[kind] <= 16 and vout * esize[kind] <= 16
        assert 0 < smem <= 227 * 1024
        assert ntiles >= 1 and ntiles * V >= vol, (dims, o2n, ntiles, V)
    assert n_tiled > 1000


def test_contraction_scratch_queries_on_malformed_and_valid_patterns(built):
    """Host-side pattern analysis without a GPU: random (mostly malformed) digital
    patterns are analysed without crashing; valid random contractions get
    scratch for the plain and the split forms, except hyper-indices in the split form."""
    L = T.lib()
    rng = np.random.default_rng(0)
    for it in range(5000):
        kind = [T.R4, T.R8, T.C4, T.C8][it % 4]
        lr, rr, dr = (int(x) for x in rng.integers(0, 5, size=3))
        cp = [int(x) for x in rng.integers(-5, 6, size=lr + rr)]
        args = (T.ivec(cp), dr, T.ivec(rng.integers(1, 5, size=dr)), lr, T.ivec(rng.integers(1, 5, size=lr)),
                rr, T.ivec(rng.integers(1, 5, size=rr)))
        L.tcTensorContractScratch(kind, *args)
        L.tcTensorContractSplitScratch(kind, *args, 6)
    for it in range(400):
        nc, lu, ru = int(rng.integers(1, 3)), int(rng.integers(1, 3)), int(rng.integers(1, 3))
        hyper = it % 4 == 3
        names = "abcdefgh"[: nc + lu + ru + (1 if hyper else 0)]
        c, lo, ro = list(names[:nc]), list(names[nc:nc + lu]), list(names[nc + lu:nc + lu + ru])
        h = [names[-1]] if hyper else []
        Li, Ri = list(rng.permutation(c + lo + h)), list(rng.permutation(c + ro + h))
        Di = list(rng.permutation(lo + ro + h))
        pat = "D(%s)+=L(%s)*R(%s)" % (",".join(Di), ",".join(Li), ",".join(Ri))
        ext = {x: int(rng.integers(2, 9)) for x in names}
        e, dig, dr, lr, rr, _ = T.parse_pattern(pat)
        assert e == 0, pat
        args = (T.ivec(dig), dr, T.ivec([ext[x] for x in Di]), lr, T.ivec([ext[x] for x in Li]), rr,
                T.ivec([ext[x] for x in Ri]))
        for kind in (T.R8, T.C8):
            assert L.tcTensorContractScratch(kind, *args) > 0, pat
            split = L.tcTensorContractSplitScratch(kind, *args, 6)
            assert (split == 0) if hyper else (split > 0), (pat, kind)
        assert L.tcTensorContractSplitScratch(T.R4, *args, 6) == 0


def test_complex_split_rank_limit(built):
    """An R operand of rank 55 would need rank 57 in the complex form's real
    contraction (MAX_TENSOR_RANK is 56): the split form does not apply (0 bytes),
    the plain form and the R8 split form still do."""
    L = T.lib()
    rank_r = 55
    dig = [rank_r, -1] + [-2] + list(range(1, rank_r))   # D(r1..r54, a) += L(a, k) * R(k, r1..r54)
    dd, ld, rd = [1] * (rank_r - 1) + [3], [3, 2], [2] + [1] * (rank_r - 1)
    args = (T.ivec(dig), rank_r, T.ivec(dd), 2, T.ivec(ld), rank_r, T.ivec(rd))
    assert L.tcTensorContractScratch(T.C8, *args) > 0
    assert L.tcTensorContractSplitScratch(T.C8, *args, 6) == 0
    assert L.tcTensorContractSplitScratch(T.R8, *args, 6) > 0


def test_pattern_sym_matches_oracle_and_round_trips(built):
    """get_contr_pattern_sym, the digital -> symbolic direction used by the
    reference's C++ layer: the known form of the reference test's digital pattern,
    the rank-0 forms, equality with the oracle's restatement on random (often
    malformed) digital patterns, and symbolic -> digital round trips."""
    g = json.load(open(os.path.join(GOLD, "patterns.json")))["nvtal_digital"]
    assert T.pattern_sym(g["digital"], g["lrank"], g["rrank"]) == (0, "D(a,b,c,d)+=L(d,c,e,f)*R(b,a,e,f)")
    assert T.pattern_sym([], 0, 0) == (0, "D()+=L()*R()")
    assert T.pattern_sym([], 0, 0, 7) == (0, "D+()+=L+()*R+()")
    assert T.pattern_sym([1, 2], 2, 0, 2) == (0, "D(a,b)+=L+(a,b)*R()")
    assert T.pattern_sym([1], -1, 0)[0] == 1
    rng = np.random.default_rng(9)
    for _ in range(3000):
        lr, rr = int(rng.integers(0, 6)), int(rng.integers(0, 6))
        dig = [int(x) for x in rng.integers(-5, 6, size=lr + rr)]
        cj = int(rng.integers(0, 8))
        got, ref = T.pattern_sym(dig, lr, rr, cj), O.pattern_sym(dig, lr, rr, cj)
        assert got == ref, (dig, lr, rr, cj, got, ref)
    for _ in range(500):
        nc, lu, ru = (int(x) for x in rng.integers(0, 5, size=3))
        names = "abcdefghijklmnopqrstuvwxyz"[: nc + lu + ru]
        c, lo, ro = list(names[:nc]), list(names[nc:nc + lu]), list(names[nc + lu:])
        Li, Ri, Di = list(rng.permutation(c + lo)), list(rng.permutation(c + ro)), list(rng.permutation(lo + ro))
        cj = int(rng.integers(0, 8))
        mark = lambda name, bit: name + ("+" if cj & bit else "")
        pat = "%s(%s)+=%s(%s)*%s(%s)" % (mark("D", 1), ",".join(Di), mark("L", 2), ",".join(Li), mark("R", 4),
                                         ",".join(Ri))
        e, dig, dr, lr, rr, conj = T.parse_pattern(pat)
        assert e == 0, pat
        ierr, sym = T.pattern_sym(dig, lr, rr, conj)
        assert ierr == 0
        assert T.parse_pattern(sym) == (0, dig, dr, lr, rr, conj), (pat, sym)


def test_host_mem_register_without_gpu(built):
    """Pinning caller memory (mem_manager.h, for the reference's C++ layer) reports
    a CUDA failure as 1 with its text kept, as the reference does; here there is no
    device, so both calls fail cleanly."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present; tests/test_runtime_gpu.py covers this")
    L = T.lib()
    buf = (C.c_double * 1024)()
    assert L.host_mem_register(C.cast(buf, C.c_void_p), C.sizeof(buf)) == 1
    assert b"host_mem_register" in L.tcLastErrorString()
    assert L.host_mem_unregister(C.cast(buf, C.c_void_p)) == 1


def _reference_tree():
    """Location of the reference sources, as the fixture generator finds them
    (None where they are absent)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLD, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.REF if os.path.isdir(mod.REF) else None


def test_reference_cpp_layer_links_against_the_library(built, tmp_path):
    """The reference's C++ layer (talshxx.hpp/.cpp, talsh_task.hpp/.cpp), compiled
    with this core's include/ in place of the reference's own C headers, links
    against libtalsh.so with no undefined symbol.  Skipped where the reference
    sources are absent."""
    import subprocess
    ref = _reference_tree()
    if ref is None or not os.path.exists(os.path.join(ref, "talshxx.cpp")):
        pytest.skip("reference sources not present")
    objs = []
    for name in ("talshxx", "talsh_task"):
        obj = tmp_path / (name + ".o")
        # -I- : quoted includes of the reference files resolve in include/ first
        subprocess.run(["g++", "-std=c++14", "-fPIC", "-w", "-c", "-I", os.path.join(ROOT, "include"), "-I-",
                        "-I", ref, os.path.join(ref, name + ".cpp"), "-o", str(obj)], check=True)
        objs.append(str(obj))
    subprocess.run(["g++", "-shared", "-o", str(tmp_path / "libtalshxx.so"), *objs, "-L",
                    os.path.join(ROOT, "tal_sh_b200"), "-ltalsh", "-Wl,--no-undefined"], check=True)


# Calls of the reference test driver's test_nvtal_c into the reference's internal
# GPU layer (device_algebra.h, its argument buffers in mem_manager.h), which this
# core replaces with the device ABI of talsh_b200.h instead of reproducing.
NVTAL_INTERNAL = ["arg_buf_allocate", "arg_buf_deallocate", "cuda_task_create", "cuda_task_destroy",
                  "cuda_task_print", "cuda_task_time", "cuda_task_wait", "gpu_print_stats",
                  "gpu_tensor_block_contract_dlf", "tensBlck_attach_body", "tensBlck_construct", "tensBlck_create",
                  "tensBlck_destroy", "tensBlck_init_host", "tensBlck_norm2_host", "tensBlck_volume"]


def test_reference_test_driver_links_against_the_library(built, tmp_path):
    """The reference's own test driver (test.cpp: test_talsh_c, _cxx, _xl, _hyper,
    _svd, _qc, _nwchem, ...) with its C++ layer, compiled against include/, links
    against libtalsh.so with nothing undefined except test_nvtal_c's internal-layer
    calls (stubbed here).  Skipped where the reference sources are absent."""
    import subprocess
    ref = _reference_tree()
    if ref is None or not os.path.exists(os.path.join(ref, "test.cpp")):
        pytest.skip("reference sources not present")
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    shim = tmp_path / "nvtal_decl.h"
    shim.write_text('#include <stddef.h>\nextern "C" int arg_buf_allocate(size_t *, int *, int, int);\n'
                    'extern "C" int arg_buf_deallocate(int, int);\n')
    stub = tmp_path / "nvtal_stub.c"
    stub.write_text("".join("int %s(void) { return -1; }\n" % n for n in NVTAL_INTERNAL))
    objs = []
    for name in ("test", "talshxx", "talsh_task"):
        obj = tmp_path / (name + ".o")
        subprocess.run(["g++", "-std=c++14", "-fPIC", "-w", "-c", "-include", str(shim), "-I",
                        os.path.join(ROOT, "include"), "-I-", "-I", ref, "-I", cuda_inc,
                        os.path.join(ref, name + ".cpp"), "-o", str(obj)], check=True)
        objs.append(str(obj))
    subprocess.run(["gcc", "-fPIC", "-c", str(stub), "-o", str(tmp_path / "stub.o")], check=True)
    subprocess.run(["g++", "-shared", "-o", str(tmp_path / "libdriver.so"), *objs, str(tmp_path / "stub.o"), "-L",
                    os.path.join(ROOT, "tal_sh_b200"), "-ltalsh", "-lm", "-Wl,--no-undefined"], check=True)


def test_fortran_bound_entry_points_without_gpu(built):
    """talsh_tensor_image_info and gpu_get_device_count, which the reference's
    Fortran module binds: image information of a Host tensor, refusal of a
    missing image, and a GPU count that reports failure without a device."""
    L = T.lib()
    hb, ha = C.c_size_t(0), C.c_int(0)
    assert L.talshInit(C.byref(hb), C.byref(ha), 0, None, 0, None, 0, None) == 0
    try:
        ext = np.asfortranarray(np.arange(12.0).reshape(3, 4, order="F"))
        t = T.Tensor([3, 4], T.R8, dev_id=0, ext=ext)
        dev, kind, ptr, buf = C.c_int(), C.c_int(), C.c_void_p(), C.c_int()
        args = (C.byref(dev), C.byref(kind), C.byref(ptr), C.byref(buf))
        assert L.talsh_tensor_image_info(t.ref, 0, *args) == 0
        assert (dev.value, kind.value, ptr.value) == (0, T.R8, ext.ctypes.data)
        assert L.talsh_tensor_image_info(t.ref, 1, *args) == T.TALSH_INVALID_ARGS
        assert t.destruct() == 0
        assert L.talsh_tensor_image_info(t.ref, 0, *args) == T.TALSH_OBJECT_IS_EMPTY
    finally:
        assert L.talshShutdown() == 0
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        n = C.c_int(7)
        assert L.gpu_get_device_count(C.byref(n)) == 1 and n.value == -1


def test_fortran_module_imports_are_exported(built):
    """Every C function the reference's Fortran module (talshf.F90) declares in its
    interface blocks is exported by libtalsh.so, so the module links against it.
    Skipped where the reference sources are absent."""
    ref = _reference_tree()
    if ref is None or not os.path.exists(os.path.join(ref, "talshf.F90")):
        pytest.skip("reference sources not present")
    text = open(os.path.join(ref, "talshf.F90")).read()
    imports = set()
    for block in re.findall(r"^\s*interface\s*$(.*?)^\s*end\s+interface", text, flags=re.M | re.S | re.I):
        imports |= set(re.findall(r"bind\s*\(\s*c\s*,\s*name\s*=\s*'(\w+)'", block, flags=re.I))
    assert len(imports) > 40
    L = T.lib()
    missing = sorted(n for n in imports if not hasattr(L, n))
    assert not missing, missing


def test_device_resource_api_without_gpu(built):
    """The device-resource descriptor API (reference tensor_algebra_gpu.cpp:278-555)
    on the Host, with the reference's return codes: attach / compare / clone /
    detach of caller memory, allocate / free of library memory, refusals."""
    L = T.lib()
    pp = C.POINTER(T.DevRsc)()
    assert L.tensDevRsc_create(C.byref(pp)) == 0
    d = pp
    assert L.tensDevRsc_is_empty(d) == T.YEP and L.tensDevRsc_device_id(d) == T.DEV_NULL
    buf = (C.c_double * 64)()
    addr = C.cast(buf, C.c_void_p).value
    assert L.tensDevRsc_attach_mem(d, -1, addr, -1) == -2
    assert L.tensDevRsc_attach_mem(d, 0, None, -1) == -3
    assert L.tensDevRsc_attach_mem(d, 0, addr, -1) == 0
    assert L.tensDevRsc_is_empty(d) == T.NOPE and L.tensDevRsc_device_id(d) == 0
    assert L.tensDevRsc_attach_mem(d, 0, addr, -1) == 2      # memory present already
    assert L.tensDevRsc_attach_mem(d, 1, addr, -1) == 1      # bound to another device
    g = C.c_void_p()
    assert L.tensDevRsc_get_gmem_ptr(d, C.byref(g)) == 0 and g.value == addr
    other = T.DevRsc()
    assert L.tensDevRsc_clean(C.byref(other)) == 0 and L.tensDevRsc_same(d, C.byref(other)) == T.NOPE
    assert L.tensDevRsc_clone(d, C.byref(other)) == 0 and L.tensDevRsc_same(d, C.byref(other)) == T.YEP
    assert L.tensDevRsc_free_mem(d) == 1                     # attached, not allocated
    assert L.tensDevRsc_detach_mem(d) == 0 and L.tensDevRsc_is_empty(d) == T.YEP
    assert L.tensDevRsc_detach_mem(d) == -2
    assert L.tensDevRsc_get_gmem_ptr(d, C.byref(g)) == 1
    assert L.tensDevRsc_allocate_mem(d, 0, 0, T.NOPE) == -3
    assert L.tensDevRsc_allocate_mem(d, 0, 4096, T.NOPE) == 0
    assert L.tensDevRsc_get_gmem_ptr(d, C.byref(g)) == 0 and g.value
    C.memset(g.value, 0, 4096)                                # the Host block is usable
    assert L.tensDevRsc_allocate_mem(d, 0, 4096, T.NOPE) == 2
    assert L.tensDevRsc_free_mem(d) == 0 and L.tensDevRsc_is_empty(d) == T.YEP
    assert L.tensDevRsc_allocate_mem(d, 1, 4096, T.NOPE) == 5  # GPU 0 not in use: no runtime here
    assert L.tensDevRsc_allocate_mem(d, 0, 4096, T.YEP) == 0
    assert L.tensDevRsc_release_all(d) == 0 and L.tensDevRsc_is_empty(d) == T.YEP
    assert L.tensDevRsc_destroy(d) == 0


def test_shape_signature_and_offset_helpers(built, capfd):
    """tensShape_reshape / _print, the tensor-signature API and the column-major
    offset <-> multi-index helpers of the reference's tensor_algebra.h."""
    L = T.lib()
    sh = C.c_void_p()
    assert L.tensShape_create(C.byref(sh)) == 0
    assert L.tensShape_construct(sh, T.NOPE, 3, T.ivec([4, 6, 5]), None, None) == 0
    assert L.tensShape_reshape(sh, 2, T.ivec([12, 10]), None, None) == 0
    assert (L.tensShape_rank(sh), L.tensShape_volume(sh)) == (2, 120)
    assert L.tensShape_reshape(sh, 2, T.ivec([12, 11]), None, None) == -2   # volume changed: flagged
    assert L.tensShape_volume(sh) == 132
    L.tensShape_print(sh)
    C.CDLL(None).fflush(None)
    assert capfd.readouterr().out.endswith("[12,11]")
    assert L.tensShape_destroy(sh) == 0
    sg = C.c_void_p()
    assert L.tensSignature_create(C.byref(sg)) == 0
    offs = (C.c_size_t * 3)(7, 0, 3)
    assert L.tensSignature_construct(sg, 3, offs) == 0
    rank = C.cast(sg, C.POINTER(C.c_int))[0]
    assert rank == 3
    assert L.tensSignature_construct(sg, 2, None) == -3
    assert L.tensSignature_construct(sg, 0, None) == 0
    assert L.tensSignature_construct(sg, -1, None) == -2
    assert L.tensSignature_destroy(sg) == 0
    rng = np.random.default_rng(5)
    for _ in range(200):
        dims = [int(x) for x in rng.integers(1, 9, size=int(rng.integers(0, 6)))]
        idx = [int(rng.integers(0, d)) for d in dims]
        off = L.tens_elem_offset_f(len(dims), (C.c_uint * max(1, len(dims)))(*dims),
                                   (C.c_uint * max(1, len(dims)))(*idx))
        assert off == (int(np.ravel_multi_index(idx, dims, order="F")) if dims else 0)
        back = (C.c_uint * max(1, len(dims)))()
        L.tens_elem_mlndx_f(off, len(dims), (C.c_uint * max(1, len(dims)))(*dims), back)
        assert list(back[:len(dims)]) == idx


def test_every_reference_header_function_is_exported(built):
    """Every function the reference's talsh.h and tensor_algebra.h declare is
    exported by libtalsh.so, except get_contr_pattern_cutensor (cuTENSOR builds
    only; this core does not use cuTENSOR).  Skipped where the reference sources
    are absent."""
    ref = _reference_tree()
    if ref is None:
        pytest.skip("reference sources not present")
    L = T.lib()
    names = set()
    for h in ("talsh.h", "tensor_algebra.h"):
        names |= declared_functions(os.path.join(ref, h))
    assert len(names) > 150
    missing = sorted(n for n in names - {"get_contr_pattern_cutensor"} if not hasattr(L, n))
    assert not missing, missing
    buf = (C.c_char * 8)()
    assert L.fortran_cptr_int(C.cast(buf, C.c_void_p)) == C.cast(buf, C.c_void_p).value


def test_slice_views_without_gpu(built):
    """Slice descriptor objects (talshTensorSliceCreate / Construct / Volume /
    Destruct / Destroy, reference talshc.cpp:1857-1932): a view of a window of a
    tensor, refused when the window leaves the tensor, reconstructible, also for a
    rank-0 tensor."""
    L = T.lib()
    hb, ha = C.c_size_t(0), C.c_int(0)
    assert L.talshInit(C.byref(hb), C.byref(ha), 0, None, 0, None, 0, None) == 0
    try:
        t = T.Tensor([6, 5, 4], T.R8, dev_id=0, init=0.0)
        sv = C.c_void_p()
        assert L.talshTensorSliceCreate(C.byref(sv)) == 0 and L.talshTensorSliceVolume(sv) == 0
        offs = (C.c_size_t * 3)(1, 0, 2)
        assert L.talshTensorSliceConstruct(sv, t.ref, offs, T.ivec([5, 5, 2]), None, None) == 0
        assert L.talshTensorSliceVolume(sv) == 50
        assert L.talshTensorSliceConstruct(sv, t.ref, offs, T.ivec([2, 2, 2]), None, None) == 0
        assert L.talshTensorSliceVolume(sv) == 8
        assert L.talshTensorSliceConstruct(sv, t.ref, (C.c_size_t * 3)(2, 0, 0), T.ivec([5, 5, 4]), None,
                                           None) == T.TALSH_INVALID_ARGS
        assert L.talshTensorSliceConstruct(sv, t.ref, offs, T.ivec([2, 0, 2]), None, None) == T.TALSH_INVALID_ARGS
        assert L.talshTensorSliceVolume(sv) == 8                  # a refused construct leaves the view as it was
        assert L.talshTensorSliceDestruct(sv) == 0 and L.talshTensorSliceVolume(sv) == 0
        s0 = T.Tensor([], T.R8, dev_id=0, init=1.0)
        for _ in range(2):
            assert L.talshTensorSliceConstruct(sv, s0.ref, None, None, None, None) == 0
            assert L.talshTensorSliceVolume(sv) == 1
        assert L.talshTensorSliceDestroy(sv) == 0
        assert L.talshTensorSliceDestroy(None) == T.TALSH_INVALID_ARGS
        for x in (t, s0):
            assert x.destruct() == 0
    finally:
        assert L.talshShutdown() == 0
