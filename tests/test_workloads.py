"""The synthetic workloads bench.py measures (CPU): C4 and C5 tasks respect the
stated caps, their digital patterns are ones the oracle contracts, and C5
chains feed each task's output into the next task's left operand."""
import os
import sys

import numpy as np

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _oracle_accepts(kind, cptrn, dd, ld, rd, rng):
    dt = np.float64 if kind == bench.R8 else np.complex128
    D = np.zeros(dd if dd else (), dtype=dt, order="F")
    L = np.asfortranarray(rng.uniform(-1, 1, ld).astype(dt))
    R = np.asfortranarray(rng.uniform(-1, 1, rd).astype(dt))
    return O.tensor_contract(D, L, R, cptrn, 1.0, 0.0, 0, False) == 0


def test_c4_tasks(built):
    rng = np.random.default_rng(0)
    tasks = bench.c4_tasks()
    assert len(tasks) == 4096
    assert {k for k, *_ in tasks} == {bench.R8, bench.C8}
    checked = 0
    for kind, cp, dd, ld, rd, mnk in tasks:
        assert max(int(np.prod(x)) if x else 1 for x in (dd, ld, rd)) <= 1 << 21
        assert 2 <= len(ld) <= 6 and 2 <= len(rd) <= 6
        if checked < 60 and max(np.prod(ld), np.prod(rd)) <= 20000:
            assert _oracle_accepts(kind, cp, dd, ld, rd, rng)
            checked += 1
    assert checked == 60


def test_c5_tasks(built):
    rng = np.random.default_rng(1)
    tasks, arrivals = bench.c5_tasks(3000, 1000.0, seed=1000)
    assert len(tasks) == 3000 and np.all(np.diff(arrivals) >= 0)
    cc = [x for x in tasks if x["cc"]]
    assert 0.02 < len(cc) / len(tasks) < 0.08
    checked = 0
    for i, x in enumerate(tasks):
        if x["l_from"]:
            p = tasks[x["l_from"] - 1]
            assert x["l_from"] - 1 < i and p["dd"] == x["ld"] and p["kind"] == x["kind"] and p["consumers"] == 1
        if not x["cc"]:
            assert max(int(np.prod(v)) if v else 1 for v in (x["dd"], x["ld"], x["rd"])) <= 1 << 21
            if checked < 60 and max(np.prod(x["ld"]), np.prod(x["rd"])) <= 20000:
                assert _oracle_accepts(x["kind"], x["cptrn"], x["dd"], x["ld"], x["rd"], rng)
                checked += 1
    assert checked == 60
    lengths = {}
    for x in tasks:
        if x["chain"]:
            lengths[x["chain"]] = lengths.get(x["chain"], 0) + 1
    assert max(lengths.values()) <= 8
