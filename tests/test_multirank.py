"""The N > 1 host logic of bench.py on CPU: world_size-2 `gloo` ranks run the
replicas' timing aggregation (max over ranks of the per-rank time, all ranks'
units over it), exactly as the GPU ranks do over NCCL."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = 1.0 + rank  # rank 1 is the slow one
        slow = bench.slowest_rank(mine, world, torch.device("cpu"))
        rate = bench.whole_job_rate(1000.0, world, slow)
        dist.barrier()
        out.put((rank, slow, rate))
    finally:
        dist.destroy_process_group()


def test_replica_timing_max_over_ranks():
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [2.0, 2.0]          # both ranks see the slowest time
    assert [r[2] for r in res] == [1000.0, 1000.0]    # 2 ranks x 1000 units / 2 s


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.slowest_rank(1.5, 1, None) == 1.5
    assert bench.whole_job_rate(300.0, 1, 1.5) == 200.0
