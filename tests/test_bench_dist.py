"""The multi-rank plumbing of bench.py (replicas: one process per GPU, the
timing reported as the max over ranks) on CPU with the gloo backend and two
ranks."""
import os
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        bench.barrier(ws)
        m = bench.all_max(float(rank + 1) * 1.5, ws)
        bench.barrier(ws)
        out.put((rank, m))
    finally:
        dist.destroy_process_group()


def test_all_max_and_barrier_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 3.0), (1, 3.0)]
