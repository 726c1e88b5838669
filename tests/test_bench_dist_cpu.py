"""The multi-rank plumbing of bench.py on CPU, with gloo and two ranks: each rank gets its own reads (independent
tables, weak scaling, no data-path collective), and the job's time is the slowest rank's."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200")]
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    ws, r, local = bench.dist_env()
    ins, held = bench.workload(r, scale=0.01)
    t = bench.max_over_ranks(dist, 10.0 + r, "cpu")
    out.put((r, ws, local, t, bytes(ins[0][:300]), bench.rank_seeds(r)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ws0, l0, t0, b0, s0), (r1, ws1, l1, t1, b1, s1) = res
    assert (r0, r1, ws0, ws1) == (0, 1, 2, 2)
    assert t0 == t1 == 11.0          # max over ranks
    assert b0 != b1 and s0 != s1     # each rank its own reads
