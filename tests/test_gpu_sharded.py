"""The partitioned table (kache-hash_b200/sharded.py) with GPU shards: two ranks (processes sharing this GPU, each with
its own table, exchanging runs over gloo on the host; no kernel of one waits for the other's) and the GPU describer,
against one GPU table holding everything: totals, every rank's per-position lookups and counts, the dump."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _batches(rank):
    import synth
    from kache import Batch
    g = synth.genome(200_000, seed=81)
    up = Batch(*synth.reads_variable(g, 2.0, 150, 0.8, 20, 3000, seed=82 + rank))
    q = Batch(*synth.reads_variable(g, 0.5, 150, 0.8, 5, 3000, seed=182 + rank))
    return up, q


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")]
    import torch.distributed as dist
    from datetime import timedelta
    import kache
    import sharded
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    up, q = _batches(rank)
    T = sharded.ShardedTable(31, 8, expected_keys=600_000)
    ins = T.upsert(up, kache.ADD_WRAP, 1, 1)
    f, v, w = T.lookup(q)
    counts = T.count(q)
    keys, vals = T.dump()
    out.put((rank, ins, f, v, w, counts, keys, vals, T.size()))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_gpu_shards_match_one_table():
    sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")]
    import kache
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + (os.getpid() % 1000)
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted((q.get(timeout=300) for _ in ps), key=lambda x: x[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    T = kache.Table(31, 8, 600_000)
    u = T.register()
    ins = sum(T.upsert(u, _batches(r)[0], kache.ADD_WRAP, 1, 1) for r in range(2))
    keys, vals = T.dump()
    assert ins > 10_000
    for rank, r_ins, f, v, w, counts, r_keys, r_vals, size in res:
        qb = _batches(rank)[1]
        ef, ev, ew = T.lookup(qb, values=True, fwd=True)
        assert r_ins == ins and size == T.size()
        assert np.array_equal(f, ef) and np.array_equal(v, ev.astype(np.uint64)) and np.array_equal(w, ew)
        assert np.array_equal(counts, T.count(qb))
        assert np.array_equal(r_keys, keys) and np.array_equal(r_vals, vals)
    T.close()


def test_sharded_single_rank_is_the_plain_table():
    """Without a process group the partitioned table is one shard: runs cut and re-described on this GPU give the
    plain table's results."""
    import kache
    import sharded
    up, q = _batches(0)
    S = sharded.ShardedTable(31, 8, expected_keys=600_000)
    T = kache.Table(31, 8, 600_000)
    assert S.upsert(up, kache.ADD_WRAP, 1, 1) == T.upsert(T.register(), up, kache.ADD_WRAP, 1, 1)
    f, v, w = S.lookup(q)
    ef, ev, ew = T.lookup(q, values=True, fwd=True)
    assert np.array_equal(f, ef) and np.array_equal(v, ev.astype(np.uint64)) and np.array_equal(w, ew)
    assert np.array_equal(S.dump()[0], T.dump()[0])
