"""One logical table over two ranks (kache-hash_b200/sharded.py) on CPU, with gloo: each rank's shard is the
checker's exact table and its describer the checker's, so what is tested is the partition by primary-bucket range,
the cutting of batches into runs, the all-to-all of runs and the routing of per-position results back, against one
table holding everything. Every rank upserts and queries its own reads; the totals, every rank's per-position lookups
and per-sequence counts, the oriented strand bits and the concatenated dump must equal the one table's, and each
shard may hold only the keys its rank owns."""
import os
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORLD = 2


def _batches(rank):
    import synth
    from kache import Batch
    g = synth.genome(150_000, seed=91)
    up = Batch(*synth.reads_variable(g, 1.5, 150, 0.8, 20, 2000, seed=92 + rank))
    q = Batch(*synth.reads_variable(g, 0.5, 150, 0.8, 5, 2000, seed=192 + rank))
    return up, q


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")]
    import torch.distributed as dist
    from datetime import timedelta
    import kache
    import oracle
    import sharded
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    up, q = _batches(rank)
    describe = lambda b: oracle.describe(b, 31, 22)
    T = sharded.ShardedTable(31, 8, make_shard=lambda: oracle.OracleTable(31, 8, 400_000), describe=describe)
    ins = T.upsert(up, kache.ADD_WRAP, 1, 1)
    present = T.update(q, kache.ADD_WRAP, 2)
    f, v, w = T.lookup(q)
    counts = T.count(q)
    keys, vals = T.dump()
    own_keys = T.shard.dump()[0]
    o = oracle.oracle().L
    owners = sharded.owner_of(np.array([o.orc_minimizer_hash(int(x), 31, 22) for x in own_keys], dtype=np.uint64), world)
    S = sharded.ShardedTable(31, 1, make_shard=lambda: oracle.OracleTable(31, 1, 400_000), describe=describe)
    ins_o = S.insert_oriented(up, kache.OR, 1, 2)
    fo, vo, wo = S.lookup(q)
    out.put((rank, ins, present, f, v, w, counts, keys, vals, bool((owners == rank).all()), len(own_keys), T.size(),
             ins_o, fo, vo, wo))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_table_matches_one_table():
    sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")]
    import kache
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + (os.getpid() % 1000)
    ps = [ctx.Process(target=_rank, args=(r, WORLD, port, q)) for r in range(WORLD)]
    for p in ps:
        p.start()
    res = sorted((q.get(timeout=300) for _ in ps), key=lambda x: x[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0

    # The one table: every rank's upserts (rank order does not matter: the op commutes), then every rank's updates.
    O = oracle.OracleTable(31, 8, 400_000)
    S = oracle.OracleTable(31, 1, 400_000)
    u, us = O.register(), S.register()
    ins = sum(O.upsert(u, _batches(r)[0], kache.ADD_WRAP, 1, 1) for r in range(WORLD))
    ins_o = sum(S.insert_oriented(us, _batches(r)[0], kache.OR, 1, 2) for r in range(WORLD))
    present = sum(O.update(_batches(r)[1], kache.ADD_WRAP, 2) for r in range(WORLD))
    keys, vals = O.dump()
    assert ins > 10_000 and present > 10_000
    shard_sizes = 0
    for (rank, r_ins, r_present, f, v, w, counts, r_keys, r_vals, owned, n_own, size, r_ins_o, fo, vo, wo) in res:
        qb = _batches(rank)[1]
        assert r_ins == ins and r_present == present and r_ins_o == ins_o and size == O.size()
        ef, ev, ew = O.lookup(qb)
        assert np.array_equal(f, ef) and np.array_equal(v, ev) and np.array_equal(w, ew)
        assert np.array_equal(counts, O.count(qb))
        sf, sv, sw = S.lookup(qb)
        assert np.array_equal(fo, sf) and np.array_equal(vo, sv) and np.array_equal(wo, sw)
        assert np.array_equal(r_keys, keys) and np.array_equal(r_vals, vals)
        assert owned and n_own > 0
        shard_sizes += n_own
    assert shard_sizes == O.size()      # every key in exactly one shard


def test_cut_runs_edges():
    """Runs of consecutive valid positions with one owner: none from empty or short sequences or invalid positions,
    one sequence and one owner each, and together exactly the valid positions, in output order."""
    sys.path[:0] = [ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")]
    import kache
    import sharded
    k = 31
    rng = np.random.default_rng(5)
    seqs = ["", "ACG", "A" * 30, "C" * 31, "ACGT" * 10 + "N" + "TTGCA" * 9, "G" * 35, "N" * 40]
    b = kache.Batch.of(seqs)
    P = int(b.positions(k).sum())
    valid = np.ones(P, bool)
    start = np.concatenate([[0], np.cumsum(b.positions(k))[:-1]])
    # Positions whose window holds the N of sequence 4, and every position of the N-only sequence, are not k-mers.
    n_at = 40
    for i in range(int(b.positions(k)[4])):
        if i <= n_at < i + k:
            valid[start[4] + i] = False
    valid[start[6]:start[6] + int(b.positions(k)[6])] = False
    for n in (1, 2, 3):
        h = rng.integers(0, 2**63, P, dtype=np.uint64)
        own, seq, p0, cnt, first = sharded.cut_runs(b, k, h, valid, n)
        covered = np.zeros(P, bool)
        owners = sharded.owner_of(h, n)
        for o, q, a, c, f in zip(own, seq, p0, cnt, first):
            assert c > 0 and f == start[q] + a and a + c <= b.positions(k)[q]
            assert valid[f:f + c].all() and (owners[f:f + c] == o).all() and not covered[f:f + c].any()
            covered[f:f + c] = True
        assert np.array_equal(covered, valid)
        assert list(first) == sorted(first)
        # Maximal: the position after a run is invalid, in another sequence, or owned elsewhere.
        for q, a, c, f in zip(seq, p0, cnt, first):
            e = f + c
            if a + c < b.positions(k)[q]:
                assert not valid[e] or owners[e] != owners[e - 1]
    z = sharded.cut_runs(kache.Batch.of([]), k, np.zeros(0, np.uint64), np.zeros(0, bool), 2)
    assert all(len(x) == 0 for x in z)
