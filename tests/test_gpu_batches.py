"""Several device batches run as one call (kache_b200_run_dev_batches) against the oracle, through the C interface.

Each kind of the call is checked bit-exact: upserts (the table's dump, size, capacity and the sum of the per-batch
inserted counts; per batch exact where the batches share no k-mer), oriented upserts, present-only updates (per-batch
present counts and the final table), per-position lookups (each batch's own found, value and orientation arrays, and
its positions found) and per-sequence counts (each batch's own array, and their sum). The batches are ragged: empty batches, batches without a k-mer,
sequences shorter than k, non-ACGT characters, lowercase runs, offsets that do not start at 0 (a batch that is a
window of a larger buffer), more sequences than one block sums, and more batches than one block lists.
"""
import numpy as np
import pytest

import kache
import oracle
import synth
from kache import Batch

pytestmark = pytest.mark.gpu

K = 31


def _pieces():
    """Host batches, cut from ragged and fixed-length reads of one genome, with the odd cases mixed in."""
    g = synth.genome(200_000, seed=61)
    fixed = Batch(*synth.reads_fixed(g, 6000, 150, seed=62))
    ragged = Batch(*synth.reads_variable(g, 0.5, 300, 1.0, 1, 3000, seed=63))
    odd = Batch.of([b"", b"ACGT", b"N" * 40, b"a" * 31, b"acgtNNacgt" * 9, b"C" * 31])
    rng = np.random.default_rng(64)
    out = []
    for src in (fixed, ragged):
        s = 0
        while s < src.n:
            e = min(src.n, s + int(rng.integers(0, 300)))
            out.append(src.slice(s, e))
            s = e
    out.insert(3, odd)
    out.insert(5, Batch.of([]))
    return out


def _dev(batches, window=False):
    """The batches in device memory as (bases, offsets, n) tensors; with `window`, every third batch is a window of a
    larger buffer: its offsets start past 0."""
    import torch
    dev = torch.device("cuda", 0)
    out = []
    for i, b in enumerate(batches):
        pad = 37 if window and i % 3 == 0 else 0
        bases = np.concatenate([np.full(pad, ord("G"), np.uint8), b.bases, np.zeros(16, np.uint8)])
        off = (b.off + np.uint64(pad)).view(np.int64)
        out.append((torch.from_numpy(bases).to(dev), torch.from_numpy(off.copy()).to(dev), b.n))
    return out


def _concat(batches):
    seqs = []
    for b in batches:
        seqs += [bytes(b.bases[int(b.off[i]):int(b.off[i + 1])]) for i in range(b.n)]
    return Batch.of(seqs)


def _positions(b):
    return int(b.positions(K).sum())


@pytest.mark.parametrize("vb", [8, 4, 1])
def test_upsert_lookup_count_update(vb):
    import torch
    host = _pieces()
    devb = _dev(host, window=True)
    allb = _concat(host)
    G = kache.Table(K, vb, 50_000)
    O = oracle.OracleTable(K, vb, 50_000)
    u, uo = G.register(), O.register()
    res = G.run_dev_batches(kache.RUN_UPSERT, [(b.data_ptr(), o.data_ptr(), n) for b, o, n in devb], kache.ADD_WRAP, 1, 1, u)
    assert sum(res) == O.upsert(uo, allb, kache.ADD_WRAP, 1, 1)
    assert G.size() == O.size() and G.capacity() == O.capacity()
    kg, vg = G.dump()
    ko, vo = O.dump()
    assert np.array_equal(kg, ko) and np.array_equal(vg, vo)

    # Lookups: each batch's own arrays, as a lookup of that batch alone. The found flags lie in one buffer at offsets
    # of every residue mod 4, so the per-batch count of found flags reads unaligned heads and tails.
    dev = torch.device("cuda", 0)
    outs = []
    fbuf = torch.full((sum(max(1, _positions(b)) + 1 for b in host) + 1,), 7, dtype=torch.uint8, device=dev)
    at = 1
    for b in host:
        P = max(1, _positions(b))
        outs.append((fbuf[at:at + P], torch.zeros(P * vb, dtype=torch.uint8, device=dev),
                     torch.full((P,), 7, dtype=torch.uint8, device=dev)))
        at += P + 1
    hits = G.run_dev_batches(kache.RUN_LOOKUP, [(b.data_ptr(), o.data_ptr(), n, f.data_ptr(), v.data_ptr(), w.data_ptr())
                                                 for (b, o, n), (f, v, w) in zip(devb, outs)])
    dt = {8: np.uint64, 4: np.uint32, 1: np.uint8}[vb]
    for hb, (f, v, w), h in zip(host, outs, hits):
        P = _positions(hb)
        fo, vo_, wo = O.lookup(hb)
        assert h == int((fo == 1).sum())
        assert np.array_equal(f.cpu().numpy()[:P], fo)
        assert np.array_equal(v.cpu().numpy().view(dt)[:P], vo_.astype(dt))
        assert np.array_equal(w.cpu().numpy()[:P], wo)

    # Per-sequence counts into each batch's array.
    counts = [torch.full((max(1, n),), 99, dtype=torch.int64, device=dev) for _, _, n in devb]
    sums = G.run_dev_batches(kache.RUN_COUNT, [(b.data_ptr(), o.data_ptr(), n, c.data_ptr()) for (b, o, n), c in zip(devb, counts)])
    for hb, c, sm in zip(host, counts, sums):
        assert np.array_equal(c.cpu().numpy().view(np.uint64)[:hb.n], O.count(hb))
        assert sm == int(O.count(hb).sum())

    # Present-only update: per-batch present counts, then the same table.
    res = G.run_dev_batches(kache.RUN_UPDATE, [(b.data_ptr(), o.data_ptr(), n) for b, o, n in devb], kache.ADD_WRAP, 3)
    assert res == [O.update(hb, kache.ADD_WRAP, 3) for hb in host]
    kg, vg = G.dump()
    ko, vo = O.dump()
    assert np.array_equal(kg, ko) and np.array_equal(vg, vo)
    G.close()


def test_per_batch_inserted_and_many_batches():
    """Batches from different genomes share no k-mer, so each batch's inserted count is exact; 5,000 batches and more
    than 4,096 sequences take the listing and staging paths for large merged batches."""
    genomes = [synth.genome(20_000, seed=70 + i) for i in range(4)]
    host = []
    for i in range(5000):
        g = genomes[i % 4]
        n = (i * 7) % 5
        host.append(Batch(*synth.reads_fixed(g, n, 150, seed=1000 + i)) if n else Batch.of([]))
    devb = _dev(host)
    G = kache.Table(K, 8, 10_000)
    O = oracle.OracleTable(K, 8, 10_000)
    u, uo = G.register(), O.register()
    res = G.run_dev_batches(kache.RUN_UPSERT, [(b.data_ptr(), o.data_ptr(), n) for b, o, n in devb], kache.ADD_WRAP, 1, 1, u)
    # Per genome, the keys its batches inserted: the genome's distinct k-mers among them, exactly.
    for j in range(4):
        Oj = oracle.OracleTable(K, 8, 10_000)
        uj = Oj.register()
        assert sum(res[j::4]) == Oj.upsert(uj, _concat(host[j::4]), kache.ADD_WRAP, 1, 1)
    assert sum(res) == O.upsert(uo, _concat(host), kache.ADD_WRAP, 1, 1)
    assert G.capacity() == O.capacity()
    kg, vg = G.dump()
    ko, vo = O.dump()
    assert np.array_equal(kg, ko) and np.array_equal(vg, vo)
    G.close()


def test_oriented_and_set():
    import torch
    host = _pieces()
    devb = _dev(host, window=True)
    allb = _concat(host)
    G = kache.Table(27, 1, 50_000)
    O = oracle.OracleTable(27, 1, 50_000)
    u, uo = G.register(), O.register()
    res = G.run_dev_batches(kache.RUN_UPSERT_ORIENTED, [(b.data_ptr(), o.data_ptr(), n) for b, o, n in devb], kache.OR, 1, 2, u)
    assert sum(res) == O.insert_oriented(uo, allb, kache.OR, 1, 2)
    kg, vg = G.dump()
    ko, vo = O.dump()
    assert np.array_equal(kg, ko) and np.array_equal(vg, vo)
    G.close()

    S = kache.Table(32, 0, 20_000)
    SO = oracle.OracleTable(32, 0, 20_000)
    us, uso = S.register(), SO.register()
    res = S.run_dev_batches(kache.RUN_UPSERT, [(b.data_ptr(), o.data_ptr(), n) for b, o, n in devb], kache.KEEP, 0, 0, us)
    assert sum(res) == SO.insert(uso, allb)
    assert S.capacity() == SO.capacity()
    assert np.array_equal(S.dump()[0], SO.dump()[0])
    dev = torch.device("cuda", 0)
    found = [torch.full((max(1, int(b.positions(32).sum())),), 7, dtype=torch.uint8, device=dev) for b in host]
    hits = S.run_dev_batches(kache.RUN_LOOKUP, [(b.data_ptr(), o.data_ptr(), n, f.data_ptr()) for (b, o, n), f in zip(devb, found)])
    for hb, f, h in zip(host, found, hits):
        P = int(hb.positions(32).sum())
        fo = SO.lookup(hb)[0]
        assert np.array_equal(f.cpu().numpy()[:P], fo)
        assert h == int((fo == 1).sum())
    S.close()


def test_validation():
    host = _pieces()[:4]
    devb = _dev(host)
    T = kache.Table(K, 8, 10_000)
    u = T.register()
    S = kache.Table(32, 0, 10_000)
    S.register()
    plain = [(b.data_ptr(), o.data_ptr(), n) for b, o, n in devb]
    for fn in (lambda: T.run_dev_batches(5, plain),                                    # no such kind
               lambda: T.run_dev_batches(kache.RUN_LOOKUP, plain),                     # lookups need out0
               lambda: T.run_dev_batches(kache.RUN_COUNT, plain),                      # counts need out0
               lambda: T.run_dev_batches(kache.RUN_UPSERT, plain, kache.ADD, 1, 1, u + 5),     # not a registered user
               lambda: T.run_dev_batches(kache.RUN_UPSERT, plain, 99, 1, 1, u),        # no such op
               lambda: T.run_dev_batches(kache.RUN_UPSERT, [(0, 0, 3)], kache.ADD, 1, 1, u),   # null pointers
               lambda: S.run_dev_batches(kache.RUN_UPSERT_ORIENTED, plain, kache.OR, 1, 2, 0),  # sets have no values
               lambda: S.run_dev_batches(kache.RUN_UPDATE, plain, kache.ADD, 1)):
        with pytest.raises(kache.KacheError) as e:
            fn()
        assert e.value.code == kache.KACHE_EINVAL
    assert T.run_dev_batches(kache.RUN_UPSERT, [], kache.ADD, 1, 1, u) == []
    assert T.run_dev_batches(kache.RUN_UPSERT, [(0, 0, 0)], kache.ADD, 1, 1, u) == [0]
    assert T.size() == 0
    T.close()
    S.close()
