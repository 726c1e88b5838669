"""Configurations 2-5 at their stated sizes (config 5 at a twentieth), compared bit for bit with the reference's own
table (oracle/_ref, built from the reference's sources) run on the same inputs beside the GPU:

- config 2, Kmer_Set_Counter: primed size, present k-mers counted per batch, histogram(10000) (the reference's own
  check, test/counter.cpp:479), count_of on sampled k-mers, and the whole table (key, count);
- config 3, the oriented strand map: keys inserted and capacity after every call, the whole table (key, strand bits),
  and the per-position oriented find (found, strand bits, orientation) of every read;
- config 4, the resize-heavy set: keys inserted and capacity after every call (nine doublings), the final set;
- config 5, the served mix: every find's and count's result from the request server against the reference running
  the requests one by one in arrival order, the inserted keys of every run of consecutive upserts, the final table.

Tables too large to sort in a test are compared through an order-independent digest of their (key, value) pairs
(oracle.digest). Where the reference's table is driven by one user per call (configs 3 and 4), its capacity after
each call is the reference's own, compared with the GPU table's."""
import os
import threading

import numpy as np
import pytest

import kache
import oracle
import synth
from kache import Batch

pytestmark = pytest.mark.gpu


def threads():
    return min(128, os.cpu_count() or 1)


def reference():
    if oracle.ref() is None:
        pytest.fail("the reference's table (oracle/_ref) is not built: run oracle/Makefile's `ref` target")


def pieces(b, per):
    return [b.slice(s, min(b.n, s + per)) for s in range(0, b.n, per)]


def table_digest(t):
    keys, vals = t.for_each()
    return oracle.digest(keys, None if vals is None else vals.astype(np.uint64))


def ref_digest(r):
    keys, vals = r.raw_dump()
    return oracle.digest(keys, vals)


def test_config2_counter_against_reference():
    """Kmer_Set_Counter (<31, u32, 22>, lf 0.9, power-of-2 capacity): prime with a 100 Mbp genome with 5 % segmental
    duplications, count its 30x reads in batches of 2^20 reads, histogram(10000)."""
    reference()
    g, index, reads = synth.config2()
    bi, br = Batch(*index), Batch(*reads)
    C = kache.Counter(100_000_000, 16, 0.9)
    R = oracle.RefTable(31, 4, 100_000_000, 0.9, True, workers=threads())
    C.prime_batch(bi)
    _, primed = R.bench_upsert(bi, kache.KEEP, 0, threads())     # prime: upsert(v -> v, init 0)
    assert C.size() == R.size() == primed
    for p in pieces(br, 1 << 20):
        _, present = R.bench_update(p, kache.ADD_WRAP, 1, threads())     # count: update(v -> v + 1)
        assert C.count_batch(p) == present
    h = C.histogram(10000)
    keys, vals = R.raw_dump()
    inrange = (vals >= 1) & (vals <= 10000)
    h_ref = np.bincount(vals[inrange].astype(np.int64), minlength=10001).astype(np.uint64)
    assert h[0] == 0 and np.array_equal(h, h_ref)
    assert table_digest(C.table()) == oracle.digest(keys, vals)
    del keys, vals
    rng = np.random.default_rng(23)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    for p in rng.integers(0, len(g) - 31, 200):
        kmer = acgt[g[int(p):int(p) + 31]].tobytes()
        assert C.count_of(kmer) == R.get(kmer)[1]
    C.close()


def test_config3_strand_map_against_reference():
    """<27, u8, 16> upsert_oriented(OR, fwd 1, rev 2) of 5x long reads with indels in calls of 4,096 reads, then the
    oriented find of every read."""
    reference()
    g, r = synth.config3()
    b = Batch(*r)
    T = kache.Table(27, 1, 50_000_000, 0.8, False, capi=False)
    R = oracle.RefTable(27, 1, 50_000_000, 0.8, False)
    u, ur = T.register(), R.register()
    ps = pieces(b, 4096)
    for p in ps:
        assert T.insert_oriented(u, p, kache.OR, 1, 2, capi=False) == R.insert_oriented(ur, p, kache.OR, 1, 2)
        assert T.capacity() == R.capacity()
    assert T.size() == R.size()
    assert table_digest(T) == ref_digest(R)
    for p in ps:
        f, v, w = T.lookup(p, values=True, fwd=True)
        fr, vr, wr = R.lookup(p)
        assert np.array_equal(f, fr)
        assert np.array_equal(v.astype(np.uint64), vr)
        assert np.array_equal(w, wr)
    T.close()


def test_config4_resize_heavy_set_against_reference():
    """<32, void, 20> sized for 1M keys (lf 0.8, exact): a 400 Mbp uniform genome as 150 bp pieces at 1x, in calls of
    65,536 pieces; the table doubles nine times."""
    reference()
    g, st = synth.config4()
    b = Batch(*st)
    T = kache.Table(32, 0, 1_000_000, 0.8, False, capi=False)
    R = oracle.RefTable(32, 0, 1_000_000, 0.8, False)
    u, ur = T.register(), R.register()
    cap0 = T.capacity()
    for p in pieces(b, 65_536):
        assert T.insert(u, p) == R.insert(ur, p, kache.KEEP, 0)
        assert T.capacity() == R.capacity()
    assert T.capacity() == 512 * cap0       # nine doublings
    assert T.size() == R.size() == T.reduce(kache.REDUCE_KEYS)
    assert table_digest(T) == ref_digest(R)
    T.close()


def _served(S, group, outs):
    """Submits the group's requests from four threads at once; returns each request's result."""
    tickets = [None] * len(group)

    def client(idx):
        for i in idx:
            kind, b = group[i]
            o = outs[i]
            tickets[i] = S.submit(kind, b, op=kache.ADD, x=1, init=1, out0=o[0], out1=o[1])

    th = [threading.Thread(target=client, args=(range(j, len(group), 4),)) for j in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return [S.wait(t)[0] for t in tickets]


def test_config5_served_mix_against_reference():
    """<31, u32, 22> primed with a 100 Mbp genome's 31-mers (config 5 at a twentieth), then 300 requests (upsert ADD 1 /
    find / count at 60/30/10) through the request server. Consecutive requests of one class (upserts; queries) are
    submitted together from four threads and merge on the device; the next group waits for them, so every query sees
    exactly the upserts before it in arrival order, as in the reference run one request at a time."""
    reference()
    g, primer, reqs = synth.config5(0.05, 300)
    bp = Batch(*primer)
    T = kache.Table(31, 4, len(g), 0.8, False)
    R = oracle.RefTable(31, 4, len(g), 0.8, False)
    u, ur = T.register(), R.register()
    T.upsert(u, bp, kache.KEEP, 0, 0)
    R.upsert(ur, bp, kache.KEEP, 0)
    assert T.size() == R.size()

    groups, cur = [], []
    for kind, b in reqs:
        if cur and (kind == 0) != (cur[-1][0] == 0):
            groups.append(cur)
            cur = []
        cur.append((kind, b))
    groups.append(cur)
    assert sum(len(x) for x in groups) == len(reqs) and len(groups) > 20

    S = kache.Server(T)
    checked = 0
    for group in groups:
        outs = []
        for kind, b in group:
            P = int(b.positions(31).sum())
            if kind == 1:
                outs.append((np.full(max(P, 1), 255, np.uint8), np.zeros(max(P, 1), np.uint32)))
            elif kind == 2:
                outs.append((np.zeros(max(b.n, 1), np.uint64), None))
            else:
                outs.append((None, None))
        got = _served(S, group, outs)
        if group[0][0] == 0:
            expect = sum(R.upsert(ur, b, kache.ADD, 1) for _, b in group)
            assert sum(got) == expect
            continue
        for (kind, b), o, res in zip(group, outs, got):
            P = int(b.positions(31).sum())
            fr, vr, _ = R.lookup(b)
            if kind == 1:
                assert np.array_equal(o[0][:P], fr)
                assert np.array_equal(o[1][:P].astype(np.uint64), vr)
                assert res == int((fr == 1).sum())
            else:
                pos = b.positions(31)
                ends = np.cumsum(pos)
                hits = np.concatenate([[0], np.cumsum(fr == 1)])
                per_seq = (hits[ends] - hits[ends - pos]).astype(np.uint64)
                assert np.array_equal(o[0][:b.n], per_seq)
                assert res == int(per_seq.sum())
            checked += 1
    _, served = S.stats()
    S.close()
    assert served == len(reqs) and checked == sum(1 for k, _ in reqs if k != 0)
    assert T.size() == R.size()
    assert table_digest(T) == ref_digest(R)
    T.close()
