"""The request server (kache_b200_server_*): requests submitted together from several threads are merged into runs,
and each one's result is the one it gets alone. Lookups and counts of a primed table, bit-exact against the plain
calls; upserts from several threads leave the same table (sorted dump, size) and the same total of inserted keys as
the same upserts run one by one."""
import threading

import numpy as np
import pytest

import kache
import synth
from kache import Batch

pytestmark = pytest.mark.gpu


def reads(seed, n, length=150):
    g = synth.genome(200_000, seed=7)
    return Batch(*synth.reads_fixed(g, n, length, seed=seed, sub=0.01, n_rate=0.001))


def sizes(rng, count):
    return np.clip(rng.lognormal(np.log(200), 1.2, size=count), 1, 4000).astype(int)


def test_queries_alone_and_in_the_mix():
    T = kache.Table(31, 4, 1_000_000, 0.8, False)
    u = T.register()
    T.upsert(u, reads(1, 20_000), kache.ADD, 1, 1)
    rng = np.random.default_rng(3)
    pool = reads(2, 60_000)
    reqs = []
    at = 0
    for i, m in enumerate(sizes(rng, 60)):
        m = int(min(m, pool.n - at)) or 1
        reqs.append(("lookup" if i % 3 else "count", pool.slice(at, at + m)))
        at = (at + m) % (pool.n - 4000)
    alone = [T.lookup(b, values=True, fwd=True) if kind == "lookup" else T.count(b) for kind, b in reqs]

    S = kache.Server(T)
    outs = [None] * len(reqs)
    tickets = [None] * len(reqs)

    def submit(idx):
        for i in idx:
            kind, b = reqs[i]
            P = int(b.positions(31).sum())
            if kind == "lookup":
                o = (np.full(P, 7, np.uint8), np.zeros(P, np.uint32), np.full(P, 7, np.uint8))
                tickets[i] = S.submit(kache.REQ_LOOKUP, b, out0=o[0], out1=o[1], out2=o[2])
            else:
                o = np.zeros(b.n, np.uint64)
                tickets[i] = S.submit(kache.REQ_COUNT, b, out0=o)
            outs[i] = o

    threads = [threading.Thread(target=submit, args=(range(j, len(reqs), 4),)) for j in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    results = [S.wait(t)[0] for t in tickets]
    runs, done = S.stats()
    S.close()
    assert done == len(reqs)
    for (kind, b), want, got, r in zip(reqs, alone, outs, results):
        if kind == "lookup":
            f, v, w = want
            np.testing.assert_array_equal(got[0], f)
            np.testing.assert_array_equal(got[1], v)
            np.testing.assert_array_equal(got[2], w)
            assert r == int((f == 1).sum())
        else:
            np.testing.assert_array_equal(got, want)
            assert r == int(want.sum())
    T.close()


def test_upserts_from_threads_match_one_by_one():
    rng = np.random.default_rng(5)
    pool = reads(4, 40_000)
    parts, at = [], 0
    for m in sizes(rng, 40):
        m = int(min(m, pool.n - at))
        if m == 0:
            break
        parts.append(pool.slice(at, at + m))
        at += m

    A = kache.Table(31, 4, 50_000, 0.8, False)
    ua = A.register()
    total_a = sum(A.upsert(ua, b, kache.ADD, 1, 1) for b in parts)

    B = kache.Table(31, 4, 50_000, 0.8, False)
    S = kache.Server(B)
    tickets = [None] * len(parts)

    def submit(idx):
        for i in idx:
            tickets[i] = S.submit(kache.REQ_UPSERT, parts[i], op=kache.ADD, x=1, init=1)

    threads = [threading.Thread(target=submit, args=(range(j, len(parts), 3),)) for j in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    total_b = sum(S.wait(t)[0] for t in tickets)
    S.close()
    assert total_b == total_a
    assert B.size() == A.size()
    ka, va = A.dump()
    kb, vb = B.dump()
    np.testing.assert_array_equal(ka, kb)
    np.testing.assert_array_equal(va, vb)
    A.close(), B.close()


def test_server_rejects_bad_requests():
    T = kache.Table(31, 8, 1000, 0.8, False)
    S = kache.Server(T)
    b = Batch.of(["ACGT" * 10])
    with pytest.raises(kache.KacheError):
        S.submit(7, b)
    with pytest.raises(kache.KacheError):
        S.submit(kache.REQ_LOOKUP, b)     # no output array
    with pytest.raises(kache.KacheError):
        S.submit(kache.REQ_UPSERT, b, op=9)
    with pytest.raises(kache.KacheError):
        S.wait(12345)
    S.close()
    T.close()
