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


def _on_device(b, dev):
    """A host batch's bases and offsets as device tensors (kache_b200_server_submit_dev's layout)."""
    import torch
    bases = torch.from_numpy(np.concatenate([b.bases, np.zeros(16, np.uint8)])).to(dev)
    off = torch.from_numpy(b.off.view(np.int64).copy()).to(dev)
    return bases, off


def test_device_requests_alone_and_in_the_mix():
    """Requests resident in device memory, submitted from four threads together with host requests: each device
    request's outputs and result equal the plain call on the same reads; device upserts from several threads leave the
    table the host upserts one by one leave."""
    import torch
    dev = torch.device("cuda", 0)
    T = kache.Table(31, 4, 1_000_000, 0.8, False)
    u = T.register()
    T.upsert(u, reads(1, 20_000), kache.ADD, 1, 1)
    rng = np.random.default_rng(9)
    pool = reads(2, 60_000)
    reqs, at = [], 0
    for i, m in enumerate(sizes(rng, 48)):
        m = int(min(m, pool.n - at)) or 1
        reqs.append(("lookup" if i % 3 else "count", i % 2 == 0, pool.slice(at, at + m)))
        at = (at + m) % (pool.n - 4000)
    reqs.append(("lookup", True, Batch.of([])))
    reqs.append(("count", True, Batch.of([b"ACGT", b"N" * 50])))
    alone = [T.lookup(b, values=True, fwd=True) if kind == "lookup" else T.count(b) for kind, _, b in reqs]

    # Device requests' reads and output arrays, written before any is submitted.
    held = {}
    for i, (kind, on_dev, b) in enumerate(reqs):
        if on_dev:
            P = max(1, int(b.positions(31).sum()))
            o = (torch.full((P,), 7, dtype=torch.uint8, device=dev), torch.zeros(P * 4, dtype=torch.uint8, device=dev),
                 torch.full((P,), 7, dtype=torch.uint8, device=dev)) if kind == "lookup" else \
                torch.full((max(1, b.n),), 99, dtype=torch.int64, device=dev)
            held[i] = _on_device(b, dev) + (o,)
    torch.cuda.synchronize()

    S = kache.Server(T)
    outs, tickets = [None] * len(reqs), [None] * len(reqs)

    def submit(idx):
        for i in idx:
            kind, on_dev, b = reqs[i]
            P = max(1, int(b.positions(31).sum()))
            if on_dev:
                bases, off, o = held[i]
                if kind == "lookup":
                    tickets[i] = S.submit_dev(kache.REQ_LOOKUP, bases.data_ptr(), off.data_ptr(), b.n, out0=o[0].data_ptr(),
                                              out1=o[1].data_ptr(), out2=o[2].data_ptr())
                else:
                    tickets[i] = S.submit_dev(kache.REQ_COUNT, bases.data_ptr(), off.data_ptr(), b.n, out0=o.data_ptr())
            elif kind == "lookup":
                o = (np.full(P, 7, np.uint8), np.zeros(P, np.uint32), np.full(P, 7, np.uint8))
                tickets[i] = S.submit(kache.REQ_LOOKUP, b, out0=o[0], out1=o[1], out2=o[2])
            else:
                o = np.zeros(max(1, b.n), np.uint64)
                tickets[i] = S.submit(kache.REQ_COUNT, b, out0=o)
            outs[i] = o

    threads = [threading.Thread(target=submit, args=(range(j, len(reqs), 4),)) for j in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    results = [S.wait(t)[0] for t in tickets]
    S.close()
    for (kind, on_dev, b), want, got, r in zip(reqs, alone, outs, results):
        P = int(b.positions(31).sum())
        if kind == "lookup":
            f, v, w = want
            if on_dev:
                got = (got[0].cpu().numpy(), got[1].cpu().numpy().view(np.uint32), got[2].cpu().numpy())
            np.testing.assert_array_equal(got[0][:P], f)
            np.testing.assert_array_equal(got[1][:P], v)
            np.testing.assert_array_equal(got[2][:P], w)
            assert r == int((f == 1).sum())
        else:
            if on_dev:
                got = got.cpu().numpy().view(np.uint64)
            np.testing.assert_array_equal(got[:b.n], want)
            assert r == int(want.sum())
    T.close()

    # Device upserts from three threads against host upserts one by one.
    parts, at = [], 0
    for m in sizes(np.random.default_rng(11), 30):
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
    held = [_on_device(b, dev) for b in parts]
    torch.cuda.synchronize()
    tickets = [None] * len(parts)

    def submit_up(idx):
        for i in idx:
            bases, off = held[i]
            tickets[i] = S.submit_dev(kache.REQ_UPSERT, bases.data_ptr(), off.data_ptr(), parts[i].n, op=kache.ADD, x=1, init=1)

    threads = [threading.Thread(target=submit_up, args=(range(j, len(parts), 3),)) for j in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    total_b = sum(S.wait(t)[0] for t in tickets)
    S.close()
    assert total_b == total_a and B.size() == A.size() and B.capacity() == A.capacity()
    ka, va = A.dump()
    kb, vb = B.dump()
    np.testing.assert_array_equal(ka, kb)
    np.testing.assert_array_equal(va, vb)
    A.close(), B.close()


def test_server_rejects_bad_device_requests():
    import torch
    dev = torch.device("cuda", 0)
    T = kache.Table(31, 0, 1000, 0.8, False)
    S = kache.Server(T)
    bases, off = _on_device(Batch.of(["ACGT" * 10]), dev)
    out = torch.zeros(16, dtype=torch.uint8, device=dev)
    with pytest.raises(kache.KacheError):
        S.submit_dev(7, bases.data_ptr(), off.data_ptr(), 1)
    with pytest.raises(kache.KacheError):
        S.submit_dev(kache.REQ_LOOKUP, bases.data_ptr(), off.data_ptr(), 1)              # no output array
    with pytest.raises(kache.KacheError):
        S.submit_dev(kache.REQ_LOOKUP, bases.data_ptr(), off.data_ptr(), 1, out0=out.data_ptr(), out1=out.data_ptr())  # a set has no values
    with pytest.raises(kache.KacheError):
        S.submit_dev(kache.REQ_COUNT, None, None, 1, out0=out.data_ptr())
    S.close()
    T.close()
