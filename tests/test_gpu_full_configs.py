"""Configurations 2-4 at their full sizes, checked through properties that do not need the exact dictionary at that
size: capacities after every call against the reference's schedule replayed from the per-call inserted counts
(oracle.replay_capacity, pinned against the reference in test_oracle_pinning.py), key counts against the distinct
k-mers of the input, presence of sampled k-mers, the strand bits of oriented upserts, and the counter's histogram
against its counted occurrences."""
import numpy as np
import pytest

import kache
import oracle
import synth
from kache import Batch

pytestmark = pytest.mark.gpu


def pieces(b, per):
    return [b.slice(s, min(b.n, s + per)) for s in range(0, b.n, per)]


def test_config4_resize_heavy_set():
    """<32, void, 20> sized for 1M keys (lf 0.8, exact): a 400 Mbp uniform genome as 150 bp pieces at 1x, in calls of
    65,536 pieces; the table doubles nine times."""
    g, st = synth.config4()
    b = Batch(*st)
    T = kache.Table(32, 0, 1_000_000, 0.8, False, capi=False)
    u = T.register()
    cap0 = T.capacity()
    ins, caps = [], []
    for p in pieces(b, 65_536):
        ins.append(T.insert(u, p))
        caps.append(T.capacity())
    assert caps == list(oracle.replay_capacity(1_000_000, 0.8, False, ins))
    assert caps[-1] == 512 * cap0        # nine doublings
    total = sum(ins)
    assert T.size() == total == T.reduce(kache.REDUCE_KEYS)
    # A uniform 400 Mbp genome repeats hardly any 32-mer: every position inserts.
    P = int(b.positions(32).sum())
    assert P - 1000 <= total <= P
    # Sampled pieces are found whole; random 32-mers are not.
    rng = np.random.default_rng(41)
    sample = [b.slice(int(i), int(i) + 1) for i in rng.integers(0, b.n, 200)]
    for s in sample:
        f, _, _ = T.lookup(s, values=False, fwd=False)
        assert (f == 1).all()
    acgt = np.frombuffer(b"ACGT", np.uint8)
    rand = Batch.of([acgt[rng.integers(0, 4, 64)].tobytes() for _ in range(200)])
    f, _, _ = T.lookup(rand, values=False, fwd=False)
    assert (f == 1).sum() <= 2
    T.close()


def test_config3_strand_map():
    """<27, u8, 16> upsert_oriented(OR, fwd 1, rev 2) of 5x long reads with indels, in calls of 4,096 reads."""
    g, r = synth.config3()
    b = Batch(*r)
    T = kache.Table(27, 1, 50_000_000, 0.8, False, capi=False)
    u = T.register()
    ins, caps = [], []
    for p in pieces(b, 4096):
        ins.append(T.insert_oriented(u, p, kache.OR, 1, 2, capi=False))
        caps.append(T.capacity())
    assert caps == list(oracle.replay_capacity(50_000_000, 0.8, False, ins))
    assert T.size() == sum(ins) == T.reduce(kache.REDUCE_KEYS)
    # Every value is a nonempty set of strands, and a k-mer seen both ways has both bits.
    assert T.reduce(kache.REDUCE_POPCOUNT, 0xFC) == 0
    both_ways = T.reduce(kache.REDUCE_POPCOUNT, 0x3) - T.size()
    assert 0 <= both_ways <= T.size()
    # Each position of sampled reads is present with its own strand's bit.
    rng = np.random.default_rng(33)
    for i in rng.integers(0, b.n, 40):
        s = b.slice(int(i), int(i) + 1)
        f, v, w = T.lookup(s, values=True, fwd=True)
        _, _, _, fw, va = oracle.describe(s, 27, 16)
        assert (f[va == 1] == 1).all() and (f[va == 0] == 2).all()
        assert np.array_equal(w[va == 1], fw[va == 1])
        bit = np.where(fw == 1, 1, 2).astype(np.uint8)
        assert ((v[va == 1] & bit[va == 1]) != 0).all()
    T.close()


def test_config2_counter():
    """Kmer_Set_Counter (<31, u32, 22>, lf 0.9, power-of-2 capacity): prime with a 100 Mbp genome with 5 % segmental
    duplications, count its 30x reads; the primed set is the genome's distinct 31-mers, and histogram(10000) accounts
    for every counted occurrence."""
    g, index, reads = synth.config2()
    bi, br = Batch(*index), Batch(*reads)
    C = kache.Counter(100_000_000, 16, 0.9)
    C.prime_batch(bi)
    key, _, _, _, va = oracle.describe(bi, 31, 22)
    distinct = len(np.unique(key[va == 1]))
    del key, va
    assert C.size() == distinct
    found = sum(C.count_batch(p) for p in pieces(br, 1 << 20))
    h = C.histogram(10000)
    assert h[0] == 0
    assert int(h.sum()) <= C.size()
    counts = np.arange(len(h), dtype=np.uint64)
    assert int((h * counts).sum()) == found
    # Sampled genome 31-mers, each covered by about 25 error-free reads on average, were all counted.
    rng = np.random.default_rng(23)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    for p in rng.integers(0, len(g) - 31, 50):
        assert C.count_of(acgt[g[int(p):int(p) + 31]].tobytes().decode()) >= 1
    C.close()
