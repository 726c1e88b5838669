"""Parity of the CUDA table with the oracle, through the C interface, on seeded synthetic inputs.

Modelled on the reference's own checks (kache-hash test/check.cpp, test/oriented.cpp, test/capi.cpp): sizes and
per-call inserted totals, per-position lookups (found, value, orientation), per-sequence counts, masked counts and
sums, single-k-mer lookups in both orientations and with an N, iteration over shares, reductions, present-only
updates, every C-interface operation at every value width, presized and resizing tables, and forced spills into the
overflow table. Everything integer is compared bit-exact.
"""
import numpy as np
import pytest

import kache
import oracle
import synth
from kache import Batch

pytestmark = pytest.mark.gpu

K, L = 31, 22


def make_inputs(seed=3, glen=300_000, nreads=20_000):
    g = synth.genome(glen, seed=seed)
    reads = Batch(*synth.reads_fixed(g, nreads, 150, seed=seed + 1))
    g2 = synth.genome(100_000, seed=seed + 7)
    neg = Batch(*synth.reads_fixed(g2, 3000, 150, seed=seed + 8))
    return g, reads, neg


@pytest.fixture(scope="module")
def inputs():
    return make_inputs()


def ragged_pieces(g, seed=5, n=400):
    """Raw pieces of ragged lengths with lowercase runs and non-ACGT characters (check.cpp multi mode, oriented.cpp)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L_ = int(rng.integers(0, 700))
        st = int(rng.integers(0, len(g) - L_ + 1))
        s = bytearray(synth.ASCII[g[st:st + L_]].tobytes())
        if i % 4 == 1 and L_ > 8:
            for j in range(L_ // 4, L_ // 2):
                s[j] |= 0x20
        if i % 7 == 2 and L_ > 200:
            s[50], s[90], s[130], s[170] = ord("N"), ord("n"), ord("R"), ord("-")
        if i % 3 == 0:
            s = bytearray(revcomp(bytes(s)))
        out.append(bytes(s))
    out += [b"", b"ACGT", b"A" * 30, b"N" * 40, b"a" * 31, b"NNNNACGTACGTACGTACGTACGTACGTACGTACGTNNNN", b"C" * 31]
    return out


_COMP = bytes.maketrans(b"ACGTacgt", b"TGCAtgca")


def revcomp(s):
    return s.translate(_COMP)[::-1]


def batches(b, size):
    return [b.slice(i, min(i + size, b.n)) for i in range(0, b.n, size)]


def both(vb, n, pow2=False, k=K):
    G = kache.Table(k, vb, n, 0.8, pow2)
    O = oracle.OracleTable(k, vb, n, 0.8, pow2)
    return G, O


def assert_same_table(G, O):
    kg, vg = G.dump()
    ko, vo = O.dump()
    assert G.size() == O.size() == len(ko)
    assert np.array_equal(kg, ko)
    if vo is not None:
        assert np.array_equal(vg, vo)
    assert G.capacity() == O.capacity()


def assert_same_queries(G, O, qs):
    for q in qs:
        fg, vg, wg = G.lookup(q)
        fo, vo, wo = O.lookup(q)
        assert np.array_equal(fg, fo)
        assert np.array_equal(wg, wo)
        if G.vb:
            assert np.array_equal(vg.astype(np.uint64), vo)
        assert np.array_equal(G.count(q), O.count(q))
        if G.vb:
            assert np.array_equal(G.sum(q), O.sum(q))
            assert np.array_equal(G.count_masked(q, 1, 2), O.count_masked(q, 1, 2))


@pytest.mark.parametrize("vb", [0, 1, 2, 4, 8])
@pytest.mark.parametrize("init", ["exact", 100_000, 10])
def test_counting_build_and_queries(inputs, vb, init):
    """check.cpp's matrix: upsert(v + 1, init 1) (insert for a set), from exact, large and tiny initial sizes."""
    g, reads, neg = inputs
    n = 560_000 if init == "exact" else init
    G, O = both(vb, n)
    ug, uo = G.register(), O.register()
    for b in batches(reads, 97):
        if vb:
            ig, io = G.upsert(ug, b, kache.ADD_WRAP, 1, 1), O.upsert(uo, b, kache.ADD_WRAP, 1, 1)
        else:
            ig, io = G.insert(ug, b), O.insert(uo, b)
        assert ig == io
        assert G.capacity() == O.capacity()
    assert_same_table(G, O)
    assert_same_queries(G, O, [reads.slice(0, 2000), neg, Batch.of(ragged_pieces(g))])
    # Present-only updates over everything again and the negatives (check.cpp:272-321).
    if vb:
        for b in batches(reads, 1000) + [neg]:
            assert G.update(b, kache.ADD_WRAP, 1, capi=False) == O.update(b, kache.ADD_WRAP, 1)
        assert_same_table(G, O)


@pytest.mark.parametrize("pow2", [False, True])
def test_sizing_matches(pow2):
    """capi.cpp: 1000 keys at 0.8 size to 1280 slots, or 2048 rounded to a power of 2."""
    t = kache.Table(31, 0, 1000, 0.8, pow2)
    assert t.capacity() == (2048 if pow2 else 1280)


def operand(op, b, bits):
    """capi.cpp:130-142: some sums saturate, ORs set one bit each."""
    mx = (1 << bits) - 1
    h = ((b + 1) * 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    if op == kache.ADD:
        return mx // 2 + 1 if b % 5 == 0 else 1 + b % 7
    if op == kache.OR:
        return 1 << ((h >> 32) % bits)
    return (h >> 7) & mx


@pytest.mark.parametrize("vb", [1, 2, 4, 8])
@pytest.mark.parametrize("op", [kache.KEEP, kache.ASSIGN, kache.ADD, kache.OR, kache.MIN, kache.MAX])
def test_capi_ops(inputs, vb, op):
    """Each C-interface operation at each width, from a tiny table that resizes, then updated by the same op."""
    g, reads, neg = inputs
    G, O = both(vb, 1000)
    ug, uo = G.register(), O.register()
    parts = batches(reads.slice(0, 6000), 500)
    for i, b in enumerate(parts):
        x = operand(op, i, 8 * vb)
        assert G.insert(ug, b, op, x) == O.insert(uo, b, op, x)
    assert_same_table(G, O)
    for i, b in enumerate(parts[:4]):
        x = operand(op, i + 100, 8 * vb)
        assert G.update(b, op, x) == O.update(b, op, x)
    assert_same_table(G, O)
    for what in (kache.REDUCE_KEYS, kache.REDUCE_POPCOUNT, kache.REDUCE_SUM):
        for m in (0xFFFFFFFFFFFFFFFF, 0x5):
            assert G.reduce(what, m) == O.reduce(what, m)


@pytest.mark.parametrize("vb,op,xf,xr", [(1, kache.OR, 1, 2), (8, kache.ADD, 1, 1 << 32), (4, kache.MAX, 7, 3), (2, kache.ADD, 1, 300)])
def test_oriented(inputs, vb, op, xf, xr):
    """oriented.cpp: the orientation mask and per-orientation counts, with forward and reverse pieces, lowercase and
    non-ACGT characters, and minimizer groups that spill into the overflow table."""
    g, reads, neg = inputs
    pieces = ragged_pieces(g, seed=11, n=600) + minimizer_group_seqs()
    b = Batch.of(pieces)
    for init in (len(pieces) * 200, 10):
        G, O = both(vb, init)
        ug, uo = G.register(), O.register()
        for part in batches(b, 13):
            assert G.insert_oriented(ug, part, op, xf, xr) == O.insert_oriented(uo, part, op, xf, xr)
        assert_same_table(G, O)
        assert_same_queries(G, O, [b, neg])
        for mf, mr in ((1, 2), (2, 1), (3, 0)):
            assert np.array_equal(G.count_masked(b, mf, mr), O.count_masked(b, mf, mr))
        if init > 10:
            st = G.stats()
            assert st.overflow_keys > 0 and st.secondary_pct > 0


_groups = None


def minimizer_group_seqs(G_=6, n=160, seed=42):
    """oriented.cpp:123-152: groups of k-mers sharing a minimizer, hence their primary and secondary buckets; only 96
    of a group fit in the main table. Each group's k-mers are inserted forward, reversed, or both."""
    global _groups
    if _groups is not None:
        return _groups
    o = oracle.oracle().L
    rng = np.random.default_rng(seed)
    acgt = b"ACGT"

    def enc(s):
        x = 0
        for c in s:
            x = (x << 2) | acgt.index(c)
        return x

    def lmer_hash(s):
        f = enc(s)
        r = o.orc_revcomp(f, L)
        return o.orc_wang(min(f, r))

    out, seen = [], set()
    for gi in range(G_):
        while True:
            X = bytes(acgt[i] for i in rng.integers(0, 4, L))
            if lmer_hash(X) <= (0xFFFFFFFFFFFFFFFF >> 10):
                break
        target = lmer_hash(X)
        group = []
        while len(group) < n:
            s = bytearray(acgt[i] for i in rng.integers(0, 4, K))
            p = int(rng.integers(0, K - L + 1))
            s[p:p + L] = X
            s = bytes(s)
            f = enc(s)
            r = o.orc_revcomp(f, K)
            key = min(f, r)
            if o.orc_minimizer_hash(key, K, L) != target or key in seen:
                continue
            seen.add(key)
            group.append(s)
        for s in group:
            if gi % 3 != 1:
                out.append(s)
            if gi % 3 != 0:
                out.append(revcomp(s))
    _groups = out
    return out


def test_single_kmer_get(inputs):
    """check.cpp:199-230: single lookups of k-mers in both orientations, with an N at varying positions, and of
    windows of the negatives."""
    g, reads, neg = inputs
    G, O = both(8, 560_000)
    ug, uo = G.register(), O.register()
    sub = reads.slice(0, 3000)
    G.upsert(ug, sub, kache.ADD_WRAP, 1, 1), O.upsert(uo, sub, kache.ADD_WRAP, 1, 1)
    seqs = [bytes(reads.bases[int(reads.off[i]):int(reads.off[i + 1])]) for i in range(0, 40)]
    seqs += [bytes(neg.bases[int(neg.off[i]):int(neg.off[i + 1])]) for i in range(0, 10)]
    for s in seqs:
        for j in range(0, len(s) - K + 1, 7):
            x = s[j:j + K]
            for y in (x, revcomp(x), x[:j % K] + b"N" + x[j % K + 1:]):
                assert G.get(y) == O.get(y)


def test_for_each_shares(inputs):
    """Iteration over 3 shares visits every key once (check.cpp:233-268)."""
    g, reads, neg = inputs
    G, O = both(8, 10)
    ug, uo = G.register(), O.register()
    sub = reads.slice(0, 4000)
    G.upsert(ug, sub, kache.ADD_WRAP, 1, 1), O.upsert(uo, sub, kache.ADD_WRAP, 1, 1)
    ks, vs = [], []
    for s in range(3):
        k_, v_ = G.for_each(3, s)
        ks.append(k_), vs.append(v_)
    keys = np.concatenate(ks)
    vals = np.concatenate(vs).astype(np.uint64)
    o = np.argsort(keys)
    ko, vo = O.dump()
    assert np.array_equal(keys[o], ko) and np.array_equal(vals[o], vo)
    # A callback that stops is not called again.
    k1, _ = G.for_each(1, 0, stop_after=1)
    assert len(k1) == 4096


def test_histogram(inputs):
    g, reads, neg = inputs
    G, O = both(4, 560_000)
    ug, uo = G.register(), O.register()
    G.upsert(ug, reads, kache.ADD_WRAP, 1, 1), O.upsert(uo, reads, kache.ADD_WRAP, 1, 1)
    for m in (3, 10, 10000):
        assert np.array_equal(G.histogram(m), O.histogram(m))


@pytest.mark.parametrize("k,l", [(31, 22), (27, 16), (32, 20)])
def test_describer(inputs, k, l):
    """describers.cpp: canonical key, checksum, minimizer hash and orientation per position, over stretches with
    non-ACGT characters and ragged lengths, against the restated describer."""
    g, reads, neg = inputs
    b = Batch.of(ragged_pieces(g, seed=21, n=300) + [bytes(reads.bases[int(reads.off[i]):int(reads.off[i + 1])]) for i in range(50)])
    G = kache.Table(k, 0, 1000, 0.8, False, capi=False)
    got = G.describe(b)
    exp = oracle.describe(b, k, l)
    for a, e in zip(got, exp):
        assert np.array_equal(a, e)


@pytest.mark.parametrize("k,vb", [(27, 1), (32, 0), (27, 8)])
def test_other_k(k, vb):
    """The template configurations beyond the C interface: <27, u8, 16> oriented and <32, void, 20> resizing."""
    g = synth.genome(200_000, seed=31)
    b = Batch(*synth.reads_variable(g, 3, 2000, 0.8, 500, 8000, seed=32, sub=0.03, ins=0.01, dele=0.01))
    G = kache.Table(k, vb, 1000, 0.8, False, capi=False)
    O = oracle.OracleTable(k, vb, 1000, 0.8, False)
    ug, uo = G.register(), O.register()
    for part in batches(b, 17):
        if vb == 1:
            assert G.insert_oriented(ug, part, kache.OR, 1, 2, capi=False) == O.insert_oriented(uo, part, kache.OR, 1, 2)
        elif vb:
            assert G.upsert(ug, part, kache.ADD_WRAP, 1, 1) == O.upsert(uo, part, kache.ADD_WRAP, 1, 1)
        else:
            assert G.insert(ug, part) == O.insert(uo, part)
    assert_same_table(G, O)
    assert_same_queries(G, O, [b.slice(0, 20)])


def test_edge_batches():
    """Empty batches, empty, short and all-N sequences, exactly k bases."""
    G, O = both(8, 1000)
    ug, uo = G.register(), O.register()
    empty = Batch.of([])
    assert G.insert(ug, empty, kache.ADD, 1) == 0
    assert len(G.count(empty)) == 0
    f, v, w = G.lookup(empty)
    assert len(f) == 0
    b = Batch.of([b"", b"A" * 30, b"N" * 100, b"ACGT" * 8, b"T" * 31, b"acgtn" * 20, b""])
    assert G.insert(ug, b, kache.ADD, 1) == O.insert(uo, b, kache.ADD, 1)
    assert_same_table(G, O)
    assert_same_queries(G, O, [b])


def test_argument_validation():
    """capi.cpp:405-447: validation, sizing, the user bound."""
    L_ = kache.lib()
    t = kache.Table(31, 1, 1000)
    for i in range(kache.MAX_USERS):
        assert t.register() == i
    with pytest.raises(kache.KacheError) as e:
        t.register()
    assert e.value.code == kache.KACHE_EUSERS
    b = Batch.of([b"ACGT" * 10])
    with pytest.raises(kache.KacheError):
        t.insert(200, b, kache.ADD, 1)          # unregistered user
    with pytest.raises(kache.KacheError):
        t.insert(0, b, kache.ADD, 256)          # operand too wide for u8
    with pytest.raises(kache.KacheError):
        t.insert(0, b, 9, 1)                    # no such op
    with pytest.raises(kache.KacheError):
        t.insert_oriented(0, b, kache.KEEP, 1, 1)
    s = kache.Table(31, 0, 1000)
    with pytest.raises(kache.KacheError):
        s.sum(b)
    with pytest.raises(kache.KacheError):
        s.reduce(kache.REDUCE_SUM)


def test_config1_full_parity():
    """The benchmark workload at full size: 333,333 reads of 150 bp into <31, u64, 22> sized for 10M keys with
    upsert(c + 1, init 1), then lookups of held-out reads; sorted dump and per-position results bit-exact."""
    g, ins, held = synth.config1()
    I = Batch(*ins)
    H = Batch(*held).slice(0, 100_000)
    G, O = both(8, 10_000_000)
    ug, uo = G.register(), O.register()
    assert G.upsert(ug, I, kache.ADD_WRAP, 1, 1) == O.upsert(uo, I, kache.ADD_WRAP, 1, 1)
    assert_same_table(G, O)
    fg, vg, wg = G.lookup(H)
    fo, vo, wo = O.lookup(H)
    assert np.array_equal(fg, fo) and np.array_equal(vg, vo) and np.array_equal(wg, wo)
