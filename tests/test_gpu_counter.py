"""The counter library on the GPU against the oracle (reference test/counter.cpp:374-497): a fully synthetic set,
primed from a FASTA file, counted from FASTQ reads; size, occurrences found, count_of in both orientations, in
lowercase, with an N and for absent k-mers, and histogram(3) / histogram(10000), bit-exact."""
import numpy as np
import pytest

import kache
import oracle
import synth
from kache import Batch

pytestmark = pytest.mark.gpu


def write_fasta(path, b, width=80):
    with open(path, "wb") as f:
        for i in range(b.n):
            s = bytes(b.bases[int(b.off[i]):int(b.off[i + 1])])
            f.write(b">s%d\n" % i)
            for j in range(0, len(s), width):
                f.write(s[j:j + width] + b"\n")


def write_fastq(path, b):
    with open(path, "wb") as f:
        for i in range(b.n):
            s = bytes(b.bases[int(b.off[i]):int(b.off[i + 1])])
            f.write(b"@r%d\n%s\n+\n%s\n" % (i, s, b"I" * len(s)))


@pytest.mark.parametrize("n_hint", ["exact", "small"])
def test_counter_files(tmp_path, n_hint):
    g = synth.genome(400_000, seed=1, dup_frac=0.05, dup_len=(1000, 5000))
    index = Batch(*synth.stretches(g, 5000))
    reads = Batch(*synth.reads_variable(g, 8, 150, 0.6, 50, 1000, seed=2))
    fa, fq = str(tmp_path / "index.fa"), str(tmp_path / "reads.fq")
    write_fasta(fa, index)
    write_fastq(fq, reads)
    n = 400_000 if n_hint == "exact" else 1000
    C = kache.Counter(n, threads=4)
    O = oracle.OracleTable(31, 4, n, 0.9, True)
    uo = O.register()
    C.prime(fa)
    O.upsert(uo, index, kache.KEEP, 0, 0)
    assert C.size() == O.size()
    found = C.count(fq)
    assert found == O.update(reads, kache.ADD_WRAP, 1)
    for m in (3, 10_000):
        assert np.array_equal(C.histogram(m), O.histogram(m))
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    s = bytes(synth.ASCII[g[1000:4000]])
    for j in range(0, len(s) - 31, 13):
        x = s[j:j + 31]
        exp = O.get(x)[1]
        assert C.count_of(x) == exp
        assert C.count_of(x.translate(comp)[::-1]) == exp
        assert C.count_of(x.lower()) == exp
        assert C.count_of(x[:5] + b"N" + x[6:]) == 0
    rng = np.random.default_rng(3)
    for _ in range(2000):
        x = bytes(synth.ASCII[rng.integers(0, 4, 31)])
        assert C.count_of(x) == O.get(x)[1]
    # The capacity: rounded to a power of two at load 0.9, resized where the reference would be.
    t = kache.Table.__new__(kache.Table)
    t.h = kache.lib().kache_counter_table(C.h)
    s_ = kache.Stats()
    assert kache.lib().kache_get_stats(t.h, kache.ctypes.byref(s_)) == 0
    assert s_.capacity == O.capacity()
    t.h = None


def test_counter_batches():
    """In-memory batches, counted three times over."""
    g = synth.genome(50_000, seed=9)
    b = Batch(*synth.reads_fixed(g, 3000, 150, seed=10))
    C = kache.Counter(100_000)
    O = oracle.OracleTable(31, 4, 100_000, 0.9, True)
    uo = O.register()
    C.prime_batch(b)
    O.upsert(uo, b, kache.KEEP, 0, 0)
    for _ in range(3):
        assert C.count_batch(b) == O.update(b, kache.ADD_WRAP, 1)
    assert np.array_equal(C.histogram(100), O.histogram(100))


def test_counter_rejects():
    with pytest.raises(kache.KacheError):
        kache.Counter(1000, k=25)
    with pytest.raises(kache.KacheError):
        kache.Counter(1000, threads=0)
    with pytest.raises(kache.KacheError):
        kache.Counter(1000, threads=129)
    C = kache.Counter(1000)
    with pytest.raises(kache.KacheError):
        C.prime("/nonexistent.fa")
