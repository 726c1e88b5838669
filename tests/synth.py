"""Seeded synthetic genomes and reads with the shapes of the benchmark workloads.

The reference measures on real genomes and read sets (E. coli, chr21, CHM13, SRR5833294; kache-hash
scripts/data.sha256) that are not available here; these generators stand in for them with the workloads' stated
shapes: uniform genomes, segmental duplications, reads of fixed or log-normal lengths, reverse complements,
substitutions, insertions, deletions and N's. Everything is numpy and deterministic per seed.
"""
import numpy as np

ASCII = np.frombuffer(b"ACGTN", dtype=np.uint8)


def genome(n, seed, dup_frac=0.0, dup_len=(1000, 20000), dup_div=0.02):
    """A uniform random genome of n bases as codes 0..3; with dup_frac > 0, that share of it is made of copies of
    earlier stretches of dup_len bases, each mutated at rate dup_div (segmental duplications)."""
    rng = np.random.default_rng(seed)
    g = rng.integers(0, 4, size=n, dtype=np.uint8)
    if dup_frac > 0:
        target = int(n * dup_frac)
        done = 0
        while done < target:
            L = int(rng.integers(dup_len[0], dup_len[1] + 1))
            src = int(rng.integers(0, n - L))
            dst = int(rng.integers(0, n - L))
            piece = g[src:src + L].copy()
            m = rng.random(L) < dup_div
            piece[m] = (piece[m] + rng.integers(1, 4, size=int(m.sum()), dtype=np.uint8)) % 4
            g[dst:dst + L] = piece
            done += L
    return g


def _pack(reads):
    lens = np.array([len(r) for r in reads], dtype=np.uint64)
    off = np.zeros(len(reads) + 1, np.uint64)
    np.cumsum(lens, out=off[1:])
    bases = np.concatenate(reads) if reads else np.zeros(0, np.uint8)
    return np.concatenate([bases, np.zeros(16, np.uint8)]), off


def reads_fixed(g, n, length, seed, rc=0.5, sub=0.005, n_rate=0.0005, chunk=200000):
    """n reads of `length` bases at uniform starts: (bases ASCII uint8, offsets uint64[n+1])."""
    rng = np.random.default_rng(seed)
    win = np.lib.stride_tricks.sliding_window_view(g, length)
    parts = []
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        st = rng.integers(0, len(g) - length + 1, size=m)
        r = win[st].copy()
        flip = rng.random(m) < rc
        r[flip] = 3 - r[flip][:, ::-1]
        if sub > 0:
            mask = rng.random(r.shape) < sub
            r[mask] = (r[mask] + rng.integers(1, 4, size=int(mask.sum()), dtype=np.uint8)) % 4
        if n_rate > 0:
            r[rng.random(r.shape) < n_rate] = 4
        parts.append(ASCII[r].reshape(-1))
    bases = np.concatenate(parts) if parts else np.zeros(0, np.uint8)
    off = np.arange(n + 1, dtype=np.uint64) * np.uint64(length)
    return np.concatenate([bases, np.zeros(16, np.uint8)]), off


def reads_variable(g, coverage, median, sigma, lo, hi, seed, rc=0.5, sub=0.005, ins=0.0, dele=0.0, n_rate=0.0005, max_reads=None):
    """Reads of log-normal lengths (median, sigma) clipped to [lo, hi], to `coverage` x of g, with substitutions,
    insertions and deletions at the given per-base rates and N's; as (bases, offsets)."""
    rng = np.random.default_rng(seed)
    total = int(len(g) * coverage)
    reads, got = [], 0
    while got < total and (max_reads is None or len(reads) < max_reads):
        L = int(np.clip(rng.lognormal(np.log(median), sigma), lo, hi))
        L = min(L, len(g))
        st = int(rng.integers(0, len(g) - L + 1))
        r = g[st:st + L].copy()
        if ins > 0 or dele > 0:
            u = rng.random(L)
            keep = u >= dele
            r = r[keep]
            u2 = rng.random(len(r))
            at = np.nonzero(u2 < ins)[0]
            if len(at):
                r = np.insert(r, at, rng.integers(0, 4, size=len(at), dtype=np.uint8))
        if sub > 0:
            m = rng.random(len(r)) < sub
            r[m] = (r[m] + rng.integers(1, 4, size=int(m.sum()), dtype=np.uint8)) % 4
        if rng.random() < rc:
            r = 3 - r[::-1]
        if n_rate > 0:
            r = r.copy()
            r[rng.random(len(r)) < n_rate] = 4
        reads.append(ASCII[r])
        got += L
    return _pack(reads)


def reads_lognormal(g, coverage, median, sigma, lo, hi, seed, rc=0.5, sub=0.005, n_rate=0.0005, chunk=1 << 24):
    """Vectorised reads of log-normal lengths clipped to [lo, hi], to `coverage` x of g, with substitutions and N's
    (no indels): as (bases, offsets)."""
    rng = np.random.default_rng(seed)
    total = int(len(g) * coverage)
    est = int(total / (median * np.exp(sigma * sigma / 2))) + 16
    lens = np.clip(rng.lognormal(np.log(median), sigma, size=est * 2), lo, hi).astype(np.int64)
    cut = int(np.searchsorted(np.cumsum(lens), total)) + 1
    lens = np.minimum(lens[:cut], len(g))
    n = len(lens)
    starts = (rng.random(n) * (len(g) - lens + 1)).astype(np.int64)
    flip = rng.random(n) < rc
    off = np.zeros(n + 1, np.uint64)
    np.cumsum(lens, out=off[1:])
    out = np.empty(int(off[-1]) + 16, np.uint8)
    out[-16:] = 0
    # Read i's base j comes from first[i] + j * step[i]: forward from its start, or backward from its end.
    first = starts + np.where(flip, lens - 1, 0)
    step = np.where(flip, -1, 1).astype(np.int64)
    xor = np.where(flip, 3, 0).astype(np.uint8)
    offi = off.astype(np.int64)
    b = 0
    while b < n:
        e = min(n, int(np.searchsorted(off, off[b] + chunk, side="right")))
        e = max(e, b + 1)
        L = lens[b:e]
        rid = np.repeat(np.arange(b, e), L)
        j = np.arange(offi[b], offi[e], dtype=np.int64)
        j -= offi[rid]
        j *= step[rid]
        j += first[rid]
        r = g[j]
        r ^= xor[rid]
        u = rng.integers(0, 1 << 16, size=len(r), dtype=np.uint16)
        if sub > 0:
            m = np.flatnonzero(u < int(sub * 65536))
            r[m] = (r[m] + rng.integers(1, 4, size=len(m), dtype=np.uint8)) % 4
        if n_rate > 0:
            r[(u >= 65535 - int(n_rate * 65536))] = 4
        out[int(off[b]):int(off[e])] = ASCII[r]
        b = e
    return out, off


def stretches(g, length):
    """The genome as pieces of `length` bases (the last one shorter), as (bases, offsets): a 1x streaming of it."""
    n = (len(g) + length - 1) // length
    off = np.minimum(np.arange(n + 1, dtype=np.uint64) * np.uint64(length), np.uint64(len(g)))
    return np.concatenate([ASCII[g], np.zeros(16, np.uint8)]), off


# The counter workload: a 100 Mbp genome, 5 % of it segmental duplications of 1-20 kb at 2 % divergence, primed
# with its 31-mers; counted from 30x reads of log-normal lengths (median 150, sigma 0.6) clipped to 50-1000 bp.
def config2(scale=1.0):
    g = genome(int(100_000_000 * scale), seed=21, dup_frac=0.05, dup_len=(1000, 20000), dup_div=0.02)
    index = stretches(g, 1_000_000)
    reads = reads_lognormal(g, 30, 150, 0.6, 50, 1000, seed=22)
    return g, index, reads


# The oriented workload: a 50 Mbp genome, reads of log-normal lengths (median 10 kb, sigma 0.8) clipped to 1-100 kb at
# 5x, 5 % errors split 3:1:1 substitution:insertion:deletion, half reverse-complemented.
def config3(scale=1.0):
    g = genome(int(50_000_000 * scale), seed=31)
    reads = reads_variable(g, 5, 10_000, 0.8, 1000, 100_000, seed=32, rc=0.5, sub=0.03, ins=0.01, dele=0.01)
    return g, reads


# The resize-heavy set: a 400 Mbp genome streamed as 150 bp pieces at 1x into a set sized for 1M keys.
def config4(scale=1.0):
    g = genome(int(400_000_000 * scale), seed=41)
    return g, stretches(g, 150)


# The served mix: a <31, u32, 22> map primed with a genome's 31-mers (2 Gbp at full size), then requests of 150 bp reads
# with 1 % substitutions, upsert / find / count at 60/30/10, each of lognormal(2000 reads, sigma 1.5) clipped to
# 1-1M reads, drawn from a pool of reads of the genome. Returns the genome, the priming pieces and (kind, batch) per
# request (kind 0 upsert, 1 find, 2 count).
def config5(scale=1.0, requests=300):
    from kache import Batch
    glen = int(2_000_000_000 * scale)
    g = genome(glen, seed=51)
    primer = stretches(g, 1_000_000)
    pool = Batch(*reads_fixed(g, min(4_000_000, max(100_000, glen // 100)), 150, seed=52, sub=0.01, n_rate=0.0005))
    rng = np.random.default_rng(53)
    reqs = []
    for _ in range(requests):
        kind = rng.choice(3, p=[0.6, 0.3, 0.1])
        m = int(np.clip(rng.lognormal(np.log(2000), 1.5), 1, min(1_000_000, pool.n)))
        s = int(rng.integers(0, pool.n - m + 1))
        reqs.append((int(kind), pool.slice(s, s + m)))
    return g, primer, reqs


# The benchmark workload of the headline metric: a map <31, u64, 22> sized for 10M keys; upsert(c + 1, init 1) of
# 333,333 reads of 150 bp at 10x over a 5 Mbp genome (seed 1), then lookups of 1M held-out reads (seed 2).
def config1(scale=1.0):
    g = genome(int(5_000_000 * scale), seed=1)
    ins = reads_fixed(g, int(333_333 * scale), 150, seed=11)
    held = reads_fixed(g, int(1_000_000 * scale), 150, seed=2)
    return g, ins, held
