"""The count entry point that allocates nothing (kache_b200_count_dev_noalloc) against the one that may allocate
(kache_b200_count_dev), through the C interface.

Callers inside their own memory pool, inside a CUDA graph capture, or in a process that budgets all of HBM itself
cannot have the library call cudaMalloc when they query; the no-allocation variant keeps its scratch in a fixed
device array instead. Its per-sequence counts must equal the allocating entry point's exactly (they are integers),
on two calls in a row, since every call reuses, and first clears, the same scratch. This file is collected last.
"""
import ctypes

import numpy as np
import pytest

import kache
import synth
from kache import Batch

pytestmark = pytest.mark.gpu

MAX_SEGMENTS = 1048544


def _noalloc():
    f = kache.lib().kache_b200_count_dev_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    return f


@pytest.mark.parametrize("value_bytes", [8, 0])
def test_noalloc_count_equals_count_dev(value_bytes):
    import torch
    g = synth.genome(200_000, seed=41)
    build = Batch(*synth.reads_fixed(g, 20_000, 150, seed=42))
    # Queries of ragged lengths, from shorter than k to several segments.
    q = Batch(*synth.reads_variable(g, 1.0, 150, 1.0, 5, 4000, seed=43))
    t = kache.Table(31, value_bytes, 500_000)
    u = t.register()
    t.insert(u, build, kache.ADD if value_bytes else kache.KEEP, 1 if value_bytes else 0)

    dev = torch.device("cuda", 0)
    d_bases = torch.from_numpy(q.bases).to(dev)
    d_off = torch.from_numpy(q.off.view(np.int64)).to(dev)
    expect = torch.zeros(q.n, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()    # The table runs on its own stream: the fill must land first.
    t.count_dev(d_bases.data_ptr(), d_off.data_ptr(), q.n, expect.data_ptr())
    torch.cuda.synchronize()
    assert int(expect.sum()) > 0
    assert np.array_equal(expect.cpu().numpy().view(np.uint64), t.count(q))

    f = _noalloc()
    for _ in range(2):
        got = torch.full((q.n,), -1, dtype=torch.int64, device=dev)
        torch.cuda.synchronize()    # The table runs on its own stream: the fill must land first.
        assert f(t.h, d_bases.data_ptr(), d_off.data_ptr(), q.n, got.data_ptr()) == kache.KACHE_OK
        assert torch.equal(got, expect)


def _device_reads(n, length, seed):
    """n random ACGT reads of `length` bases, generated on the device: (bases, offsets)."""
    import torch
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    acgt = torch.tensor(list(b"ACGT"), dtype=torch.uint8, device=dev)
    bases = acgt[torch.randint(0, 4, (n * length + 16,), generator=g, device=dev)]
    off = torch.arange(n + 1, dtype=torch.int64, device=dev) * length
    torch.cuda.synchronize()    # Made on torch's stream; the table runs on its own.
    return bases, off


def test_noalloc_segments_beyond_maximum():
    """A batch of few enough sequences whose segments do not fit the scratch: KACHE_EINVAL after listing, nothing
    counted, nothing written past d_counts[n), and the next call that fits counts as kache_b200_count_dev does. A call
    before it leaves the scratch full of segments of sequences that the overflowing batch does not have."""
    import torch
    g = synth.genome(200_000, seed=44)
    build = Batch(*synth.reads_fixed(g, 20_000, 150, seed=45))
    t = kache.Table(31, 8, 500_000)
    u = t.register()
    t.insert(u, build, kache.ADD, 1)
    size = t.size()
    dev = torch.device("cuda", 0)
    f = _noalloc()

    # 1,000,000 sequences of one segment each: entries 0..999,999 name sequences up to 999,999.
    b1, o1 = _device_reads(1_000_000, 100, seed=46)
    c1 = torch.full((1_000_000,), -1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    assert f(t.h, b1.data_ptr(), o1.data_ptr(), 1_000_000, c1.data_ptr()) == kache.KACHE_OK
    assert int(c1.min()) >= 0
    del b1, o1, c1

    # 530,000 sequences of 543 bases: 513 positions, two segments each, 1,060,000 segments in all.
    n2 = 530_000
    assert n2 <= MAX_SEGMENTS < 2 * n2
    b2, o2 = _device_reads(n2, 543, seed=47)
    canary = 0x5A5A5A5A5A5A5A5A
    c2 = torch.full((n2 + 64,), canary, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    assert f(t.h, b2.data_ptr(), o2.data_ptr(), n2, c2.data_ptr()) == kache.KACHE_EINVAL
    torch.cuda.synchronize()
    assert int(c2[:n2].abs().max()) == 0
    assert bool((c2[n2:] == canary).all())
    del b2, o2, c2
    assert t.size() == size

    q = Batch(*synth.reads_variable(g, 1.0, 150, 1.0, 5, 4000, seed=48))
    d_bases = torch.from_numpy(q.bases).to(dev)
    d_off = torch.from_numpy(q.off.view(np.int64)).to(dev)
    expect = torch.zeros(q.n, dtype=torch.int64, device=dev)
    got = torch.full((q.n,), -1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    t.count_dev(d_bases.data_ptr(), d_off.data_ptr(), q.n, expect.data_ptr())
    assert f(t.h, d_bases.data_ptr(), d_off.data_ptr(), q.n, got.data_ptr()) == kache.KACHE_OK
    torch.cuda.synchronize()
    assert int(expect.sum()) > 0
    assert torch.equal(got, expect)


def test_noalloc_rejects_beyond_maximum():
    import torch
    t = kache.Table(31, 8, 1000)
    dev = torch.device("cuda", 0)
    d = torch.zeros(16, dtype=torch.int64, device=dev)
    # Rejected before any work: the pointers are never read.
    assert _noalloc()(t.h, d.data_ptr(), d.data_ptr(), MAX_SEGMENTS + 1, d.data_ptr()) == kache.KACHE_EINVAL
