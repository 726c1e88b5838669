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
    t.count_dev(d_bases.data_ptr(), d_off.data_ptr(), q.n, expect.data_ptr())
    torch.cuda.synchronize()
    assert int(expect.sum()) > 0
    assert np.array_equal(expect.cpu().numpy().view(np.uint64), t.count(q))

    f = _noalloc()
    for _ in range(2):
        got = torch.full((q.n,), -1, dtype=torch.int64, device=dev)
        assert f(t.h, d_bases.data_ptr(), d_off.data_ptr(), q.n, got.data_ptr()) == kache.KACHE_OK
        assert torch.equal(got, expect)


def test_noalloc_rejects_beyond_maximum():
    import torch
    t = kache.Table(31, 8, 1000)
    dev = torch.device("cuda", 0)
    d = torch.zeros(16, dtype=torch.int64, device=dev)
    # Rejected before any work: the pointers are never read.
    assert _noalloc()(t.h, d.data_ptr(), d.data_ptr(), MAX_SEGMENTS + 1, d.data_ptr()) == kache.KACHE_EINVAL
