"""Page-locked caller buffers: reads laid end to end in page-locked memory are copied to the device as they lie, and
lookup outputs in page-locked memory are written by the kernel directly; the results are the same as with pageable
buffers, bit for bit."""
import numpy as np
import pytest
import torch

import kache
import synth
from kache import Batch

pytestmark = pytest.mark.gpu


def pinned_like(a):
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    v = t.numpy().view(a.dtype)
    v[:] = a
    return t, v


def test_pinned_inputs_and_outputs_match_pageable():
    g = synth.genome(300_000, seed=9)
    b = Batch(*synth.reads_fixed(g, 30_000, 150, seed=10, n_rate=0.002))
    t_in, pb_bases = pinned_like(b.bases)
    pb = Batch(pb_bases, b.off)

    A = kache.Table(31, 8, 100_000, 0.8, False)
    B = kache.Table(31, 8, 100_000, 0.8, False)
    ua, ub = A.register(), B.register()
    assert A.insert(ua, b, kache.ADD, 1) == B.insert(ub, pb, kache.ADD, 1)
    ka, va = A.dump()
    kb, vb = B.dump()
    np.testing.assert_array_equal(ka, kb)
    np.testing.assert_array_equal(va, vb)

    f, v, w = A.lookup(b, values=True, fwd=True)
    P = len(f)
    tf, pf = pinned_like(np.full(P, 9, np.uint8))
    tv, pv = pinned_like(np.zeros(P, np.uint64))
    tw, pw = pinned_like(np.full(P, 9, np.uint8))
    kache._check(kache.lib().kache_lookup(A.h, *pb.args(), pf.ctypes.data, pv.ctypes.data, pw.ctypes.data), "kache_lookup")
    np.testing.assert_array_equal(pf, f)
    np.testing.assert_array_equal(pv, v)
    np.testing.assert_array_equal(pw, w)
    # Pinned found flags with pageable values: the library falls back to its staged copies for all three.
    v2 = np.zeros(P, np.uint64)
    pf[:] = 9
    kache._check(kache.lib().kache_lookup(A.h, *b.args(), pf.ctypes.data, v2.ctypes.data, None), "kache_lookup")
    np.testing.assert_array_equal(pf, f)
    np.testing.assert_array_equal(v2, v)
    A.close(), B.close()
