"""Page-locked caller buffers: reads laid end to end in page-locked memory are copied to the device as they lie, and
lookup outputs in page-locked memory are copied there piece by piece while the next piece computes (batches of at
least 2^22 positions); the results are the same as with pageable buffers, bit for bit."""
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
    b = Batch(*synth.reads_fixed(g, 40_000, 150, seed=10, n_rate=0.002))
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


def test_pinned_lookup_pieces_of_ragged_reads():
    """Reads of uneven lengths (some shorter than k) in page-locked memory, more than 2^22 positions: the lookup runs
    in pieces of sequences whose outputs land at their own positions."""
    g = synth.genome(400_000, seed=11)
    build = Batch(*synth.reads_fixed(g, 20_000, 150, seed=12))
    q = Batch(*synth.reads_variable(g, 30.0, 400, 1.0, 5, 5000, seed=13))
    assert int(q.positions(31).sum()) >= 1 << 22
    t_in, qb = pinned_like(q.bases)
    pq = Batch(qb, q.off)
    T = kache.Table(31, 4, 200_000, 0.8, False)
    T.insert(T.register(), build, kache.ADD, 1)
    f, v, w = T.lookup(q, values=True, fwd=True)
    P = len(f)
    tf, pf = pinned_like(np.full(P, 9, np.uint8))
    tv, pv = pinned_like(np.full(P, 7, np.uint32))
    tw, pw = pinned_like(np.full(P, 9, np.uint8))
    kache._check(kache.lib().kache_lookup(T.h, *pq.args(), pf.ctypes.data, pv.ctypes.data, pw.ctypes.data), "kache_lookup")
    np.testing.assert_array_equal(pf, f)
    np.testing.assert_array_equal(pv, v)
    np.testing.assert_array_equal(pw, w)
    assert (f == 1).sum() > 0 and (f == 0).sum() > 0
    T.close()
