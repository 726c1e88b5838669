"""Failure paths, made on the host (include/kache_b200_testing.h), none of which faults or hangs the GPU:

- a device or page-locked allocation that fails surfaces as KACHE_ENOMEM, from kache_new and from an insert that
  needs staging memory, and the table answers correctly once allocations succeed again;
- an insert whose operation must see a racing inserter's value first (KACHE_ASSIGN) meets a claim that is never
  published: the kernel's bounded wait runs out, the kernel ends, and the call returns KACHE_EINTERNAL; an operation
  that commutes (KACHE_ADD) applies itself without waiting and succeeds."""
import ctypes
import time

import numpy as np
import pytest

import kache
import oracle
import synth
from kache import Batch, Options

pytestmark = pytest.mark.gpu


def test_allocation_failure_is_enomem():
    L = kache.lib()
    o = Options(31, 8, 100_000, 0.8, 16, 0)
    h = ctypes.c_void_p()
    try:
        assert L.kache_b200_testing_fail_allocation(0) == kache.KACHE_OK
        assert L.kache_new(ctypes.byref(o), ctypes.byref(h)) == kache.KACHE_ENOMEM and not h.value
    finally:
        L.kache_b200_testing_fail_allocation(-1)
    assert L.kache_new(ctypes.byref(o), ctypes.byref(h)) == kache.KACHE_OK
    L.kache_free(h)

    # An insert into a fresh set, whose first call allocates its staging memory: every allocation of the call in turn
    # fails, until the call gets through; inserting the keys again then leaves the set the oracle makes.
    g = synth.genome(300_000, seed=71)
    b = Batch(*synth.reads_fixed(g, 20_000, 150, seed=72))
    T = kache.Table(31, 0, 400_000)
    u = T.register()
    codes = []
    for after in range(64):
        L.kache_b200_testing_fail_allocation(after)
        r = ctypes.c_uint64()
        codes.append(L.kache_insert(T.h, u, *b.args(), kache.KEEP, 0, ctypes.byref(r)))
        L.kache_b200_testing_fail_allocation(-1)
        if codes[-1] == kache.KACHE_OK:
            break
    assert codes[0] == kache.KACHE_ENOMEM and codes[-1] == kache.KACHE_OK
    assert set(codes[:-1]) == {kache.KACHE_ENOMEM}
    T.insert(u, b)
    O = oracle.OracleTable(31, 0, 400_000)
    O.insert(O.register(), b)
    assert np.array_equal(T.dump()[0], O.dump()[0])
    f, _, _ = T.lookup(b, values=False, fwd=False)
    fo, _, _ = O.lookup(b)
    assert np.array_equal(f, fo)
    T.close()


def _planted(op, wait_polls=1000):
    """A map with some keys, a k-mer of a new read claimed and left unpublished, then an insert of that read."""
    g = synth.genome(100_000, seed=73)
    T = kache.Table(31, 8, 200_000)
    u = T.register()
    T.insert(u, Batch(*synth.reads_fixed(g, 2000, 150, seed=74)), kache.ADD, 1)
    acgt = np.frombuffer(b"ACGT", np.uint8)
    rng = np.random.default_rng(75)
    read = acgt[rng.integers(0, 4, 60)].tobytes()
    assert kache.lib().kache_b200_testing_plant_claim(T.h, read[10:41], wait_polls) == kache.KACHE_OK
    r = ctypes.c_uint64()
    t0 = time.perf_counter()
    code = kache.lib().kache_insert(T.h, u, *Batch.of([read]).args(), op, 5, ctypes.byref(r))
    return code, time.perf_counter() - t0, T


def test_unpublished_claim_ends_the_wait_with_einternal():
    code, seconds, T = _planted(kache.ASSIGN)
    assert code == kache.KACHE_EINTERNAL
    assert seconds < 30     # The kernel ended on its own bound.
    T.close()


def test_commuting_insert_does_not_wait():
    code, _, T = _planted(kache.ADD)
    assert code == kache.KACHE_OK
    T.close()


def test_plant_rejects_present_and_invalid_kmers():
    g = synth.genome(50_000, seed=76)
    b = Batch(*synth.reads_fixed(g, 500, 150, seed=77))
    T = kache.Table(31, 8, 100_000)
    T.insert(T.register(), b, kache.ADD, 1)
    L = kache.lib()
    present = bytes(b.bases[int(b.off[0]):int(b.off[0]) + 31])
    if b"N" not in present:
        assert L.kache_b200_testing_plant_claim(T.h, present, 10) == kache.KACHE_EINVAL
    assert L.kache_b200_testing_plant_claim(T.h, b"ACGTN" * 7, 10) == kache.KACHE_EINVAL
    assert L.kache_b200_testing_plant_claim(None, b"A" * 31, 10) == kache.KACHE_EINVAL
    T.close()
