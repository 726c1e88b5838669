"""The device memory roofs (kache_b200_memory_roof), the GPU analog of the reference's tools/memory-roof.cpp: each
kind runs and reports a positive rate, the random-sector read rate stays below the sequential one in bytes, and
argument errors are rejected."""
import pytest

import kache

pytestmark = pytest.mark.gpu

MB = 1 << 20


def test_roofs_run_and_order():
    _, seq = kache.memory_roof(512 * MB, kache.ROOF_SEQ_READ, 0)
    _, rd = kache.memory_roof(512 * MB, kache.ROOF_RANDOM_READ, 1 << 24)
    _, up = kache.memory_roof(512 * MB, kache.ROOF_RANDOM_UPDATE, 1 << 24)
    ms, ch = kache.memory_roof(512 * MB, kache.ROOF_CHASE, 148 * 32 * 64)    # 64 dependent loads per thread.
    assert seq > 1e11 and rd > 1e9 and up > 1e9 and ch > 1e6 and ms > 0
    assert rd * 32 < 2 * seq
    # A dependent load from HBM takes between 100 ns and 20 us.
    assert 100 < ms * 1e6 / 64 < 20000


def test_roof_rejects_bad_arguments():
    with pytest.raises(kache.KacheError):
        kache.memory_roof(1024, kache.ROOF_SEQ_READ, 0)
    with pytest.raises(kache.KacheError):
        kache.memory_roof(64 * MB, 7, 1 << 20)
    with pytest.raises(kache.KacheError):
        kache.memory_roof(64 * MB, kache.ROOF_RANDOM_READ, 0)
