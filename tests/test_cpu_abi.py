"""The C-interface library without a GPU: it loads, exports every function include/*.h declares, and validates
arguments before any device work, answering as the reference's capi/kache_capi.cpp does."""
import ctypes
import os
import re

import pytest

import kache

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in ("kache_capi.h", "kache_b200.h", "kache_b200_testing.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"\b(kache_\w+)\s*\([^;]*\)\s*KACHE_NOEXCEPT\s*;", src)
    return sorted(set(names))


def test_exports_every_declared_function():
    L = kache.lib()
    names = declared()
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_supports_and_defaults():
    L = kache.lib()
    assert all(L.kache_supports(31, w) for w in (0, 1, 2, 4, 8))
    assert not any(L.kache_supports(k, w) for k, w in ((25, 0), (31, 3), (31, 16), (32, 8)))
    o = L.kache_default_options(31, 4)
    assert (o.k, o.value_bytes, o.expected_keys, o.load_factor, o.resize_workers, o.pow2_capacity) == (31, 4, 1 << 22, 0.8, 16, 0)


def test_new_rejects_before_any_device_work():
    """capi.cpp:411-440: null arguments, unsupported tables, load factors, worker counts, sizing, tables beyond the
    most buckets."""
    L = kache.lib()
    h = ctypes.c_void_p()
    o = L.kache_default_options(31, 4)
    assert L.kache_new(ctypes.byref(o), None) == kache.KACHE_EINVAL
    assert L.kache_new(None, ctypes.byref(h)) == kache.KACHE_EINVAL and not h.value
    for k, w in ((25, 4), (31, 3)):
        x = L.kache_default_options(31, 4)
        x.k, x.value_bytes = k, w
        assert L.kache_new(ctypes.byref(x), ctypes.byref(h)) == kache.KACHE_EINVAL and not h.value
    for lf in (0.0, 1.0, 1.5, float("nan")):
        x = L.kache_default_options(31, 4)
        x.load_factor = lf
        assert L.kache_new(ctypes.byref(x), ctypes.byref(h)) == kache.KACHE_EINVAL
    x = L.kache_default_options(31, 4)
    x.resize_workers = 0
    assert L.kache_new(ctypes.byref(x), ctypes.byref(h)) == kache.KACHE_EINVAL
    x = L.kache_default_options(31, 4)
    x.pow2_capacity = 2
    assert L.kache_new(ctypes.byref(x), ctypes.byref(h)) == kache.KACHE_EINVAL
    for n, p in ((1 << 37, 0), (55 << 30, 1), (0xFFFFFFFFFFFFFFFF, 0)):
        x = L.kache_default_options(31, 4)
        x.expected_keys, x.pow2_capacity = n, p
        assert L.kache_new(ctypes.byref(x), ctypes.byref(h)) == kache.KACHE_EINVAL and not h.value
    assert L.kache_b200_new(25, 22, 8, 1000, 0.8, 0, ctypes.byref(h)) == kache.KACHE_EINVAL
    assert L.kache_b200_new(31, 20, 8, 1000, 0.8, 0, ctypes.byref(h)) == kache.KACHE_EINVAL


def test_null_table_and_strerror():
    L = kache.lib()
    L.kache_free(None)
    u = ctypes.c_uint32()
    assert L.kache_register(None, ctypes.byref(u)) == kache.KACHE_EINVAL
    assert L.kache_insert(None, 0, None, None, 0, 0, 0, None) == kache.KACHE_EINVAL
    assert L.kache_count(None, None, None, 0, None) == kache.KACHE_EINVAL
    assert L.kache_lookup(None, None, None, 0, None, None, None) == kache.KACHE_EINVAL
    assert L.kache_size(None, None) == kache.KACHE_EINVAL
    assert L.kache_get_stats(None, None) == kache.KACHE_EINVAL
    assert L.kache_b200_clear(None) == kache.KACHE_EINVAL
    t = ctypes.c_uint64()
    assert L.kache_b200_server_submit(None, 0, None, None, 0, 0, 0, 0, None, None, None, ctypes.byref(t)) == kache.KACHE_EINVAL
    assert L.kache_b200_server_submit_dev(None, 0, None, None, 0, 0, 0, 0, None, None, None, ctypes.byref(t)) == kache.KACHE_EINVAL
    names = {0: b"success", 1: b"invalid argument", 2: b"too many users registered", 3: b"out of memory", 4: b"internal error", 9: b"unknown status"}
    for c, s in names.items():
        assert L.kache_strerror(c) == s


def test_no_cpu_fallback_without_gpu():
    """Without a GPU a table cannot be made: the library reports an error instead of computing on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(kache.KacheError) as e:
        kache.Table(31, 8, 1000)
    assert e.value.code == kache.KACHE_EINTERNAL


def test_exports_the_counter_class():
    """The counter's C++ surface (include/Kmer_Set_Counter.hpp): every member of the reference's class is exported by
    the library, with the reference's signatures (counter/Kmer_Set_Counter.hpp:41-74)."""
    import subprocess
    lib = os.path.join(ROOT, "kache-hash_b200", "_build", "libkache_b200.so")
    out = subprocess.run(["nm", "-DC", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    for sig in ("kache_hash::Kmer_Set_Counter::supports(unsigned short)",
                "kache_hash::Kmer_Set_Counter::Kmer_Set_Counter(unsigned short, unsigned long, unsigned long, double)",
                "kache_hash::Kmer_Set_Counter::~Kmer_Set_Counter()",
                "kache_hash::Kmer_Set_Counter::prime(std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> > const&)",
                "kache_hash::Kmer_Set_Counter::count(std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> > const&)",
                "kache_hash::Kmer_Set_Counter::histogram(unsigned long)",
                "kache_hash::Kmer_Set_Counter::count_of(char const*) const",
                "kache_hash::Kmer_Set_Counter::size() const",
                "kache_hash::Kmer_Set_Counter::timings() const"):
        assert sig in out, sig
