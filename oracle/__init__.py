"""The checker: the C restatement of kache-hash's table semantics (oracle.c) and, where it was built here, the
reference's own table (ref_table.cpp over the reference headers, under _ref/).

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference legs may
import this package, and only to check results or to time the CPU baseline. The product never uses it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_u64 = ctypes.c_uint64
_vp = ctypes.c_void_p


def _cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            return "avx512f" in f.read()
    except OSError:
        return False


class Oracle:
    """ctypes view of liboracle.so."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle not built: {ORACLE_SO}")
        L = ctypes.CDLL(ORACLE_SO)
        sig = {
            "orc_wang": (_u64, [_u64]),
            "orc_checksum": (ctypes.c_uint8, [_u64]),
            "orc_revcomp": (_u64, [_u64, ctypes.c_int]),
            "orc_minimizer_hash": (_u64, [_u64, ctypes.c_int, ctypes.c_int]),
            "orc_describe": (_u64, [_vp, _u64, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
            "orc_cap_for": (_u64, [_u64, ctypes.c_double, ctypes.c_int]),
            "orc_replay_capacity": (None, [_u64, ctypes.c_double, ctypes.c_int, _vp, _u64, _vp]),
            "orc_fits": (ctypes.c_int, [_u64, ctypes.c_double, ctypes.c_int]),
            "orc_new": (_vp, [ctypes.c_int, ctypes.c_int, _u64, ctypes.c_double, ctypes.c_int]),
            "orc_free": (None, [_vp]),
            "orc_register": (ctypes.c_uint32, [_vp]),
            "orc_upsert": (_u64, [_vp, ctypes.c_uint32, _vp, _vp, _u64, ctypes.c_uint32, _u64, _u64]),
            "orc_upsert_oriented": (_u64, [_vp, ctypes.c_uint32, _vp, _vp, _u64, ctypes.c_uint32, _u64, _u64]),
            "orc_update": (_u64, [_vp, _vp, _vp, _u64, ctypes.c_uint32, _u64]),
            "orc_lookup": (None, [_vp, _vp, _vp, _u64, _vp, _vp, _vp]),
            "orc_count": (None, [_vp, _vp, _vp, _u64, _vp]),
            "orc_count_masked": (None, [_vp, _vp, _vp, _u64, _u64, _u64, _vp]),
            "orc_sum": (None, [_vp, _vp, _vp, _u64, _vp]),
            "orc_get": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_u64)]),
            "orc_size": (_u64, [_vp]),
            "orc_capacity": (_u64, [_vp]),
            "orc_dump": (_u64, [_vp, _vp, _vp]),
            "orc_reduce": (_u64, [_vp, ctypes.c_uint32, _u64]),
            "orc_histogram": (None, [_vp, _u64, _vp]),
            "orc_digest": (None, [_vp, _vp, _u64, _vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        self.L = L


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        _oracle = Oracle()
    return _oracle


def _b(batch):
    return batch.bases.ctypes.data, batch.off.ctypes.data, batch.n


class OracleTable:
    """The exact model: same call surface as kache.Table for the operations the tests compare."""

    def __init__(self, k=31, value_bytes=8, expected_keys=1 << 22, load_factor=0.8, pow2=False, l=None):
        self.o = oracle().L
        self.k, self.vb = k, value_bytes
        self.l = l if l is not None else {31: 22, 27: 16, 32: 20}[k]
        self.h = self.o.orc_new(k, value_bytes, expected_keys, load_factor, 1 if pow2 else 0)

    def __del__(self):
        try:
            self.o.orc_free(self.h)
        except Exception:
            pass

    def register(self):
        return self.o.orc_register(self.h)

    def insert(self, user, b, op=0, x=0):
        return self.o.orc_upsert(self.h, user, *_b(b), op, x, x)

    def upsert(self, user, b, op, x, init):
        return self.o.orc_upsert(self.h, user, *_b(b), op, x, init)

    def insert_oriented(self, user, b, op, x_fwd, x_rev, capi=True):
        return self.o.orc_upsert_oriented(self.h, user, *_b(b), op, x_fwd, x_rev)

    def update(self, b, op, x, capi=True):
        return self.o.orc_update(self.h, *_b(b), op, x)

    def lookup(self, b, values=True, fwd=True):
        P = int(b.positions(self.k).sum())
        found = np.zeros(max(P, 1), np.uint8)
        vals = np.zeros(max(P, 1), np.uint64)
        fw = np.zeros(max(P, 1), np.uint8)
        self.o.orc_lookup(self.h, *_b(b), found.ctypes.data, vals.ctypes.data, fw.ctypes.data)
        return found[:P], vals[:P], fw[:P]

    def count(self, b):
        out = np.zeros(max(b.n, 1), np.uint64)
        self.o.orc_count(self.h, *_b(b), out.ctypes.data)
        return out[:b.n]

    def count_masked(self, b, mf, mr):
        out = np.zeros(max(b.n, 1), np.uint64)
        self.o.orc_count_masked(self.h, *_b(b), mf, mr, out.ctypes.data)
        return out[:b.n]

    def sum(self, b):
        out = np.zeros(max(b.n, 1), np.uint64)
        self.o.orc_sum(self.h, *_b(b), out.ctypes.data)
        return out[:b.n]

    def get(self, kmer):
        v = _u64()
        kmer = kmer.encode() if isinstance(kmer, str) else kmer
        return bool(self.o.orc_get(self.h, kmer, ctypes.byref(v))), v.value

    def size(self):
        return self.o.orc_size(self.h)

    def capacity(self):
        return self.o.orc_capacity(self.h)

    def dump(self):
        n = self.size()
        keys = np.zeros(max(n, 1), np.uint64)
        vals = np.zeros(max(n, 1), np.uint64)
        c = self.o.orc_dump(self.h, keys.ctypes.data, vals.ctypes.data)
        return keys[:c], (vals[:c] if self.vb else None)

    def reduce(self, what, mask=0xFFFFFFFFFFFFFFFF):
        return self.o.orc_reduce(self.h, what, mask)

    def histogram(self, max_count):
        h = np.zeros(max_count + 1, np.uint64)
        self.o.orc_histogram(self.h, max_count, h.ctypes.data)
        return h


def digest(keys, values=None):
    """Order-independent digest of the (key, value) pairs of a dump (orc_digest): (count, sum1, sum2)."""
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    v = None if values is None else np.ascontiguousarray(values, dtype=np.uint64)
    out = np.zeros(3, np.uint64)
    oracle().L.orc_digest(k.ctypes.data, None if v is None else v.ctypes.data, len(k), out.ctypes.data)
    return tuple(int(x) for x in out)


def describe(batch, k, l):
    """The restated describer over a batch, laid out as the lookups: (key, h, cs, fwd, valid)."""
    o = oracle().L
    P = int(batch.positions(k).sum())
    n = max(P, 1)
    key, h = np.zeros(n, np.uint64), np.zeros(n, np.uint64)
    cs, fw, va = np.zeros(n, np.uint8), np.zeros(n, np.uint8), np.zeros(n, np.uint8)
    at = 0
    for i in range(batch.n):
        s, e = int(batch.off[i]), int(batch.off[i + 1])
        if e - s < k:
            continue
        c = o.orc_describe(batch.bases.ctypes.data + s, e - s, k, l, key.ctypes.data + 8 * at, h.ctypes.data + 8 * at,
                           cs.ctypes.data + at, fw.ctypes.data + at, va.ctypes.data + at)
        at += c
    return key[:P], h[:P], cs[:P], fw[:P], va[:P]


# ---- The reference's own table (built here from its sources; absent where it was not built) ----

REF_KINDS = {(31, 8): 0, (31, 4): 1, (31, 2): 2, (31, 1): 3, (31, 0): 4, (27, 1): 5, (32, 0): 6, (27, 8): 7}


def ref_lib_path():
    if os.environ.get("KACHE_REF_LIB"):
        return os.environ["KACHE_REF_LIB"]
    v4 = os.path.join(REF_DIR, "libkache_ref_v4.so")
    v3 = os.path.join(REF_DIR, "libkache_ref_v3.so")
    if _cpu_has_avx512() and os.path.exists(v4):
        return v4
    return v3 if os.path.exists(v3) else None


_ref = None


def ref():
    """The reference's table library, or None if it was not built."""
    global _ref
    if _ref is None:
        p = ref_lib_path()
        if p is None:
            return None
        L = ctypes.CDLL(p)
        sig = {
            "ref_new": (_vp, [ctypes.c_uint32, _u64, ctypes.c_double, ctypes.c_int, ctypes.c_uint]),
            "ref_free": (None, [_vp]),
            "ref_register": (ctypes.c_uint32, [_vp]),
            "ref_upsert": (_u64, [_vp, ctypes.c_uint32, _vp, _vp, _u64, ctypes.c_uint32, _u64]),
            "ref_upsert_oriented": (_u64, [_vp, ctypes.c_uint32, _vp, _vp, _u64, ctypes.c_uint32, _u64, _u64]),
            "ref_update": (_u64, [_vp, _vp, _vp, _u64, ctypes.c_uint32, _u64]),
            "ref_lookup": (None, [_vp, _vp, _vp, _u64, _vp, _vp, _vp, _vp]),
            "ref_count": (_u64, [_vp, _vp, _vp, _u64]),
            "ref_get": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_u64)]),
            "ref_size": (_u64, [_vp]),
            "ref_capacity": (_u64, [_vp]),
            "ref_overflow_size": (_u64, [_vp]),
            "ref_dump": (_u64, [_vp, _vp, _vp]),
            "ref_bench_upsert": (ctypes.c_double, [_vp, _vp, _vp, _u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u64, ctypes.POINTER(_u64)]),
            "ref_bench_count": (ctypes.c_double, [_vp, _vp, _vp, _u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(_u64)]),
            "ref_bench_upsert_oriented": (ctypes.c_double, [_vp, _vp, _vp, _u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u64, _u64, ctypes.POINTER(_u64)]),
            "ref_bench_update": (ctypes.c_double, [_vp, _vp, _vp, _u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u64, ctypes.POINTER(_u64)]),
            "ref_bench_lookup": (ctypes.c_double, [_vp, _vp, _vp, _u64, _vp, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _ref = L
    return _ref


class RefTable:
    """The reference's Streaming_Kmer_Hash_Table<k, true, V, l>, through ref_table.cpp."""

    def __init__(self, k=31, value_bytes=8, expected_keys=1 << 22, load_factor=0.8, pow2=False, workers=4):
        self.L = ref()
        if self.L is None:
            raise RuntimeError("the reference library was not built")
        self.k, self.vb = k, value_bytes
        self.h = self.L.ref_new(REF_KINDS[(k, value_bytes)], expected_keys, load_factor, 1 if pow2 else 0, workers)

    def __del__(self):
        try:
            self.L.ref_free(self.h)
        except Exception:
            pass

    def register(self):
        return self.L.ref_register(self.h)

    def upsert(self, user, b, op, x, init=None):
        assert init is None or init == x
        return self.L.ref_upsert(self.h, user, *_b(b), op, x)

    insert = upsert

    def insert_oriented(self, user, b, op, x_fwd, x_rev, capi=True):
        return self.L.ref_upsert_oriented(self.h, user, *_b(b), op, x_fwd, x_rev)

    def update(self, b, op, x, capi=True):
        return self.L.ref_update(self.h, *_b(b), op, x)

    def lookup(self, b):
        k = self.k
        lens = np.diff(b.off).astype(np.int64)
        npos = np.maximum(lens - k + 1, 0).astype(np.uint64)
        pos_off = np.zeros(b.n + 1, np.uint64)
        np.cumsum(npos, out=pos_off[1:])
        P = int(pos_off[-1])
        found = np.full(max(P, 1), 2, np.uint8)
        vals = np.zeros(max(P, 1), np.uint64)
        fw = np.zeros(max(P, 1), np.uint8)
        self.L.ref_lookup(self.h, *_b(b), pos_off.ctypes.data, found.ctypes.data, vals.ctypes.data, fw.ctypes.data)
        return found[:P], vals[:P], fw[:P]

    def get(self, kmer):
        v = _u64()
        kmer = kmer.encode() if isinstance(kmer, str) else kmer
        return bool(self.L.ref_get(self.h, kmer, ctypes.byref(v))), v.value

    def size(self):
        return self.L.ref_size(self.h)

    def capacity(self):
        return self.L.ref_capacity(self.h)

    def raw_dump(self):
        """(keys, values) in the reference's for_each order; values None for a set."""
        n = self.size()
        keys = np.zeros(max(n, 1), np.uint64)
        vals = np.zeros(max(n, 1), np.uint64)
        c = self.L.ref_dump(self.h, keys.ctypes.data, vals.ctypes.data)
        return keys[:c], (vals[:c] if self.vb else None)

    def dump(self):
        keys, vals = self.raw_dump()
        o = np.argsort(keys, kind="stable")
        return keys[o], (vals[o] if self.vb else None)

    # The reference's benchmark drivers (ref_bench_*): batches of `batch` sequences over `threads` threads, each
    # upserting thread a user of its own. Return (seconds, result).
    def bench_upsert(self, b, op, x, threads, batch=64):
        out = _u64()
        s = self.L.ref_bench_upsert(self.h, *_b(b), batch, threads, op, x, ctypes.byref(out))
        return s, out.value

    def bench_update(self, b, op, x, threads, batch=64):
        out = _u64()
        s = self.L.ref_bench_update(self.h, *_b(b), batch, threads, op, x, ctypes.byref(out))
        return s, out.value


_ref_capi = None


def ref_capi():
    """The reference's own C interface (capi/*.cpp compiled by oracle/Makefile's `capi` target into
    _ref/libkache_capi_ref.so) with the prototypes of kache_capi.h, or None where it was not built. Loaded with local
    symbol binding, so it lives beside the B200 library in one process, each answering its own calls."""
    global _ref_capi
    if _ref_capi is None:
        p = os.path.join(REF_DIR, "libkache_capi_ref.so")
        if not os.path.exists(p):
            return None
        import kache
        _ref_capi = kache.bind(ctypes.CDLL(p, mode=os.RTLD_LOCAL), kache.CAPI_SIGS)
    return _ref_capi


def replay_capacity(n, lf, pow2, inserted):
    """The capacity after each call of one user whose calls inserted `inserted` keys (orc_replay_capacity)."""
    ins = np.ascontiguousarray(inserted, dtype=np.uint64)
    caps = np.zeros(max(len(ins), 1), np.uint64)
    oracle().L.orc_replay_capacity(n, lf, 1 if pow2 else 0, ins.ctypes.data, len(ins), caps.ctypes.data)
    return caps[:len(ins)]
