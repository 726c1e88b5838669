"""Python binding of the B200 kache-hash library, over its C interface (include/kache_capi.h, include/kache_b200.h).

It mirrors the reference's C interface one to one (kache-hash capi/kache_capi.h:111-202) and adds what the C++
template API and the counter offer (include/Streaming_Kmer_Hash_Table.hpp:624-745, counter/Kmer_Set_Counter.hpp).
Batches are numpy arrays: all sequences concatenated in one uint8 buffer, plus n + 1 offsets; they are passed to the
library as the `seqs`/`lens` arrays of the C interface without copies. Statuses other than KACHE_OK raise
`KacheError`. The library is the CUDA build under `_build/`; there is no other implementation behind this module,
so importing it without the built library fails.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# The CUDA library: the in-tree build, or another build of it named by KACHE_B200_LIB.
LIB_PATH = os.environ.get("KACHE_B200_LIB") or os.path.join(HERE, "_build", "libkache_b200.so")

KACHE_OK, KACHE_EINVAL, KACHE_EUSERS, KACHE_ENOMEM, KACHE_EINTERNAL = range(5)
KEEP, ASSIGN, ADD, OR, MIN, MAX = range(6)
ADD_WRAP = 16
REDUCE_KEYS, REDUCE_POPCOUNT, REDUCE_SUM = range(3)
ABSENT, PRESENT, NOT_KMER = range(3)
MAX_USERS = 128

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_vp = ctypes.c_void_p


class KacheError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what}: {code}")
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [("k", ctypes.c_uint32), ("value_bytes", ctypes.c_uint32), ("expected_keys", ctypes.c_uint64),
                ("load_factor", ctypes.c_double), ("resize_workers", ctypes.c_uint32), ("pow2_capacity", ctypes.c_uint32)]


class Stats(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_uint64), ("bytes", ctypes.c_uint64), ("keys", ctypes.c_uint64),
                ("overflow_keys", ctypes.c_uint64), ("primary_pct", ctypes.c_double),
                ("secondary_pct", ctypes.c_double), ("overflow_pct", ctypes.c_double)]


class DevBatch(ctypes.Structure):
    """One batch of kache_b200_run_dev_batches: device pointers to its bases and n + 1 offsets, its output arrays."""
    _fields_ = [("d_bases", _vp), ("d_off", _vp), ("n", ctypes.c_uint64), ("out0", _vp), ("out1", _vp), ("out2", _vp),
                ("result", ctypes.c_uint64)]


RUN_UPSERT, RUN_UPSERT_ORIENTED, RUN_UPDATE, RUN_LOOKUP, RUN_COUNT = range(5)

KEYS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, _u64p, ctypes.c_void_p, ctypes.c_size_t)

# The reference's C interface (capi/kache_capi.h:111-202): prototypes as ctypes signatures.
CAPI_SIGS = {
    "kache_supports": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32]),
    "kache_default_options": (Options, [ctypes.c_uint32, ctypes.c_uint32]),
    "kache_new": (ctypes.c_int, [ctypes.POINTER(Options), ctypes.POINTER(_vp)]),
    "kache_free": (None, [_vp]),
    "kache_register": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint32)]),
    "kache_insert": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, _u64p]),
    "kache_insert_oriented": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u64p]),
    "kache_update": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, _u64p]),
    "kache_count": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "kache_count_masked": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64, _vp]),
    "kache_sum": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, _vp]),
    "kache_lookup": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, _vp, _vp, _vp]),
    "kache_get": (ctypes.c_int, [_vp, ctypes.c_char_p, _u8p, _u64p]),
    "kache_size": (ctypes.c_int, [_vp, _u64p]),
    "kache_reduce": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, _u64p]),
    "kache_for_each": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint32, KEYS_FN, _vp]),
    "kache_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Stats)]),
    "kache_strerror": (ctypes.c_char_p, [ctypes.c_int]),
}


def bind(L, sigs):
    """Sets restype and argtypes of the library's functions named in `sigs`."""
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    return L


_lib = None


def lib():
    """The loaded library; raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"the CUDA library is not built: {LIB_PATH} is missing (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        sig = dict(CAPI_SIGS)
        sig.update({
            "kache_b200_new": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_uint32, ctypes.POINTER(_vp)]),
            "kache_b200_set_stream": (ctypes.c_int, [_vp, _vp]),
            "kache_b200_upsert": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u64p]),
            "kache_b200_upsert_oriented": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u64p]),
            "kache_b200_update": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, _u64p]),
            "kache_b200_upsert_dev": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u64p]),
            "kache_b200_upsert_oriented_dev": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _u64p]),
            "kache_b200_update_dev": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, _u64p]),
            "kache_b200_lookup_dev": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint64, _vp, _vp, _vp]),
            "kache_b200_count_dev": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint64, _vp]),
            "kache_b200_run_dev_batches": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(DevBatch), ctypes.c_size_t]),
            "kache_b200_prepare_dev": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.POINTER(_vp)]),
            "kache_b200_prepared_free": (None, [_vp]),
            "kache_b200_lookup_prepared": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
            "kache_b200_table_epoch": (ctypes.c_int, [_vp, _u64p]),
            "kache_b200_count_prepared": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
            "kache_b200_describe": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_size_t, _vp, _vp, _vp, _vp, _vp]),
            "kache_b200_histogram": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp]),
            "kache_b200_clear": (ctypes.c_int, [_vp]),
            "kache_b200_profile": (ctypes.c_int, [_vp, ctypes.c_int]),
            "kache_b200_profile_read": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double), _u64p]),
            "kache_b200_kernel_launches": (ctypes.c_uint64, []),
            "kache_b200_server_new": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.POINTER(_vp)]),
            "kache_b200_server_free": (None, [_vp]),
            "kache_b200_server_submit": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _vp, _vp, _vp, _u64p]),
            "kache_b200_server_submit_dev": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, _vp, _vp, _vp, _u64p]),
            "kache_b200_server_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, _u64p, ctypes.POINTER(ctypes.c_double)]),
            "kache_b200_server_stats": (ctypes.c_int, [_vp, _u64p, _u64p]),
            "kache_b200_memory_roof": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
            "kache_b200_testing_fail_allocation": (ctypes.c_int, [ctypes.c_int64]),
            "kache_b200_testing_plant_claim": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_uint32]),
        })
        _lib = bind(L, sig)
    return _lib


def _check(code, what):
    if code != KACHE_OK:
        raise KacheError(code, what)


class Batch:
    """Sequences as one concatenated uint8 buffer and n + 1 offsets, viewed as the C interface's seqs/lens arrays."""

    def __init__(self, bases, off):
        self.bases = np.ascontiguousarray(bases, dtype=np.uint8)
        self.off = np.ascontiguousarray(off, dtype=np.uint64)
        self.n = len(self.off) - 1
        base = self.bases.ctypes.data
        self.ptrs = (np.uint64(base) + self.off[:-1]).astype(np.uint64)
        self.lens = np.diff(self.off).astype(np.uint64)
        if self.n == 0:
            self.ptrs = np.zeros(1, np.uint64)
            self.lens = np.zeros(1, np.uint64)

    @classmethod
    def of(cls, seqs):
        """From a list of bytes / str."""
        seqs = [s.encode() if isinstance(s, str) else bytes(s) for s in seqs]
        lens = np.array([len(s) for s in seqs], dtype=np.uint64)
        off = np.zeros(len(seqs) + 1, np.uint64)
        np.cumsum(lens, out=off[1:])
        bases = np.frombuffer(b"".join(seqs) + b"\0", dtype=np.uint8)
        return cls(bases, off)

    def slice(self, b, e):
        return Batch(self.bases[int(self.off[b]):int(self.off[e])], self.off[b:e + 1] - self.off[b])

    def positions(self, k):
        lens = np.diff(self.off).astype(np.int64)
        return np.maximum(lens - k + 1, 0)

    def args(self):
        return self.ptrs.ctypes.data, self.lens.ctypes.data, self.n


def _p(a):
    return None if a is None else a.ctypes.data


class Table:
    """A table of canonical k-mers on the GPU: a set (value_bytes 0) or a map to values of 1, 2, 4 or 8 bytes."""

    VDT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}

    def __init__(self, k=31, value_bytes=8, expected_keys=1 << 22, load_factor=0.8, pow2=False, l=None, capi=None):
        L = lib()
        h = _vp()
        if capi is None:
            capi = (k == 31 and (l is None or l == 22))
        if l is None:
            l = {31: 22, 27: 16, 32: 20}[k]
        if capi:
            o = Options(k, value_bytes, expected_keys, load_factor, 16, 1 if pow2 else 0)
            _check(L.kache_new(ctypes.byref(o), ctypes.byref(h)), "kache_new")
        else:
            _check(L.kache_b200_new(k, l, value_bytes, expected_keys, load_factor, 1 if pow2 else 0, ctypes.byref(h)), "kache_b200_new")
        self.h, self.k, self.l, self.vb = h, k, l, value_bytes
        self.vdt = self.VDT.get(value_bytes, np.uint8)
        self.owned = True

    @classmethod
    def view(cls, h, k, l, value_bytes):
        """A table owned elsewhere (a counter's): usable for queries, never freed through this object."""
        t = cls.__new__(cls)
        t.h, t.k, t.l, t.vb = _vp(h), k, l, value_bytes
        t.vdt = cls.VDT.get(value_bytes, np.uint8)
        t.owned = False
        return t

    def close(self):
        if self.h and self.owned:
            lib().kache_free(self.h)
        self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def register(self):
        u = ctypes.c_uint32()
        _check(lib().kache_register(self.h, ctypes.byref(u)), "kache_register")
        return u.value

    def set_stream(self, stream_ptr):
        _check(lib().kache_b200_set_stream(self.h, stream_ptr), "kache_b200_set_stream")

    def insert(self, user, b, op=KEEP, x=0):
        r = ctypes.c_uint64()
        _check(lib().kache_insert(self.h, user, *b.args(), op, x, ctypes.byref(r)), "kache_insert")
        return r.value

    def upsert(self, user, b, op, x, init):
        r = ctypes.c_uint64()
        _check(lib().kache_b200_upsert(self.h, user, *b.args(), op, x, init, ctypes.byref(r)), "kache_b200_upsert")
        return r.value

    def insert_oriented(self, user, b, op, x_fwd, x_rev, capi=True):
        r = ctypes.c_uint64()
        f = lib().kache_insert_oriented if capi else lib().kache_b200_upsert_oriented
        _check(f(self.h, user, *b.args(), op, x_fwd, x_rev, ctypes.byref(r)), "insert_oriented")
        return r.value

    def update(self, b, op, x, capi=True):
        r = ctypes.c_uint64()
        f = lib().kache_update if capi else lib().kache_b200_update
        _check(f(self.h, *b.args(), op, x, ctypes.byref(r)), "update")
        return r.value

    def count(self, b):
        out = np.zeros(max(b.n, 1), np.uint64)
        _check(lib().kache_count(self.h, *b.args(), out.ctypes.data), "kache_count")
        return out[:b.n]

    def count_masked(self, b, m_fwd, m_rev):
        out = np.zeros(max(b.n, 1), np.uint64)
        _check(lib().kache_count_masked(self.h, *b.args(), m_fwd, m_rev, out.ctypes.data), "kache_count_masked")
        return out[:b.n]

    def sum(self, b):
        out = np.zeros(max(b.n, 1), np.uint64)
        _check(lib().kache_sum(self.h, *b.args(), out.ctypes.data), "kache_sum")
        return out[:b.n]

    def lookup(self, b, values=True, fwd=True):
        P = int(b.positions(self.k).sum())
        found = np.full(max(P, 1), 255, np.uint8)
        vals = np.zeros(max(P, 1), self.vdt) if (values and self.vb) else None
        fw = np.zeros(max(P, 1), np.uint8) if fwd else None
        _check(lib().kache_lookup(self.h, *b.args(), found.ctypes.data, _p(vals), _p(fw)), "kache_lookup")
        return found[:P], (vals[:P] if vals is not None else None), (fw[:P] if fw is not None else None)

    def get(self, kmer):
        f, v = ctypes.c_uint8(), ctypes.c_uint64()
        kmer = kmer.encode() if isinstance(kmer, str) else kmer
        _check(lib().kache_get(self.h, kmer, ctypes.byref(f), ctypes.byref(v)), "kache_get")
        return bool(f.value), v.value

    def size(self):
        r = ctypes.c_uint64()
        _check(lib().kache_size(self.h, ctypes.byref(r)), "kache_size")
        return r.value

    def reduce(self, what, mask=~0 & 0xFFFFFFFFFFFFFFFF, workers=1):
        r = ctypes.c_uint64()
        _check(lib().kache_reduce(self.h, what, mask, workers, ctypes.byref(r)), "kache_reduce")
        return r.value

    def stats(self):
        s = Stats()
        _check(lib().kache_get_stats(self.h, ctypes.byref(s)), "kache_get_stats")
        return s

    def capacity(self):
        return self.stats().capacity

    def for_each(self, shards=1, shard=0, stop_after=None):
        """Returns (keys, values) of the share, unsorted, gathered through the C callback."""
        ks, vs = [], []
        vdt = self.vdt

        def cb(ctx, keys, values, n):
            ks.append(np.ctypeslib.as_array(keys, shape=(n,)).copy())
            if values:
                vs.append(np.ctypeslib.as_array(ctypes.cast(values, ctypes.POINTER(np.ctypeslib.as_ctypes_type(vdt))), shape=(n,)).copy())
            return 1 if (stop_after is not None and sum(len(x) for x in ks) >= stop_after) else 0

        fn = KEYS_FN(cb)
        _check(lib().kache_for_each(self.h, shards, shard, fn, None), "kache_for_each")
        keys = np.concatenate(ks) if ks else np.zeros(0, np.uint64)
        vals = np.concatenate(vs) if vs else (np.zeros(0, vdt) if self.vb else None)
        return keys, vals

    def dump(self):
        """Sorted (keys, values) of the whole table."""
        keys, vals = self.for_each()
        o = np.argsort(keys, kind="stable")
        return keys[o], (vals[o].astype(np.uint64) if vals is not None else None)

    def histogram(self, max_count):
        h = np.zeros(max_count + 1, np.uint64)
        _check(lib().kache_b200_histogram(self.h, max_count, h.ctypes.data), "kache_b200_histogram")
        return h

    def describe(self, b):
        P = int(b.positions(self.k).sum())
        n = max(P, 1)
        key, h = np.zeros(n, np.uint64), np.zeros(n, np.uint64)
        cs, fw, va = np.zeros(n, np.uint8), np.zeros(n, np.uint8), np.zeros(n, np.uint8)
        _check(lib().kache_b200_describe(self.h, *b.args(), key.ctypes.data, h.ctypes.data, cs.ctypes.data, fw.ctypes.data, va.ctypes.data), "describe")
        return key[:P], h[:P], cs[:P], fw[:P], va[:P]

    # Device-resident batches: pointers to device memory (e.g. torch tensors' data_ptr()).
    def upsert_dev(self, user, d_bases, d_off, n, op, x, init):
        r = ctypes.c_uint64()
        _check(lib().kache_b200_upsert_dev(self.h, user, d_bases, d_off, n, op, x, init, ctypes.byref(r)), "upsert_dev")
        return r.value

    def upsert_oriented_dev(self, user, d_bases, d_off, n, op, x_fwd, x_rev):
        r = ctypes.c_uint64()
        _check(lib().kache_b200_upsert_oriented_dev(self.h, user, d_bases, d_off, n, op, x_fwd, x_rev, ctypes.byref(r)), "upsert_oriented_dev")
        return r.value

    def update_dev(self, d_bases, d_off, n, op, x):
        r = ctypes.c_uint64()
        _check(lib().kache_b200_update_dev(self.h, d_bases, d_off, n, op, x, ctypes.byref(r)), "update_dev")
        return r.value

    def lookup_dev(self, d_bases, d_off, n, d_found, d_values=None, d_fwd=None):
        _check(lib().kache_b200_lookup_dev(self.h, d_bases, d_off, n, d_found, d_values, d_fwd), "lookup_dev")

    def prepare_dev(self, d_off, n):
        """Stages the batch shape of the device offsets d_off[0..n] once (kache_b200_prepare_dev); returns the handle
        for lookup_prepared. Free it with prepared_free."""
        p = _vp()
        _check(lib().kache_b200_prepare_dev(self.h, d_off, n, ctypes.byref(p)), "prepare_dev")
        return p

    @staticmethod
    def prepared_free(p):
        lib().kache_b200_prepared_free(p)

    def lookup_prepared(self, p, d_bases, d_found, d_values=None, d_fwd=None):
        """One lookup launch of a batch of the prepared shape on the table's stream; returns before it has run."""
        _check(lib().kache_b200_lookup_prepared(self.h, p, d_bases, d_found, d_values, d_fwd), "lookup_prepared")

    def count_prepared(self, p, d_bases, d_counts):
        """Per-sequence counts of a batch of the prepared shape into d_counts, one launch; returns before it has run."""
        _check(lib().kache_b200_count_prepared(self.h, p, d_bases, d_counts), "count_prepared")

    def epoch(self):
        e = ctypes.c_uint64()
        _check(lib().kache_b200_table_epoch(self.h, ctypes.byref(e)), "table_epoch")
        return e.value

    def count_dev(self, d_bases, d_off, n, d_counts):
        _check(lib().kache_b200_count_dev(self.h, d_bases, d_off, n, d_counts), "count_dev")

    def run_dev_batches(self, kind, batches, op=0, x=0, y=0, user=0):
        """Runs device batches as one call (kache_b200_run_dev_batches). `batches` holds tuples (d_bases, d_off, n[,
        out0[, out1[, out2]]]) of device pointers; returns each batch's result (keys inserted, k-mers present, positions found, or the sum of its counts)."""
        arr = (DevBatch * max(1, len(batches)))()
        for i, b in enumerate(batches):
            outs = list(b[3:]) + [None] * (6 - len(b))
            arr[i] = DevBatch(b[0], b[1], b[2], outs[0], outs[1], outs[2], 0)
        _check(lib().kache_b200_run_dev_batches(self.h, user, kind, op, x, y, arr, len(batches)), "run_dev_batches")
        return [arr[i].result for i in range(len(batches))]

    def clear(self):
        _check(lib().kache_b200_clear(self.h), "kache_b200_clear")

    def profile(self, on=True):
        _check(lib().kache_b200_profile(self.h, 1 if on else 0), "profile")

    def profile_read(self, kind):
        ms, n = ctypes.c_double(), ctypes.c_uint64()
        _check(lib().kache_b200_profile_read(self.h, kind, ctypes.byref(ms), ctypes.byref(n)), "profile_read")
        return ms.value, n.value


class Counter:
    """The counter library (counter/Kmer_Set_Counter.hpp): 31-mers primed at count 0, counted by +1 per occurrence."""

    def __init__(self, n, threads=1, load_factor=0.9, k=31):
        L = lib()
        for name, args in (("kache_counter_new", [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double, ctypes.POINTER(_vp)]),
                           ("kache_counter_free", [_vp]), ("kache_counter_prime", [_vp, ctypes.c_char_p]),
                           ("kache_counter_count", [_vp, ctypes.c_char_p, _u64p]),
                           ("kache_counter_prime_batch", [_vp, _vp, _vp, ctypes.c_size_t]),
                           ("kache_counter_count_batch", [_vp, _vp, _vp, ctypes.c_size_t, _u64p]),
                           ("kache_counter_histogram", [_vp, ctypes.c_uint64, _vp]),
                           ("kache_counter_count_of", [_vp, ctypes.c_char_p, _u64p]),
                           ("kache_counter_size", [_vp, _u64p]), ("kache_counter_table", [_vp])):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None if name == "kache_counter_free" else (_vp if name == "kache_counter_table" else ctypes.c_int)
        h = _vp()
        _check(L.kache_counter_new(k, n, threads, load_factor, ctypes.byref(h)), "kache_counter_new")
        self.h = h

    def close(self):
        if self.h:
            lib().kache_counter_free(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def prime(self, path):
        _check(lib().kache_counter_prime(self.h, path.encode()), "kache_counter_prime")

    def count(self, path):
        r = ctypes.c_uint64()
        _check(lib().kache_counter_count(self.h, path.encode(), ctypes.byref(r)), "kache_counter_count")
        return r.value

    def prime_batch(self, b):
        _check(lib().kache_counter_prime_batch(self.h, *b.args()), "kache_counter_prime_batch")

    def count_batch(self, b):
        r = ctypes.c_uint64()
        _check(lib().kache_counter_count_batch(self.h, *b.args(), ctypes.byref(r)), "kache_counter_count_batch")
        return r.value

    def histogram(self, max_count):
        h = np.zeros(max_count + 1, np.uint64)
        _check(lib().kache_counter_histogram(self.h, max_count, h.ctypes.data), "kache_counter_histogram")
        return h

    def count_of(self, kmer):
        r = ctypes.c_uint64()
        kmer = kmer.encode() if isinstance(kmer, str) else kmer
        _check(lib().kache_counter_count_of(self.h, kmer, ctypes.byref(r)), "kache_counter_count_of")
        return r.value

    def size(self):
        r = ctypes.c_uint64()
        _check(lib().kache_counter_size(self.h, ctypes.byref(r)), "kache_counter_size")
        return r.value

    def table(self):
        """The counter's <31, u32, 22> table, for queries (owned by the counter)."""
        return Table.view(lib().kache_counter_table(self.h), 31, 22, 4)


def kernel_launches():
    return lib().kache_b200_kernel_launches()


ROOF_SEQ_READ, ROOF_RANDOM_READ, ROOF_RANDOM_UPDATE, ROOF_CHASE = 0, 1, 2, 3


def memory_roof(nbytes, kind, accesses=1 << 27):
    """(ms, rate) of one of the device's memory roofs (kache_b200_memory_roof)."""
    ms, rate = ctypes.c_double(), ctypes.c_double()
    _check(lib().kache_b200_memory_roof(nbytes, kind, accesses, ctypes.byref(ms), ctypes.byref(rate)), "kache_b200_memory_roof")
    return ms.value, rate.value


REQ_UPSERT, REQ_LOOKUP, REQ_COUNT = 0, 1, 2


class Server:
    """The request server over a table (kache_b200_server_*): submit from any thread, wait for each ticket."""

    def __init__(self, table, budget_bytes=0):
        h = _vp()
        _check(lib().kache_b200_server_new(table.h, budget_bytes, ctypes.byref(h)), "kache_b200_server_new")
        self.h, self.table, self.keep = h, table, {}

    def submit(self, kind, b, op=0, x=0, init=0, out0=None, out1=None, out2=None):
        t = ctypes.c_uint64()
        _check(lib().kache_b200_server_submit(self.h, kind, *b.args(), op, x, init, _p(out0), _p(out1), _p(out2), ctypes.byref(t)),
               "kache_b200_server_submit")
        self.keep[t.value] = (b, out0, out1, out2)    # The request's buffers live until it completes.
        return t.value

    def submit_dev(self, kind, d_bases, d_off, n, op=0, x=0, init=0, out0=None, out1=None, out2=None, keep=None):
        """A request resident in device memory (kache_b200_server_submit_dev): device addresses of the bases, the n + 1
        offsets and the outputs; `keep` holds whatever owns them until the request completes."""
        t = ctypes.c_uint64()
        _check(lib().kache_b200_server_submit_dev(self.h, kind, d_bases, d_off, n, op, x, init, out0, out1, out2, ctypes.byref(t)),
               "kache_b200_server_submit_dev")
        self.keep[t.value] = keep
        return t.value

    def wait(self, ticket):
        r, ms = ctypes.c_uint64(), ctypes.c_double()
        code = lib().kache_b200_server_wait(self.h, ticket, ctypes.byref(r), ctypes.byref(ms))
        self.keep.pop(ticket, None)
        _check(code, "kache_b200_server_wait")
        return r.value, ms.value

    def stats(self):
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().kache_b200_server_stats(self.h, ctypes.byref(a), ctypes.byref(b)), "kache_b200_server_stats")
        return a.value, b.value

    def close(self):
        if self.h:
            lib().kache_b200_server_free(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
